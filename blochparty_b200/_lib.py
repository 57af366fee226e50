"""ctypes binding of ``libblochparty_b200.so`` (the C ABI of ``include/blochparty_b200.h``).

The library is built in-tree (``blochparty_b200.build``). There is no fallback: if it cannot be loaded, or no
CUDA device is present, ``lib()`` raises, and nothing computes the simulation any other way.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_int64, c_void_p
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libblochparty_b200.so"

BP_SPAN_MAP, BP_SPAN_NET_MMA, BP_SPAN_NET_F32 = 0, 1, 2
BP_BOUND_ONLY = 128  # segment flag: RF only the bound pool feels


class BpSpan(ctypes.Structure):
    """``BpSpan`` of the C ABI: one replaced pulse occurrence for ``bp_forward_spans``."""

    _fields_ = [("kind", ctypes.c_int32), ("seg0", ctypes.c_int32), ("k_steps", ctypes.c_int32),
                ("phase", c_double), ("b0off", c_float), ("map", c_void_p), ("params", c_void_p),
                ("wtiles", c_void_p), ("T", c_double), ("gz", c_double), ("thickness", c_double), ("z0", c_double),
                ("dom_df", c_float), ("dom_b1", c_float), ("dom_z", c_float), ("counts", c_void_p)]



class BpNufft(ctypes.Structure):
    """``BpNufft`` of the C ABI: the NUFFT readout runs of ``bp_forward_nufft``."""

    _fields_ = [("run_of", c_void_p), ("base", c_void_p), ("frac", c_void_p), ("shift", c_void_p),
                ("decay", c_void_p), ("tile_cells", c_void_p), ("grid", c_void_p), ("G", c_int), ("W", c_int),
                ("M", c_int), ("beta", c_float)]


class BpPhysics(ctypes.Structure):
    """``BpPhysics`` of the C ABI: the bound pool and the field model of ``bp_forward_physics``."""

    _fields_ = [("mt", c_int), ("conc_mode", c_int), ("pool", c_void_p), ("bstate", c_void_p), ("rf_freq", c_void_p),
                ("line", c_void_p), ("conc", c_void_p), ("segq", c_void_p), ("wstates", c_void_p),
                ("wstate_stride", c_int)]


class BpForwardWorkspace(ctypes.Structure):
    """``BpForwardWorkspace`` of the C ABI: the forward's device buffer sizes in bytes."""

    _fields_ = [(f, c_int64) for f in ("state", "raw", "psi", "signal", "status", "total")]


class BpAdjointWorkspace(ctypes.Structure):
    """``BpAdjointWorkspace`` of the C ABI: the checkpointed adjoint's device buffer sizes in bytes."""

    _fields_ = [(f, c_int64) for f in ("checkpoints", "wstates", "replay_state", "gseg", "seg", "lam", "gs", "gc",
                                        "h", "total")]


BP_OK, BP_E_ARG, BP_E_ALIGN, BP_E_LAUNCH, BP_E_SIZE = 0, 1, 2, 3, 4
BP_MAX_COILS = 32
BP_SEG_MAX = 160
BP_ADJ_WIN = 32
BP_MMA_MAX_COILS = 8
BP_MLP_PARAMS = 10320
BP_MLP_INPUTS = 2
BP_MLP_OUTPUTS = 16
BP_MMA_SAMPLES = 64
BP_NOALLOC_SCRATCH_BYTES = 8 * 1024 * 1024
BP_PULSE_MAP_BYTES = 96
BP_NUF_MAX_TERMS = 6
BP_SEG_DT, BP_SEG_WX, BP_SEG_WY, BP_SEG_KX, BP_SEG_KY, BP_SEG_KZ, BP_SEG_BETA = (1 << k for k in range(7))
BP_SEG_ALL = 0x7F
BP_SPIN_NO_OFFSETS = 0x80  # with seg_mask: the position and dB0 rows of the spin gradients are not wanted
BP_SPIN_NONE = 0x100  # with seg_mask: no row of the spin gradients is wanted
ERRORS = {BP_E_ARG: "invalid argument", BP_E_ALIGN: "misaligned buffer", BP_E_LAUNCH: "CUDA launch failed",
          BP_E_SIZE: "size above the documented maximum"}
STATUS_BITS = {1: "a TMA copy of a segment block did not complete (bounded wait gave up)",
               2: "a window record was invalid (outside the sequence, the interval or the samples)",
               4: "the sweep from saved states met a window whose states were not saved"}

_P = c_void_p
# (restype, argtypes) of every exported entry point, as declared in include/blochparty_b200.h
SIGNATURES = {
    "bp_plan_windows": (c_int, [_P, c_int64, c_int, c_int, _P, _P, c_int64, _P]),
    "bp_forward_samp_max": (c_int, [c_int]),
    "bp_forward_grid": (c_int, [c_int, c_int]),
    "bp_forward_mma_grid": (c_int, [c_int]),
    "bp_forward": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P]),
    "bp_forward_spans": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, _P, c_int, _P, _P, _P, c_int, _P, _P]),
    "bp_signal_finish": (c_int, [_P, _P, c_int, c_int, _P, _P]),
    "bp_ffma_peak": (c_int, [_P, c_int, _P, _P]),
    "bp_ffma2_peak": (c_int, [_P, c_int, _P, _P]),
    "bp_mma_atiles_bytes": (c_int64, [c_int]),
    "bp_mma_atiles": (c_int, [_P, c_int, c_int, _P, _P]),
    "bp_forward_mma": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P, c_int, _P, _P]),
    "bp_adjoint_grid": (c_int, [c_int, c_int]),
    "bp_adjoint": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, c_int, c_int, _P, _P, c_int, _P, _P, _P,
                           _P, c_int, c_int, _P, _P]),
    "bp_adjoint_saved": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, c_int, c_int, _P, _P, _P, c_int, _P,
                                 c_int, _P, _P, c_int, c_int, _P, _P]),
    "bp_forward_saving": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P, _P, _P, c_int, _P, _P]),
    "bp_adjoint_physics": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, c_int, c_int, _P, _P, c_int, _P,
                                   _P, _P, _P, c_int, c_int, _P, _P, _P, _P]),
    "bp_seg_reduce": (c_int, [_P, c_int, c_int, c_int, _P, _P]),
    "bp_pulse_targets": (c_int, [_P, c_int, c_double, c_double, c_double, c_double, _P, c_int, _P, _P, _P]),
    "bp_mlp_grad_ctas": (c_int, [c_int]),
    "bp_mlp_grad": (c_int, [_P, _P, _P, c_int, c_float, c_float, _P, _P, _P]),
    "bp_mlp_reduce": (c_int, [_P, _P, c_int, c_float, _P, _P, _P]),
    "bp_adam": (c_int, [_P, _P, _P, _P, c_float, c_float, c_float, c_float, c_int, _P]),
    "bp_mlp_eval": (c_int, [_P, _P, c_int, _P, _P]),
    "bp_surrogate_pulse": (c_int, [_P, _P, c_int, _P, _P, c_int, c_int, c_double, c_double, c_double, c_double,
                                   c_double, c_float, c_float, c_float, c_float, _P, _P]),
    "bp_pulse_maps": (c_int, [_P, c_int, _P, _P, c_int, c_int, _P, _P]),
    "bp_pulse_apply": (c_int, [_P, c_int, _P, c_double, _P]),
    "bp_mlp_wtiles_bytes": (c_int, []),
    "bp_mlp_wtiles": (c_int, [_P, _P, _P]),
    "bp_surrogate_pulse_mma_grid": (c_int, [c_int]),
    "bp_surrogate_pulse_mma": (c_int, [_P, _P, c_int, _P, _P, _P, c_int, c_int, c_double, c_double, c_double,
                                       c_double, c_double, c_float, c_float, c_float, c_float, _P, _P, c_int, _P]),
    "bp_adjoint_noalloc": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, c_int, c_int, _P, _P, c_int, _P,
                                   _P, _P, _P, _P, _P]),
    "bp_forward_workspace_bytes": (c_int, [c_int, c_int64, c_int, _P]),
    "bp_forward_nufft": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P, c_int, _P, _P, _P]),
    "bp_forward_physics": (c_int, [_P, _P, c_int, c_int, _P, _P, _P, c_int, c_int, _P, _P, c_int, _P, _P, _P]),
    "bp_nufft_finish": (c_int, [_P, _P, c_int, c_int, c_int, c_int, c_int, _P, _P, _P]),
    "bp_adjoint_workspace_bytes": (c_int, [c_int, c_int64, c_int64, c_int, c_int, c_int, c_int, c_int, _P]),
}

_lib = None


def load_library(path: Path = LIB_PATH) -> ctypes.CDLL:
    """The library with every entry point's signature set (no GPU needed to load it)."""
    if not path.exists():
        raise RuntimeError(f"{path.name} is not built: run `python -m blochparty_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load_library()
    return _lib


def check(code: int, what: str) -> None:
    if code != BP_OK:
        raise RuntimeError(f"{what}: {ERRORS.get(code, f'error {code}')}")


def check_status(status: torch.Tensor, what: str) -> None:
    """Raise if a kernel OR-ed an error bit into the status word (call after synchronising)."""
    v = int(status.item())
    if v:
        bits = [msg for bit, msg in STATUS_BITS.items() if v & bit]
        raise RuntimeError(f"{what}: device status {v:#x}: {'; '.join(bits) or 'unknown'}")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def forward_workspace(n: int, n_adc: int, n_coils: int) -> BpForwardWorkspace:
    """The forward's buffer sizes (``bp_forward_workspace_bytes``; host arithmetic, no GPU)."""
    out = BpForwardWorkspace()
    check(lib().bp_forward_workspace_bytes(n, n_adc, n_coils, ctypes.byref(out)), "bp_forward_workspace_bytes")
    return out


def adjoint_workspace(n: int, n_segments: int, n_adc: int, n_coils: int, every: int, max_interval_windows: int,
                      grid: int, outer_every: int = 0) -> BpAdjointWorkspace:
    """The checkpointed adjoint's buffer sizes (``bp_adjoint_workspace_bytes``; host arithmetic, no GPU)."""
    out = BpAdjointWorkspace()
    check(lib().bp_adjoint_workspace_bytes(n, n_segments, n_adc, n_coils, every, max_interval_windows, grid,
                                           outer_every, ctypes.byref(out)), "bp_adjoint_workspace_bytes")
    return out
