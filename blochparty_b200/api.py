"""``simulate``: the drop-in entry point of the b200 engine.

Keeps the signature and semantics of blochparty's ``simulate`` (``engines/__init__.py:60-144``) as its GPU
engines implement them (``engines/gpu/__init__.py:54-96``, ``engines/gpu/cuda/__init__.py:93-132``):

* inputs of any dtype are cast; the simulation computes in float32 (float64 where stated);
* the result comes back on the CPU: ``signal`` (C, n_adc) complex64, ``m`` (N, 3) float32;
* gradients come from the hand-written adjoint whenever ``torch.is_grad_enabled()`` and an input requires grad;
* unsupported features raise ``NotImplementedError`` (``capabilities``); another engine's options ``TypeError``.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import torch
from torch import Tensor

from . import capabilities, engine
from .types import SimResult

ENGINES = ("b200", "gpu", "cuda")  # "gpu" and "cuda" name this engine too, so a caller's engine= still works
# blochparty's GPU-engine options (engines/gpu/cuda/__init__.py:93-110), accepted as they are: ``readouts``
# "direct" / "nufft" is ``readout`` "fp32" / "nufft"; ``chunk`` and ``group`` (dispatch chunking and threadgroup
# size), ``mma`` (the sensitivity layout; both of its kernels reduce the coils on the CUDA cores) and
# ``nufft_width`` / ``nufft_terms`` (the NUFFT's kernel width and decay terms, defaults 6 and 3) tune the
# reference's kernels and change nothing here: the persistent kernels have no dispatch chunks, and the NUFFT here
# takes width 8 and its terms from a 5e-8 bound on the decay's interpolation (at least as accurate).
REFERENCE_GPU_OPTIONS = ("chunk", "group", "mma", "readouts", "nufft_width", "nufft_terms")
OPTIONS = ("readout", "pulses", "surrogate", "surrogate_inference", "max_ctas") + REFERENCE_GPU_OPTIONS
PULSES = ("step", "reuse", "surrogate")
READOUTS = ("fp32", "bf16x3", "nufft")


@dataclass
class Inputs:
    """One case's tensors as the engine reads them (coils complex (N, C), never None)."""

    pos: Tensor
    pd: Tensor
    t1: Tensor
    t2: Tensor
    db0: Tensor
    b1: Tensor | None
    coils: Tensor
    dt: Tensor
    rf: Tensor
    grad: Tensor
    adc_phase: Tensor
    b0_offset: Tensor | None
    is_rf: list
    adc: list
    spoil: list
    m_init: Tensor | None


def requires_grad(*objs) -> bool:
    """Whether any tensor in ``objs`` (tensors, dataclasses, tuples) requires grad (as blochparty
    ``engines/gpu/__init__.py:39-51``)."""
    for o in objs:
        if isinstance(o, Tensor):
            if o.requires_grad:
                return True
        elif dataclasses.is_dataclass(o) and not isinstance(o, type):
            if requires_grad(*(getattr(o, f.name) for f in dataclasses.fields(o))):
                return True
        elif isinstance(o, tuple) and requires_grad(*o):
            return True
    return False


def _device(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("engine='b200' needs a CUDA device (an NVIDIA B200, sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)


def simulate(phantom, seq, coils: Tensor | None = None, *, m_init: Tensor | None = None,
             checkpoint_every: int | None = None, merge_free_runs: bool = True, scanner=None, seed: int = 0,
             maps=None, engine: str = "b200", **options) -> SimResult:
    """Run ``seq`` on ``phantom`` on the GPU (blochparty ``simulate``'s arguments; see the module docstring).

    coils: (N, C) complex receive sensitivities (default: one uniform coil), C <= 32.
    m_init: (N, 3) starting magnetization (default: equilibrium, Mz = PD).
    checkpoint_every: with gradients, the adjoint stores the state every this many segments (a multiple of 32);
        default about sqrt(segments).
    options: ``readout`` "fp32" (default: float32 coil products reduced by warp shuffles), "bf16x3" (the coil
        contraction on the tensor cores in split bfloat16 with float32 accumulation) or "nufft" (readout runs
        through a nonuniform FFT: at least a few thousand spins; with gradients the float32 readout is taken, as
        blochparty's GPU engines do); ``pulses`` "step" (default), "reuse" (every recurring pulse through its exact
        per-spin map; stepped with gradients) or "surrogate"
        (shaped pulses through a trained ``surrogate``), whose ``surrogate_inference`` is "mma" (default: the
        hidden 64 x 64 layers on the tensor cores) or "fp32"; ``max_ctas`` caps the grid.
    """
    if engine not in ENGINES:
        raise ValueError(f"engine must be one of {ENGINES}, not {engine!r}")
    if unknown := sorted(set(options) - set(OPTIONS)):
        hint = " (an option of blochparty's chunked engine)" if unknown == ["spin_chunk"] else ""
        raise TypeError(f"simulate(engine={engine!r}) got unexpected keyword argument(s) {', '.join(unknown)}{hint}")
    options = _reference_options(dict(options))
    if not merge_free_runs:
        raise ValueError(f"merge_free_runs=False is the core's segment-by-segment stepping, not engine={engine!r}'s")
    readout = options.get("readout", "fp32")
    if readout not in READOUTS:
        raise ValueError(f"readout must be one of {READOUTS}, not {readout!r}")
    pulses = options.get("pulses", "step")
    if pulses not in PULSES:
        raise ValueError(f"pulses must be one of {PULSES}, not {pulses!r}")
    if pulses == "reuse" and readout != "fp32":
        raise ValueError("pulses='reuse' takes the float32 readout (readout='fp32')")
    if pulses == "surrogate" and readout == "nufft":
        raise ValueError("pulses='surrogate' takes readout='fp32' or 'bf16x3'")
    n = len(phantom.pd)
    if coils is not None and (coils.dim() != 2 or coils.shape[0] != n):
        raise ValueError(f"coils must be (N, C) = ({n}, C), got {tuple(coils.shape)}")
    bound = getattr(phantom, "bound", None)
    if m_init is not None and tuple(m_init.shape) == (n, 4) and bound is None:
        raise ValueError("m_init has a bound-pool column but the phantom has no bound pool")
    if m_init is not None and tuple(m_init.shape) not in ((n, 3), (n, 4)):
        raise ValueError(f"m_init must be (N, 3) = ({n}, 3) (or (N, 4) with a bound pool), got {tuple(m_init.shape)}")
    if checkpoint_every is not None and checkpoint_every < 1:
        raise ValueError(f"checkpoint_every must be positive, got {checkpoint_every}")
    grad = torch.is_grad_enabled() and requires_grad(phantom, seq, coils, m_init, scanner)
    capabilities.check(capabilities.features(phantom, seq, m_init, scanner, maps), grad=grad)
    dev = _device()
    if coils is None:
        coils = torch.ones(n, 1, dtype=torch.complex64)
    inp = Inputs(phantom.pos, phantom.pd, phantom.t1, phantom.t2, phantom.db0, getattr(phantom, "b1", None), coils,
                 seq.dt, seq.rf, seq.grad, seq.adc_phase, getattr(seq, "b0_offset", None), list(seq.is_rf),
                 list(seq.adc), list(seq.spoil), m_init)
    if grad:
        from .adjoint import simulate_grad

        return simulate_grad(inp, dev, checkpoint_every, options, scanner)
    bound_only = getattr(seq, "bound_only", None)
    if bound is not None or scanner is not None or (bound_only is not None and any(bound_only)):
        if options.get("readout", "fp32") != "fp32" or options.get("pulses", "step") != "step":
            raise ValueError("a bound pool, bound-only RF or a scanner field model takes readout='fp32' and "
                             "pulses='step'")
        from .physics import forward_physics

        with torch.no_grad():
            sig, m, m_bound = forward_physics(inp, dev, bound, scanner, bound_only, getattr(seq, "rf_freq", None),
                                              options.get("max_ctas", 0))
        return SimResult(sig, m, m_bound)
    with torch.no_grad():
        sig, m = _forward(inp, dev, options)
    return SimResult(sig, m)


def _reference_options(options: dict) -> dict:
    """blochparty's GPU-engine options mapped onto this engine's (``REFERENCE_GPU_OPTIONS``)."""
    if "readouts" in options:
        ro = options.pop("readouts")
        if ro not in ("direct", "nufft"):
            raise ValueError(f"readouts must be 'direct' or 'nufft', not {ro!r}")
        mapped = "fp32" if ro == "direct" else "nufft"
        if options.get("readout", mapped) != mapped:
            raise ValueError(f"readouts={ro!r} and readout={options['readout']!r} disagree")
        options["readout"] = mapped
    for k in ("chunk", "group", "nufft_width", "nufft_terms"):
        v = options.pop(k, None)
        if v is not None and (not isinstance(v, int) or v < 1):
            raise ValueError(f"{k} must be a positive int, got {v!r}")
    options.pop("mma", None)
    return options


def _forward(inp: Inputs, dev, options):
    if options.get("pulses", "step") == "reuse":
        from .pulses import forward_with_reuse

        return forward_with_reuse(inp, dev, options.get("max_ctas", 0))
    if options.get("pulses", "step") == "surrogate":
        from .surrogate import forward_with_surrogate

        return forward_with_surrogate(inp, dev, options)
    if options.get("readout", "fp32") == "bf16x3":
        from .readout_mma import forward_bf16x3

        return forward_bf16x3(inp, dev, options.get("max_ctas", 0))
    if options.get("readout", "fp32") == "nufft":
        from .nufft import forward_nufft

        return forward_nufft(inp, dev, options.get("max_ctas", 0))
    return engine.forward(inp, dev, options.get("max_ctas", 0))
