"""The forward simulation with the coil readout on the tensor cores (``simulate(..., readout="bf16x3")``).

The propagation is the float32 kernel's; the coil sum of every 16 ADC samples over a 128-spin tile is a tcgen05
matrix product in split bfloat16 (high and low parts of both the coil sensitivities and the magnetization,
three products, float32 accumulation in tensor memory), summed over each CTA's tiles and added to the float64
signal per window (``bp_forward_mma``). At most ``BP_MMA_MAX_COILS`` = 8 coils.
"""

from __future__ import annotations

import torch

from . import _lib, engine
from ._lib import ptr

F32, F64 = torch.float32, torch.float64


class MmaBuffers:
    """The tensor-core operand blocks of a packed case (``bp_mma_atiles``) and its 64-sample windows."""

    def __init__(self, pk: engine.Packed):
        if pk.n_coils > _lib.BP_MMA_MAX_COILS:
            raise ValueError(f"readout='bf16x3' supports at most {_lib.BP_MMA_MAX_COILS} coils, got {pk.n_coils}")
        lib = _lib.lib()
        nbytes = lib.bp_mma_atiles_bytes(pk.n)
        self.atiles = torch.empty(nbytes, dtype=torch.uint8, device=pk.device)
        _lib.check(lib.bp_mma_atiles(ptr(pk.sens), pk.n, pk.n_coils, ptr(self.atiles), _lib.stream_ptr()),
                   "bp_mma_atiles")
        self.windows = engine.plan_windows(pk.flags, _lib.BP_MMA_SAMPLES)
        self.windows_dev = torch.from_numpy(self.windows).to(pk.device)


def run_forward_mma(pk: engine.Packed, mb: MmaBuffers, state: torch.Tensor, raw: torch.Tensor | None,
                    status: torch.Tensor, w_begin: int = 0, w_end: int | None = None, max_ctas: int = 0) -> None:
    w_end = mb.windows.shape[0] if w_end is None else w_end
    code = _lib.lib().bp_forward_mma(ptr(pk.spins), ptr(mb.atiles), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                     ptr(mb.windows_dev), w_begin, w_end, ptr(state), ptr(raw), max_ctas, ptr(status),
                                     _lib.stream_ptr())
    _lib.check(code, "bp_forward_mma")


def forward_bf16x3(inp, device, max_ctas: int = 0):
    """Signal (C, A) complex64 and m (N, 3) float32 on the CPU, readout on the tensor cores."""
    pk = engine.pack(inp, device)
    mb = MmaBuffers(pk)
    state = engine.initial_state(inp.pd, inp.m_init, device)
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    run_forward_mma(pk, mb, state, raw if pk.n_adc else None, status, max_ctas=max_ctas)
    sig = engine.finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward_mma")
    return sig.cpu(), engine.final_m(state)
