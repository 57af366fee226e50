"""Spin sharding across GPUs: one process per GPU (``torch.distributed``, NCCL over NVLink on a GPU node), every
rank simulating a contiguous range of the spins on its own GPU.

Spins are independent and the signal is a linear sum over them (the reference's chunked engine rests on the same
fact, ``engines/chunked.py:1-14``), so the only exchange is one all-reduce of the float64 raw sums ``(A, 2 C)``
before the demodulation by exp(-i psi), plus, on request, an all-gather of the final magnetisation. Every rank takes
the same collective steps in the same order, error paths included: a rank whose local forward raised still joins
the reduction (with zeros) and the error is raised on every rank after it.
"""

from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist

from . import _lib, engine
from .api import Inputs, _device
from .types import Phantom, SimResult

F64 = torch.float64


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of rank ``rank``'s spins: contiguous ranges whose sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request: n={n}, world={world}, rank={rank}")
    return n * rank // world, n * (rank + 1) // world


def shard_phantom(phantom, coils, m_init, lo: int, hi: int):
    """The spins [lo, hi) of a phantom (every per-spin field), its coil rows and initial magnetisation."""
    cut = lambda t: None if t is None else t[lo:hi]
    ph = Phantom(phantom.pos[lo:hi], phantom.pd[lo:hi], phantom.t1[lo:hi], phantom.t2[lo:hi], phantom.db0[lo:hi],
                 b1=cut(getattr(phantom, "b1", None)))
    return ph, cut(coils), cut(m_init)


def gpu_local_forward(inp: Inputs):
    """The forward of this rank's spins on its GPU: (float64 raw sums (A, 2 C) on the device, a function turning
    the all-reduced sums into the (C, A) complex64 signal, final m (n, 3) float32 on the CPU)."""
    dev = _device()
    pk = engine.pack(inp, dev)
    samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
    if samp <= 0:
        raise ValueError(f"at most {_lib.BP_MAX_COILS} coils, got {pk.n_coils}")
    windows = engine.plan_windows(pk.flags, samp)
    wdev = torch.from_numpy(windows).to(dev)
    state = engine.initial_state(inp.pd, inp.m_init, dev)
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if pk.n:
        engine.run_forward(pk, state, wdev, 0, windows.shape[0], raw if pk.n_adc else None, status)
    torch.cuda.synchronize(dev)
    _lib.check_status(status, "bp_forward")
    return raw, lambda total: engine.finish_signal(pk, total).cpu(), engine.final_m(state)


def simulate(phantom, seq, coils=None, *, m_init=None, group=None, sharded: bool = True, gather_m: bool = True,
             local_forward: Callable | None = None) -> SimResult:
    """``simulate(phantom, seq, coils)`` over the ranks of ``group`` (default: the world).

    ``sharded`` True: every rank passes the whole phantom and simulates its ``shard_range``; False: every rank
    passes its own spins (weak scaling without the whole phantom on every host). The signal, the sum over all
    ranks' spins, is returned on every rank; m is all-gathered in rank order when ``gather_m`` (else this rank's
    spins only). ``local_forward(inputs) -> (raw, finish, m)`` computes one rank's part (default: the GPU forward);
    the raw sums of all ranks must have one shape and dtype float64.
    """
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n = len(phantom.pd)
    if coils is None:
        coils = torch.ones(n, 1, dtype=torch.complex64)
    if sharded:
        lo, hi = shard_range(n, world, rank)
        phantom, coils, m_init = shard_phantom(phantom, coils, m_init, lo, hi)
    inp = Inputs(phantom.pos, phantom.pd, phantom.t1, phantom.t2, phantom.db0, getattr(phantom, "b1", None), coils,
                 seq.dt, seq.rf, seq.grad, seq.adc_phase, getattr(seq, "b0_offset", None), list(seq.is_rf),
                 list(seq.adc), list(seq.spoil), m_init)
    fwd = local_forward or gpu_local_forward
    err = None
    try:
        raw, finish, m = fwd(inp)
    except Exception as e:  # joined below, so that no rank waits on a collective another one skipped
        err, raw, finish, m = e, None, None, None
    # the reduction's shape: every rank's raw has the same (A, 2 C); a failed rank contributes zeros
    failed = torch.tensor([1.0 if err is not None else 0.0], dtype=F64, device=_comm_device(group))
    shape = torch.zeros(2, dtype=F64, device=failed.device)
    if raw is not None:
        shape[0], shape[1] = raw.shape[0], raw.shape[1]
    dist.all_reduce(failed, group=group)
    dist.all_reduce(shape, op=dist.ReduceOp.MAX, group=group)
    total = raw.to(failed.device) if raw is not None else torch.zeros(int(shape[0]), int(shape[1]), dtype=F64,
                                                                        device=failed.device)
    dist.all_reduce(total, group=group)
    m_all = _gather_rows(m, world, group, failed.device) if gather_m else m
    if err is not None:
        raise err
    if float(failed) > 0:
        raise RuntimeError(f"{int(float(failed))} rank(s) failed in their local forward")
    return SimResult(finish(total.to(raw.device)), m_all)


def _comm_device(group) -> torch.device:
    backend = dist.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def _gather_rows(m: torch.Tensor | None, world: int, group, dev) -> torch.Tensor:
    """All-gather (n_r, 3) float32 blocks of different lengths, in rank order."""
    rows = torch.tensor([0 if m is None else m.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(rows) for _ in range(world)]
    dist.all_gather(sizes, rows, group=group)
    sizes = [int(s) for s in sizes]
    width = max(sizes) if sizes else 0
    mine = torch.zeros(width, 3, dtype=torch.float32, device=dev)
    if m is not None and m.shape[0]:
        mine[: m.shape[0]] = m.to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)]).cpu()
