"""Spin sharding across GPUs: one process per GPU (``torch.distributed``, NCCL over NVLink on a GPU node), every
rank simulating a contiguous range of the spins on its own GPU.

Spins are independent and the signal is a linear sum over them (the reference's chunked engine rests on the same
fact, ``engines/chunked.py:1-14``), so the forward's only exchange is one all-reduce of the float64 raw sums
``(A, 2 C)`` before the demodulation by exp(-i psi), plus, on request, an all-gather of the final magnetisation.

With gradients (any input requiring grad), the backward's exchanges are: a broadcast of dL/d(raw sums) from rank 0
(every rank calls backward on the same loss; rank 0's cotangent is the one used), the rank's own adjoint over its
spins, and one all-reduce of the sequence tensors' gradients (dt, RF, gradients, receiver phase, b0_offset: every
rank's spins contribute to them). The per-spin gradients stay on their rank: rank r's gradient of a sharded phantom
tensor holds its own spins' rows (zeros elsewhere), of an unsharded one its own spins.

Every rank takes the same collective steps in the same order, error paths included: a rank whose local forward or
backward raised still joins every collective (with zeros) and the error is raised on every rank after them.
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


def gpu_local_grad(inp: Inputs):
    """The differentiable forward of this rank's spins on its GPU (the checkpointed adjoint behind it): (float64 raw
    sums (A, 2 C) on the device, ``finish(total, adc_phase)`` demodulating the all-reduced sums differentiably, final
    m (n, 3) float32)."""
    from .adjoint import demodulate, simulate_raw

    raw, m = simulate_raw(inp, _device())
    return raw, lambda total, adc_phase: demodulate(total, adc_phase, inp.adc).cpu(), m


def simulate(phantom, seq, coils=None, *, m_init=None, group=None, sharded: bool = True, gather_m: bool = True,
             local_forward: Callable | None = None) -> SimResult:
    """``simulate(phantom, seq, coils)`` over the ranks of ``group`` (default: the world).

    ``sharded`` True: every rank passes the whole phantom and simulates its ``shard_range``; False: every rank
    passes its own spins (weak scaling without the whole phantom on every host). The signal, the sum over all
    ranks' spins, is returned on every rank; m is all-gathered in rank order when ``gather_m`` (else this rank's
    spins only). ``local_forward(inputs) -> (raw, finish, m)`` computes one rank's part (default: the GPU forward);
    the raw sums of all ranks must have one shape and dtype float64. With gradients (``torch.is_grad_enabled()`` and
    an input requiring grad; module docstring), ``local_forward`` is differentiable: its raw sums carry the graph to
    the inputs, and ``finish(total, adc_phase)`` is differentiable in both (default ``gpu_local_grad``).
    """
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n = len(phantom.pd)
    if coils is None:
        coils = torch.ones(n, 1, dtype=torch.complex64)
    from .api import requires_grad

    if torch.is_grad_enabled() and requires_grad(phantom, seq, coils, m_init):
        return _simulate_grad(phantom, seq, coils, m_init, group, sharded, gather_m, local_forward or gpu_local_grad)
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


def _gather_rows(m: torch.Tensor | None, world: int, group, dev, dtype=torch.float32) -> torch.Tensor:
    """All-gather (n_r, 3) blocks of different lengths (of one dtype on every rank), in rank order."""
    rows = torch.tensor([0 if m is None else m.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(rows) for _ in range(world)]
    dist.all_gather(sizes, rows, group=group)
    sizes = [int(s) for s in sizes]
    width = max(sizes) if sizes else 0
    mine = torch.zeros(width, 3, dtype=dtype, device=dev)
    if m is not None and m.shape[0]:
        mine[: m.shape[0]] = m.to(dev)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)]).cpu()


SPIN_FIELDS = ("pos", "pd", "t1", "t2", "db0", "b1", "coils", "m_init")
SEQ_FIELDS = ("dt", "rf", "grad", "adc_phase", "b0_offset")


def _group_src(group) -> int:
    """The global rank of the group's rank 0 (the source of the broadcast cotangent)."""
    return 0 if group is None else dist.get_global_rank(group, 0)


class _ShardedSimulate(torch.autograd.Function):
    """The sharded simulation with gradients (module docstring): forward = local differentiable forward + the
    all-reduce of the raw sums; backward = broadcast cotangent, local adjoint, all-reduce of the sequence gradients,
    every collective joined by every rank whatever failed."""

    @staticmethod
    def forward(ctx, opts, *tensors):
        group, lo, hi, local = opts["group"], opts["lo"], opts["hi"], opts["local"]
        nspin = len(SPIN_FIELDS)
        spin, seqt = tensors[:nspin], tensors[nspin:]
        leaf = lambda t, cut: None if t is None else (t.detach()[lo:hi] if cut else t.detach()).clone().requires_grad_(
            t.requires_grad)
        sl = [leaf(t, opts["sharded"]) for t in spin]
        ql = [leaf(t, False) for t in seqt]
        inp = Inputs(sl[0], sl[1], sl[2], sl[3], sl[4], sl[5], sl[6], ql[0], ql[1], ql[2], ql[3], ql[4],
                     opts["is_rf"], opts["adc"], opts["spoil"], sl[7])
        err = raw = finish = m = None
        try:
            with torch.enable_grad():
                raw, finish, m = local(inp)
        except Exception as e:  # joined below, so that no rank waits on a collective another one skipped
            err = e
        dev = _comm_device(group)
        failed = torch.tensor([1.0 if err is not None else 0.0], dtype=F64, device=dev)
        shape = torch.zeros(2, dtype=F64, device=dev)
        if raw is not None:
            shape[0], shape[1] = raw.shape[0], raw.shape[1]
        dist.all_reduce(failed, group=group)
        dist.all_reduce(shape, op=dist.ReduceOp.MAX, group=group)
        total = (raw.detach().to(dev).clone() if raw is not None
                 else torch.zeros(int(shape[0]), int(shape[1]), dtype=F64, device=dev))
        dist.all_reduce(total, group=group)
        m_det = None if m is None else m.detach()
        rows = torch.tensor([0 if m_det is None else m_det.shape[0]], dtype=torch.int64, device=dev)
        sizes = [torch.zeros_like(rows) for _ in range(dist.get_world_size(group))]
        dist.all_gather(sizes, rows, group=group)
        m_all = m_det
        if opts["gather_m"]:  # in float64 (exact for float32 blocks), returned in the local m's dtype
            m_all = _gather_rows(m_det, dist.get_world_size(group), group, dev, F64)
            m_all = m_all.to(m_det.dtype) if m_det is not None else m_all
        if err is not None:
            raise err
        if float(failed) > 0:
            raise RuntimeError(f"{int(float(failed))} rank(s) failed in their local forward")
        total_leaf = total.to(raw.device).requires_grad_()
        with torch.enable_grad():
            sig = finish(total_leaf, ql[3])
        ctx.save = (sl, ql, raw, m, total_leaf, sig, group, opts)
        ctx.m_off = sum(int(x) for x in sizes[: dist.get_rank(group)]) if opts["gather_m"] else 0
        ctx.set_materialize_grads(False)
        return sig.detach(), m_all

    @staticmethod
    def backward(ctx, g_sig, g_m):
        sl, ql, raw, m, total_leaf, sig, group, opts = ctx.save
        dev = _comm_device(group)
        # the cotangent of the signal: rank 0's, on every rank
        g = torch.zeros_like(sig.detach()) if g_sig is None else g_sig.to(sig.dtype)
        gb = torch.view_as_real(g.contiguous()).to(dev) if g.is_complex() else g.to(dev)
        gb = gb.contiguous().clone()
        dist.broadcast(gb, src=_group_src(group), group=group)
        g = torch.view_as_complex(gb).to(sig.device) if g.is_complex() else gb.to(sig.device)
        err = None
        local_grads = [None] * (len(sl) + len(ql))
        fin_seq = None
        try:
            fin_in = [total_leaf] + ([ql[3]] if ql[3] is not None and ql[3].requires_grad else [])
            fg = torch.autograd.grad(sig, fin_in, g, allow_unused=True, retain_graph=False)
            g_total = fg[0]
            fin_seq = fg[1] if len(fg) > 1 else None
            outs, gouts = [raw], [g_total.to(raw.dtype)]
            if g_m is not None and m is not None and m.requires_grad:
                outs.append(m)
                gouts.append(g_m[ctx.m_off: ctx.m_off + m.shape[0]].to(m.dtype).to(m.device))
            leaves = [t for t in sl + ql if t is not None and t.requires_grad]
            got = torch.autograd.grad(outs, leaves, gouts, allow_unused=True) if leaves else []
            it = iter(got)
            local_grads = [next(it) if (t is not None and t.requires_grad) else None for t in sl + ql]
        except Exception as e:  # joined below
            err = e
        # sequence gradients: summed over ranks (one flat float64 buffer of a layout every rank knows)
        failed = torch.tensor([1.0 if err is not None else 0.0], dtype=F64, device=dev)
        dist.all_reduce(failed, group=group)
        sizes = [0 if t is None else t.numel() for t in ql]
        flat = torch.zeros(sum(sizes), dtype=F64, device=dev)
        off = 0
        for t, gq, k in zip(ql, local_grads[len(sl):], sizes):
            if gq is not None:
                flat[off:off + k] = gq.detach().reshape(-1).to(F64).to(dev)
            off += k
        dist.all_reduce(flat, group=group)
        if err is not None:
            raise err
        if float(failed) > 0:
            raise RuntimeError(f"{int(float(failed))} rank(s) failed in their local backward")
        out = list(local_grads[: len(sl)])
        off = 0
        for j, (t, k) in enumerate(zip(ql, sizes)):
            gq = None
            if t is not None and t.requires_grad:
                gq = flat[off:off + k].reshape(t.shape).to(t.dtype).to(t.device)
                if j == 3 and fin_seq is not None:
                    gq = gq + fin_seq.to(gq.dtype).to(gq.device)
            out.append(gq)
            off += k
        # per-spin gradients of sharded inputs: this rank's rows in a full-size zero tensor
        lo, hi, n = opts["lo"], opts["hi"], opts["n"]
        full = []
        for gt in out[: len(sl)]:
            if gt is None or not opts["sharded"]:
                full.append(gt)
                continue
            z = torch.zeros((n,) + tuple(gt.shape[1:]), dtype=gt.dtype, device=gt.device)
            z[lo:hi] = gt
            full.append(z)
        return (None, *full, *out[len(sl):])


def _simulate_grad(phantom, seq, coils, m_init, group, sharded, gather_m, local):
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n = len(phantom.pd)
    lo, hi = shard_range(n, world, rank) if sharded else (0, n)
    opts = {"group": group, "lo": lo, "hi": hi, "n": n, "sharded": sharded, "gather_m": gather_m, "local": local,
            "is_rf": list(seq.is_rf), "adc": list(seq.adc), "spoil": list(seq.spoil)}
    spin = (phantom.pos, phantom.pd, phantom.t1, phantom.t2, phantom.db0, getattr(phantom, "b1", None), coils, m_init)
    seqt = (seq.dt, seq.rf, seq.grad, seq.adc_phase, getattr(seq, "b0_offset", None))
    sig, m = _ShardedSimulate.apply(opts, *spin, *seqt)
    return SimResult(sig, m)
