"""Spin sharding over ranks (``blochparty_b200.parallel``) with world size 2 on the CPU (gloo), the per-rank
forward being the float64 oracle: the sharded signal and the gathered magnetisation equal the single-process ones;
a rank whose forward fails makes every rank raise, none waiting on a collective. The GPU forward inside each rank is
the one the single-GPU tests cover."""

import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from blochparty_b200 import parallel
from oracle import bloch
from tests import golden_cases

F64 = torch.float64


def test_shard_ranges_partition_the_spins():
    for n in (0, 1, 7, 4096, 1000003):
        for world in (1, 2, 3, 8):
            ranges = [parallel.shard_range(n, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        parallel.shard_range(10, 2, 2)


def _oracle_forward(inp):
    """One rank's part through the oracle: its demodulated float64 signal as (A, 2 C) sums (the demodulation is
    linear, so summing demodulated parts equals demodulating the summed raw sums)."""
    case = bloch.Case(**{f: getattr(inp, f) for f in bloch.Case.__dataclass_fields__ if hasattr(inp, f)})
    sig, m = bloch.simulate(case)
    raw = torch.view_as_real(sig.T.contiguous()).reshape(sig.shape[1], -1).contiguous()
    finish = lambda total: torch.view_as_complex(total.reshape(total.shape[0], -1, 2).contiguous()).T.contiguous()
    return raw, finish, m.to(torch.float32)


def _oracle_grad_forward(inp):
    """One rank's differentiable part through the oracle (autograd through its float64 arithmetic): the demodulated
    signal as (A, 2 C) sums; ``finish`` turns the summed sums back into the (C, A) signal."""
    case = bloch.Case(**{f: getattr(inp, f) for f in bloch.Case.__dataclass_fields__ if hasattr(inp, f)})
    sig, m = bloch.simulate(case)
    raw = torch.view_as_real(sig.T.contiguous()).reshape(sig.shape[1], -1)
    finish = lambda total, adc_phase: torch.view_as_complex(total.reshape(total.shape[0], -1, 2).contiguous()).T
    return raw, finish, m


class _FailInBackward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        raise ValueError("rank 1's backward failed")


def _failing_grad_forward(inp):
    raw, finish, m = _oracle_grad_forward(inp)
    return (_FailInBackward.apply(raw) if dist.get_rank() == 1 else raw), finish, m


GRAD_NAMES = ("t1", "pd", "db0", "coils", "rf", "dt", "adc_phase", "m_init")


def _grad_leaves(case):
    """The golden case's inputs, the ones in GRAD_NAMES as leaves requiring grad."""
    from dataclasses import replace

    return replace(case, **{k: getattr(case, k).detach().clone().requires_grad_() for k in GRAD_NAMES})


def _grad_loss(sig, m, z):
    wr, wi, wm = (torch.from_numpy(z[k]).to(F64) for k in ("w_re", "w_im", "w_m"))
    return (sig.real * wr).sum() + (sig.imag * wi).sum() + (m.to(F64) * wm).sum()


def _failing_forward(inp):
    if dist.get_rank() == 1:
        raise ValueError("rank 1's forward failed")
    return _oracle_forward(inp)


def _by_value(x, back=False):
    """Tensors as numpy arrays (and back): a queue then carries them by value, not as shared memory whose file
    descriptor the receiver could only open while the sending process still runs."""
    if isinstance(x, dict):
        return {k: _by_value(v, back) for k, v in x.items()}
    if isinstance(x, tuple):
        return tuple(_by_value(v, back) for v in x)
    if back and isinstance(x, np.ndarray):
        return torch.from_numpy(x)
    if not back and isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy().copy()
    return x


def _worker(rank, world, port, mode, out):
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    put = out.put
    out = type("Out", (), {"put": staticmethod(lambda item: put(_by_value(item)))})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        case, _, _, _ = golden_cases.load("busy")
        ph, seq, coils, m_init = golden_cases.objects(case)
        if mode == "sharded":
            r = parallel.simulate(ph, seq, coils, m_init=m_init, local_forward=_oracle_forward)
            out.put((rank, "ok", r.signal, r.m))
        elif mode == "own_spins":
            lo, hi = parallel.shard_range(len(ph.pd), world, rank)
            mine, c, m0 = parallel.shard_phantom(ph, coils, m_init, lo, hi)
            r = parallel.simulate(mine, seq, c, m_init=m0, sharded=False, local_forward=_oracle_forward)
            out.put((rank, "ok", r.signal, r.m))
        elif mode in ("grad", "grad_fail"):
            case, _, _, z = golden_cases.load("grad_busy")
            c = _grad_leaves(case)
            ph, seq, coils, m_init = golden_cases.objects(c)
            fwd = _oracle_grad_forward if mode == "grad" else _failing_grad_forward
            try:
                r = parallel.simulate(ph, seq, coils, m_init=m_init, local_forward=fwd)
                _grad_loss(r.signal, r.m, z).backward()
                out.put((rank, "ok", {k: getattr(c, k).grad.detach().clone() for k in GRAD_NAMES}, r.signal.detach()))
            except Exception as e:
                out.put((rank, type(e).__name__, str(e), None))
        else:
            try:
                parallel.simulate(ph, seq, coils, m_init=m_init, local_forward=_failing_forward)
                out.put((rank, "no error", None, None))
            except Exception as e:
                out.put((rank, type(e).__name__, str(e), None))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [_by_value(out.get(timeout=120), back=True) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res, key=lambda r: r[0])


@pytest.mark.parametrize("mode", ["sharded", "own_spins"])
def test_two_ranks_equal_one_process(mode):
    case, _, _, _ = golden_cases.load("busy")
    sig, m = bloch.simulate(case)
    for rank, status, s, mm in _run(mode):
        assert status == "ok"
        assert float((s - sig).abs().max() / sig.abs().max()) < 1e-12
        assert torch.equal(mm, m.to(torch.float32))  # gathered in rank order: every spin


def test_a_failed_rank_fails_every_rank():
    res = _run("fail")
    assert res[0][1] == "RuntimeError" and "1 rank(s) failed" in res[0][2]
    assert res[1][1] == "ValueError" and "rank 1" in res[1][2]


SEQ = ("rf", "dt", "adc_phase")


def test_two_ranks_gradients_equal_one_process():
    """The sharded simulation with gradients (world size 2, each rank's part through the oracle's autograd): the
    sequence tensors' gradients (all-reduced) are the single process's on every rank; the per-spin gradients are
    local, and their sum over the ranks is the single process's."""
    case, _, _, z = golden_cases.load("grad_busy")
    c = _grad_leaves(case)
    sig, m = bloch.simulate(c)
    _grad_loss(sig, m, z).backward()
    ref = {k: getattr(c, k).grad for k in GRAD_NAMES}
    res = _run("grad")
    assert all(r[1] == "ok" for r in res), res
    for k in GRAD_NAMES:
        if k in SEQ:
            for r in res:
                assert float((r[2][k] - ref[k]).abs().max() / ref[k].abs().max()) < 1e-12, k
        else:
            tot = res[0][2][k] + res[1][2][k]
            assert float((tot - ref[k]).abs().max() / ref[k].abs().max()) < 1e-12, (k, float((tot - ref[k]).abs().max() / ref[k].abs().max()))
            lo, hi = parallel.shard_range(len(case.pd), 2, 1)
            assert float(res[0][2][k][lo:hi].abs().max()) == 0.0  # rank 0 holds only its own rows


def test_a_failed_backward_fails_every_rank():
    res = _run("grad_fail")
    assert res[0][1] == "RuntimeError" and "failed in their local backward" in res[0][2]
    assert res[1][1] == "ValueError" and "rank 1" in res[1][2]
