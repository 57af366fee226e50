"""The NUFFT readout (``simulate(..., readout="nufft")``) on the GPU against the float64 oracle (its C restatement)
fed the engine's float32 inputs, and against the plain float32 readout: a 3D GRE with two echoes per TR, and
configuration 5's spins and sequence (4,096 seeded spins of the 128^3 head phantom, its first 256 TRs). Bars: 1e-6
relative L2 between the NUFFT and the plain readout (the spreading and the float32 tables; the float64 prototype of
the same arithmetic is at 1.1e-7); against float64, 1e-6 or 1.5 times the plain readout's own error, whichever is
larger (over 256 TRs the float32 state's rounding alone reaches 1.1e-6); 1e-5 on m (its state update is the plain
path's closed form)."""

import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import workloads
from oracle import bloch, fast
from test_configs_gpu import f32_inputs, l2, rel, subsample
from test_nufft_host import _case

pytestmark = pytest.mark.gpu


def _check(ph, seq, coils, label):
    ph32, c32 = f32_inputs(ph, coils)
    sig32, m32 = fast.simulate(bloch.case_from(ph32, seq, c32))
    r = bpb.simulate(ph, seq, coils, readout="nufft")
    plain = bpb.simulate(ph, seq, coils)
    e = {"nufft": l2(r.signal, sig32), "plain": l2(plain.signal, sig32), "nufft_vs_plain": l2(r.signal, plain.signal),
         "m": rel(r.m, m32)}
    print(f"\n{label}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert r.signal.shape == plain.signal.shape and r.signal.dtype == torch.complex64
    assert e["nufft_vs_plain"] < 1e-6 and e["nufft"] < max(1e-6, 1.5 * e["plain"]) and e["m"] < 1e-5
    return e


def test_two_echo_gre_against_the_oracle():
    inp, seq = _case()
    ph = bpb.Phantom(inp.pos, inp.pd, inp.t1, inp.t2, inp.db0)
    _check(ph, seq, inp.coils, "3D GRE 2 echoes, 6,000 random spins")


def test_config5_prefix_against_the_oracle():
    ph, seq, coils = workloads.gre3d_128_4echo()
    ph, coils = subsample(ph, coils, 4096, seed=6)
    seq = workloads.first_n_trs(seq, 256)
    _check(ph, seq, coils, f"config 5, 4,096 spins x {len(seq):,} segments")


def test_refusals():
    inp, seq = _case(n_spins=300)
    ph = bpb.Phantom(inp.pos, inp.pd, inp.t1, inp.t2, inp.db0)
    with pytest.raises(ValueError, match="too few spins"):
        bpb.simulate(ph, seq, inp.coils, readout="nufft")
    # with gradients the readout runs take the float32 readout, as blochparty's GPU engines do: the gradient is
    # the float32 readout's bit for bit (and the NUFFT's spin-count floor does not apply)
    grads = []
    for readout in ("nufft", "fp32"):
        t1 = inp.t1.clone().requires_grad_()
        r = bpb.simulate(bpb.Phantom(inp.pos, inp.pd, t1, inp.t2, inp.db0), seq, inp.coils, readout=readout)
        (g,) = torch.autograd.grad(r.signal.abs().pow(2).sum(), [t1])
        grads.append(g)
    assert torch.equal(grads[0], grads[1])
