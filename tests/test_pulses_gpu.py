"""Reused pulses on the GPU (``simulate(..., pulses="reuse")``): the same signal and magnetization as stepping
every pulse (within 1e-5 relative L2: the maps are composed and applied in float64, while the stepped pulse
rounds its per-step rotation factors to float32, so reuse is the closer of the two to float64) and within 1e-5 of
the float64 oracle fed the engine's float32 spin inputs, on an RF-spoiled 3D GRE with sub-voxel spins, the
3-slice TSE and the reference-core golden cases; a memory cap that leaves pulses stepped; with gradients the pulses are stepped."""

from dataclasses import replace

import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import pulses, workloads
from blochparty_b200.api import Inputs
from oracle import bloch
from tests import golden_cases

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = a.to(torch.complex128), b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def f32_spins(ph):
    """The phantom with the engine's float32 spin inputs (positions, PD, rates, dB0) back in float64."""
    r = lambda t: t.to(torch.float32).to(torch.float64)
    return bpb.Phantom(r(ph.pos), r(ph.pd), 1.0 / r(1.0 / ph.t1), 1.0 / r(1.0 / ph.t2), r(ph.db0))


@pytest.mark.parametrize("name", ["gre3d_16", "tse_32"])
def test_reuse_matches_stepping_and_the_oracle(name):
    ph, seq, coils = workloads.gre3d_64(16) if name == "gre3d_16" else workloads.tse_3slice_128(32)
    step = bpb.simulate(ph, seq, coils)
    reuse = bpb.simulate(ph, seq, coils, pulses="reuse")
    sig64, _ = bloch.simulate(bloch.case_from(ph, seq, coils))
    sig64q, _ = bloch.simulate(bloch.case_from(f32_spins(ph), seq, coils))
    e_step = rel_l2(reuse.signal, step.signal)
    e_m = float((reuse.m.double() - step.m.double()).abs().max())
    print(f"\n{name}: reuse vs stepping {e_step:.1e} (m {e_m:.1e}); vs float64 with float32 spin inputs: reuse "
          f"{rel_l2(reuse.signal, sig64q):.1e}, stepping {rel_l2(step.signal, sig64q):.1e}; vs float64: reuse "
          f"{rel_l2(reuse.signal, sig64):.1e}, stepping {rel_l2(step.signal, sig64):.1e}")
    assert e_step < 1e-5 and e_m < 1e-5
    assert rel_l2(reuse.signal, sig64q) < 1e-5
    assert rel_l2(reuse.signal, sig64q) <= rel_l2(step.signal, sig64q) * 1.05


@pytest.mark.parametrize("name", ["busy", "sinc3d", "gre16"])
def test_reuse_on_golden_cases(name):
    case, sig, m, _ = golden_cases.load(name)
    ph, seq, coils, m_init = golden_cases.objects(case)
    r = bpb.simulate(ph, seq, coils, m_init=m_init, pulses="reuse")
    assert rel_l2(r.signal, sig) < 1e-5
    assert float((r.m.double() - m).abs().max()) < 1e-5


def test_memory_cap_leaves_pulses_stepped():
    ph, seq, coils = workloads.tse_3slice_128(32)
    inp = Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase, None,
                 list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    dev = torch.device("cuda", 0)
    full, _ = pulses.forward_with_reuse(inp, dev)
    two, _ = pulses.forward_with_reuse(inp, dev, memory=2 * 96 * len(ph.pd))  # the two most-used pulses only
    none, _ = pulses.forward_with_reuse(inp, dev, memory=0)
    step = bpb.simulate(ph, seq, coils).signal
    assert torch.equal(none, step)  # nothing reused: the stepped forward itself
    for sig in (full, two):
        assert rel_l2(sig, step) < 1e-5


def test_reuse_with_gradients_steps_the_pulses():
    """Reuse is a forward-only acceleration: with gradients the pulses are stepped (as blochparty's GPU engines
    do), so the gradient is the stepped run's bit for bit."""
    ph, seq, coils = workloads.gre3d_64(8)
    grads = []
    for pulses in ("reuse", "step"):
        t1 = ph.t1.clone().requires_grad_()
        r = bpb.simulate(replace(ph, t1=t1), seq, coils, pulses=pulses)
        (g,) = torch.autograd.grad(r.signal.abs().pow(2).sum(), [t1])
        grads.append(g)
    assert torch.equal(grads[0], grads[1])
