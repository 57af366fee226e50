"""Reused pulses on the GPU (``simulate(..., pulses="reuse")``): the same signal and magnetization as stepping
every pulse (within 2e-6 relative L2; the maps are composed and applied in float64, the stepped state is the
compensated float32 one) and within 1e-5 of the float64 oracle, on an RF-spoiled 3D GRE, the 3-slice TSE and the
reference-core golden cases; a memory cap that leaves pulses stepped; forward only."""

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


@pytest.mark.parametrize("name", ["gre3d_16", "tse_32"])
def test_reuse_matches_stepping_and_the_oracle(name):
    ph, seq, coils = workloads.gre3d_64(16) if name == "gre3d_16" else workloads.tse_3slice_128(32)
    step = bpb.simulate(ph, seq, coils)
    reuse = bpb.simulate(ph, seq, coils, pulses="reuse")
    sig64, m64 = bloch.simulate(bloch.case_from(ph, seq, coils))
    e_step, e_reuse = rel_l2(reuse.signal, step.signal), rel_l2(reuse.signal, sig64)
    e_m = float((reuse.m.double() - step.m.double()).abs().max())
    print(f"\n{name}: reuse vs stepping {e_step:.1e} (m {e_m:.1e}), vs float64 {e_reuse:.1e}, "
          f"stepping vs float64 {rel_l2(step.signal, sig64):.1e}")
    assert e_step < 2e-6 and e_m < 2e-6
    assert e_reuse < 1e-5


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
    for sig in (full, two, none):
        assert rel_l2(sig, step) < 2e-6


def test_reuse_is_forward_only():
    ph, seq, coils = workloads.gre3d_64(8)
    t1 = ph.t1.clone().requires_grad_()
    ph.t1 = t1
    with pytest.raises(ValueError, match="forward only"):
        bpb.simulate(ph, seq, coils, pulses="reuse")
