"""The split-bfloat16 tensor-core readout (``readout="bf16x3"``) on the GPU.

The state propagation is the float32 kernel's, so the final magnetization matches as tightly; the signal carries
the split-bfloat16 representation error (~2^-17 relative per operand, ~2^-18 for the dropped low x low product),
so its bar is 3e-5 relative L2 against the float64 oracle and the reference core's golden outputs (the float32
readout's bar is 1e-5), and 1e-4 max-norm.
"""

import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import workloads
from golden_cases import NAMES, load, objects
from oracle import bloch

pytestmark = pytest.mark.gpu
F64 = torch.float64
L2, MX, MM = 3e-5, 1e-4, 1e-5


def rel_l2(a, b):
    a = a.to(b.dtype)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b).clamp_min(1e-300))


def rel_max(a, b):
    a = a.to(b.dtype)
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300)) if b.numel() else 0.0


def check(r, sig, m):
    assert r.signal.shape == sig.shape and r.signal.dtype == torch.complex64
    e = (rel_l2(r.signal, sig), rel_max(r.signal, sig), rel_max(r.m, m))
    assert e[0] < L2 and e[1] < MX and e[2] < MM, e
    return e


@pytest.mark.parametrize("name", NAMES)
def test_bf16x3_matches_reference_core_golden(name):
    case, sig, m, _ = load(name)
    ph, seq, coils, m_init = objects(case)
    check(bpb.simulate(ph, seq, coils, m_init=m_init, readout="bf16x3"), sig, m)


def test_bf16x3_gre2d_64_against_oracle_and_fp32():
    ph, seq, coils = workloads.gre2d_64()
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils))
    r = bpb.simulate(ph, seq, coils, readout="bf16x3")
    e = check(r, sig, m)
    f = bpb.simulate(ph, seq, coils)
    print("\ngre2d_64 bf16x3 vs float64: rel L2 %.2e, rel max %.2e, m %.2e; fp32 readout: rel L2 %.2e" % (
        *e, rel_l2(f.signal, sig)))
    assert torch.equal(r.m, f.m)  # the same propagation


def test_bf16x3_3d_slab_against_fp32_readout():
    """The 3D GRE workload at 16^3 voxels (16,384 spins, many tiles per CTA, windows of up to 64 samples)."""
    ph, seq, coils = workloads.gre3d_64(16)
    f = bpb.simulate(ph, seq, coils)
    r = bpb.simulate(ph, seq, coils, readout="bf16x3")
    assert rel_l2(r.signal, f.signal.to(torch.complex128)) < L2
    assert torch.equal(r.m, f.m)


@pytest.mark.parametrize("n_coils", [1, 3, 8])
def test_bf16x3_coil_counts_and_ragged_spins(n_coils):
    n = 1000
    g = torch.Generator().manual_seed(40 + n_coils)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    ph = bpb.Phantom((rnd(n, 3) - 0.5) * 0.2, 0.5 + rnd(n), 0.2 + rnd(n), 0.02 + 0.1 * rnd(n), (rnd(n) - 0.5) * 200)
    b = bpb.SequenceBuilder()
    for i in range(3):
        b.rf(100e-6, flip_deg=30.0, phase=0.7 * i, n_steps=4)
        b.delay(0.5e-3, grad=(2000.0, 500.0 * (i - 1), 0.0))
        b.readout(70, 10e-6, grad=(-2000.0, 0.0, 300.0), phase=0.3 * i)  # 70 samples: two windows
        b.delay(1e-3, grad=(30000.0, 0.0, 0.0))
    seq = b.build()
    coils = torch.complex(rnd(n, n_coils) - 0.5, rnd(n, n_coils) - 0.5)
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils))
    check(bpb.simulate(ph, seq, coils, readout="bf16x3"), sig, m)


def test_bf16x3_repeatable_and_refuses_many_coils():
    ph, seq, coils = workloads.gre2d_64()
    a = bpb.simulate(ph, seq, coils, readout="bf16x3").signal
    b = bpb.simulate(ph, seq, coils, readout="bf16x3").signal
    assert rel_l2(a, b.to(torch.complex128)) < 1e-6  # float64 atomics across CTAs: the order varies
    with pytest.raises(ValueError, match="at most 8 coils"):
        bpb.simulate(ph, seq, torch.ones(len(ph.pd), 9, dtype=torch.complex64), readout="bf16x3")
