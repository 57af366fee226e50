"""Forward parity on the GPU, through the public ``simulate`` (and so the C ABI of the sm_100a library).

Mirrors blochparty ``tests/engines/test_gpu.py`` (:15-83, :307-334): float32 GPU engine against the float64 core.
Here the references are the reference core's own float64 outputs (golden fixtures) and the float64 CPU oracle
(``oracle/bloch.py``, pinned to those fixtures). Tolerances: relative L2 over the signal 1e-5 (the plain-float32
bar), max-norm relative 1e-4 on the signal and 1e-5 on the final magnetization (the reference's own GPU tests).
"""

import math

import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import sequences, workloads
from golden_cases import NAMES, load, objects
from oracle import bloch

pytestmark = pytest.mark.gpu
F64 = torch.float64
SIG_L2, SIG_MAX, M_MAX = 1e-5, 1e-4, 1e-5


def rel_l2(a, b):
    a = a.to(b.dtype)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b).clamp_min(1e-300))


def rel_max(a, b):
    a = a.to(b.dtype)
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300)) if b.numel() else 0.0


def check(r, sig, m, l2=SIG_L2, mx=SIG_MAX, mm=M_MAX):
    assert r.signal.shape == sig.shape and r.signal.dtype == torch.complex64 and r.signal.device.type == "cpu"
    assert r.m.shape == m.shape and r.m.dtype == torch.float32
    assert torch.isfinite(torch.view_as_real(r.signal)).all()
    e = (rel_l2(r.signal, sig), rel_max(r.signal, sig), rel_max(r.m, m))
    assert e[0] < l2 and e[1] < mx and e[2] < mm, e
    return e


@pytest.mark.parametrize("name", NAMES)
def test_matches_reference_core_golden(name):
    case, sig, m, _ = load(name)
    ph, seq, coils, m_init = objects(case)
    check(bpb.simulate(ph, seq, coils, m_init=m_init), sig, m)


def test_gre2d_64_full_against_oracle():
    ph, seq, coils = workloads.gre2d_64()
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils))
    e = check(bpb.simulate(ph, seq, coils), sig, m)
    print("\ngre2d_64 fp32 vs float64 oracle: rel L2 %.2e, rel max %.2e, m %.2e" % e)


def _random_phantom(n, seed, b1=True):
    g = torch.Generator().manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    ph = bpb.Phantom(pos=(rnd(n, 3) - 0.5) * 0.2, pd=0.5 + rnd(n), t1=0.2 + rnd(n), t2=0.02 + 0.1 * rnd(n),
                     db0=(rnd(n) - 0.5) * 200, b1=(0.8 + 0.4 * rnd(n)) if b1 else None)
    return ph, g


def _busy_sequence(g, n_rep=4):
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    b = sequences.SequenceBuilder()
    for i in range(n_rep):
        b.rf_waveform(((rnd(30, 2) - 0.5) * 3000).numpy(), 10e-6, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.delay(0.4e-3, grad=(2000.0, float(rnd(1) - 0.5) * 3000, 0.0))
        b.readout(40, 10e-6, grad=(-2000.0, 0.0, 400.0), phase=0.3 * i)
        b.rf(60e-6, amplitude=2000.0, phase=1.1 * i, n_steps=3)
        b.readout(7, 15e-6, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.delay(1e-3, grad=((rnd(3) - 0.5) * 20000).numpy()).spoil()
    return b.build()


def test_ragged_spin_count_and_m_init():
    """N not a multiple of the 128-spin tile, a starting magnetization, several windows per readout."""
    n = 1000
    ph, g = _random_phantom(n, 5)
    seq = _busy_sequence(g)
    seq.b0_offset = (torch.rand(len(seq), generator=g, dtype=F64) - 0.5) * 30
    m_init = torch.stack([(torch.rand(n, generator=g, dtype=F64) - 0.5) * 0.5,
                          (torch.rand(n, generator=g, dtype=F64) - 0.5) * 0.5,
                          torch.rand(n, generator=g, dtype=F64)], -1)
    coils = bpb.birdcage_sensitivities(ph.pos, 8)
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils, m_init))
    check(bpb.simulate(ph, seq, coils, m_init=m_init), sig, m)


@pytest.mark.parametrize("n_coils", [1, 3, 8, 13, 32])
def test_coil_counts(n_coils):
    """One to 32 coils: one to four coil groups of the readout, padded groups."""
    n = 300
    ph, g = _random_phantom(n, 11 + n_coils)
    seq = _busy_sequence(g, 3)
    coils = torch.complex(torch.rand(n, n_coils, generator=g, dtype=F64) - 0.5,
                          torch.rand(n, n_coils, generator=g, dtype=F64) - 0.5)
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils))
    check(bpb.simulate(ph, seq, coils), sig, m)


def test_default_coil_and_no_adc():
    n = 200
    ph, g = _random_phantom(n, 21, b1=False)
    b = sequences.SequenceBuilder().rf(200e-6, flip_deg=70.0, n_steps=5).delay(3e-3, grad=(900.0, 0.0, 0.0))
    seq = b.build()
    r = bpb.simulate(ph, seq)
    sig, m = bloch.simulate(bloch.case_from(ph, seq))
    assert r.signal.shape == (1, 0)
    assert rel_max(r.m, m) < M_MAX


def test_hard_pulse_fid_closed_form():
    """90-degree hard pulse then free decay sampled every ms: i M0 exp(-t/T2) exp(-i 2 pi f t)
    (blochparty tests/engines/test_gpu.py:71-83, 1e-5 absolute). The pulse lasts 1 ns so that the 37 Hz offset
    tilts its axis by only 2e-7 rad (the closed form ignores precession during the pulse)."""
    t2, f = 0.05, 37.0
    ph = bpb.Phantom(torch.zeros(1, 3, dtype=F64), torch.ones(1, dtype=F64), torch.full((1,), 1e9, dtype=F64),
                     torch.full((1,), t2, dtype=F64), torch.full((1,), f, dtype=F64))
    b = sequences.SequenceBuilder().rf(1e-9, flip_deg=90.0)
    for _ in range(20):
        b.delay(1e-3)
        b._adc[-1] = True
    r = bpb.simulate(ph, b.build())
    assert r.signal.shape == (1, 20)
    for j in range(20):
        t = (j + 1) * 1e-3
        expect = 1j * math.exp(-t / t2) * complex(math.cos(-2 * math.pi * f * t), math.sin(-2 * math.pi * f * t))
        got = complex(r.signal[0, j])
        assert abs(got - expect) < 1e-5, (j, got, expect, r.m)


@pytest.mark.parametrize("n_seg", [5000, 20000])
def test_long_rf_trains_do_not_drift(n_seg):
    """Continuous-wave saturation as 10 us RF segments, blochparty's own case and tolerance
    (tests/engines/test_gpu.py:307-334): 32 spins at offsets -2..2 kHz, 1.5 uT-equivalent RF, m within 1e-5
    absolute of the float64 oracle and the signal within 1e-5 per spin."""
    n = 32
    one = torch.ones(n, dtype=F64)
    ph = bpb.Phantom(torch.zeros(n, 3, dtype=F64), one, one, 0.05 * one, -torch.linspace(-2000, 2000, n, dtype=F64))
    seq = sequences.SequenceBuilder().rf(n_seg * 10e-6, amplitude=42.577 * 1.5, n_steps=n_seg).readout(4, 10e-6).build()
    sig, m = bloch.simulate(bloch.case_from(ph, seq))
    r = bpb.simulate(ph, seq)
    assert float((r.m.double() - m).abs().max()) < 1e-5
    assert float((r.signal.to(sig.dtype) - sig).abs().max()) < 1e-5 * n


def test_strong_rf_train_coherent_rounding():
    """A stronger train (250 Hz, 5000 segments, random spins with B1 and a gradient): the per-segment rotation
    angle carries float32 rounding that adds up coherently over the train (~1e-7 relative per segment over
    78 rad); bounded at 5e-5 relative here, the same order as the float32 reference engines."""
    n = 64
    ph, g = _random_phantom(n, 31)
    b = sequences.SequenceBuilder().rf(5000 * 10e-6, amplitude=250.0, n_steps=5000, grad=(0.0, 0.0, 300.0))
    b.readout(8, 10e-6, grad=(500.0, 0.0, 0.0))
    seq = b.build()
    coils = bpb.birdcage_sensitivities(ph.pos, 2)
    sig, m = bloch.simulate(bloch.case_from(ph, seq, coils))
    check(bpb.simulate(ph, seq, coils), sig, m, l2=5e-5, mx=5e-5, mm=5e-5)


def test_spin_sets_add_up():
    """The signal is linear in the spins: two halves simulated apart sum to the whole (a size-independent
    property, here on the 64^3 GRE with 16^3 voxels to keep it short)."""
    ph, seq, coils = workloads.gre3d_64(16)
    whole = bpb.simulate(ph, seq, coils).signal.to(torch.complex128)
    half = len(ph.pd) // 2
    take = lambda sl: bpb.Phantom(ph.pos[sl], ph.pd[sl], ph.t1[sl], ph.t2[sl], ph.db0[sl])
    a = bpb.simulate(take(slice(0, half)), seq, coils[:half]).signal.to(torch.complex128)
    b = bpb.simulate(take(slice(half, None)), seq, coils[half:]).signal.to(torch.complex128)
    assert rel_l2(a + b, whole) < 1e-6


def test_repeatable():
    ph, seq, coils = workloads.gre2d_64()
    r1, r2 = bpb.simulate(ph, seq, coils), bpb.simulate(ph, seq, coils)
    assert rel_l2(r1.signal, r2.signal.to(torch.complex128)) < 1e-6  # float64 atomics: order varies
    assert torch.equal(r1.m, r2.m)
