"""The bound pool (magnetization transfer) and the scanner field model on the GPU (``bp_forward_physics``).

Mirrors blochparty ``tests/engines/test_gpu.py:86-125`` (``test_scanner_field_model``, ``test_magnetization_transfer``):
the engine against the reference's own float64 core on the fixtures ``tests/golden/mt_*.npz`` and ``field_*.npz``
(bound pool with the super-Lorentzian and the Lorentzian lineshape, bound-only RF, a four-column m_init; on a 3D
slab GRE: gradient nonlinearity alone, leading-order and exact concomitant fields (10 % of the signal), and a bound
pool with the field model). Bars: the reference's own for its GPU engines against its core (1e-4 on the signal, m
and the bound pool's Mz, max-norm relative; m 1e-3 with the field model), and 1e-5 against the float64 oracle fed
the engine's float32-rounded inputs (the engine's own arithmetic, without the inputs' rounding: the plain kernel's
bar on every configuration; a 3D slab GRE's long RF trains alone put the float32 engine at 3-8e-6). Also: the variant
with nothing switched on is the plain kernel's result, and a 3D GRE with a pool against the oracle.
"""

from dataclasses import replace

import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import phantoms, physics, sequences
from golden_cases import PHYSICS, load_physics
from oracle import bloch

pytestmark = pytest.mark.gpu
F64 = torch.float64


def rel(a, b):
    b = b.to(torch.float64)
    return float((a.to(torch.float64) - b).abs().max() / b.abs().max())


def f32_case(ph, seq, coils, m0, sc):
    """The oracle's case on the engine's float32 inputs: encoding positions, PD, 1/T1, 1/T2, dB0, B1, coils, the
    concomitant coefficients and the pool's f, k, 1/T1b, T2b, dw each rounded once from float64."""
    r = lambda t: t.to(torch.float32).to(F64)
    c = bloch.case_from(ph, seq, coils, m0, sc)
    c.pos, c.pd, c.db0 = r(c.pos), r(c.pd), r(c.db0)
    c.t1, c.t2 = 1.0 / r(1.0 / c.t1), 1.0 / r(1.0 / c.t2)
    c.b1 = None if c.b1 is None else r(c.b1)
    c.coils = c.coils.to(torch.complex64).to(torch.complex128)
    if c.conc is not None:
        c.conc = r(c.conc)
    if c.bound is not None:
        b = c.bound
        c.bound = replace(b, f=r(b.f), k=r(b.k), t1=1.0 / r(1.0 / b.t1), t2=r(b.t2), dw=r(b.dw))
        c.f_rf = r(c.f_rf)
    return c


@pytest.mark.parametrize("name", PHYSICS)
def test_against_the_reference_core(name):
    (ph, seq, coils, m0, sc), (sig, m, mb), z = load_physics(name)
    r = bpb.simulate(ph, seq, coils, m_init=m0, scanner=sc)
    s32, m32, mb32 = bloch.simulate_with_pool(f32_case(ph, seq, coils, m0, sc))
    e = {"signal": rel(r.signal, sig), "m": rel(r.m, m), "signal_f32_inputs": rel(r.signal, s32),
         "m_f32_inputs": rel(r.m, m32)}
    if mb is not None:
        e["m_bound"] = float((r.m_bound.double() - mb).abs().max() / m.abs().max())
        e["m_bound_f32_inputs"] = float((r.m_bound.double() - mb32).abs().max() / m32.abs().max())
    else:
        assert r.m_bound is None
    print(f"\n{name}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert r.signal.dtype == torch.complex64 and r.m.dtype == torch.float32
    field = sc is not None
    assert e["signal"] < 1e-4 and e["m"] < (1e-3 if field else 1e-4) and e.get("m_bound", 0.0) < 1e-4, e
    assert max(v for k, v in e.items() if k.endswith("f32_inputs")) < 1e-5, e


def test_without_physics_is_the_plain_kernel():
    """A scanner with a zero nonlinearity and no concomitant fields runs the physics variant with nothing switched
    on: the plain kernel's result to float32 rounding (the variant steps every RF segment alone)."""
    p = phantoms.ellipse_phantom_2d(16, 0.25, seed=3)
    seq = sequences.gre((16, 16), 0.25, flip_deg=30.0, tr=6e-3, te=3e-3, n_dummy=4, dwell=20e-6)
    coils = phantoms.birdcage_sensitivities(p.pos, 4)
    zero = physics.GradientNonlinearity(torch.zeros(3, 4, 4, dtype=torch.float64),
                                        torch.zeros(3, 4, 4, dtype=torch.float64), 0.25)
    a = bpb.simulate(p, seq, coils, scanner=physics.Scanner(nonlinearity=zero))
    b = bpb.simulate(p, seq, coils)
    assert rel(a.signal, b.signal) < 2e-6 and rel(a.m, b.m) < 2e-6


def test_3d_slab_gre_with_pool_and_field_model_against_the_oracle():
    """A 3D GRE (8 x 8 x 4, 2 spins per voxel, two echoes) with a 40-step sinc slab pulse, every spin with a
    super-Lorentzian bound pool, at 0.55 T with leading-order concomitant fields, against the float64 oracle."""
    p = phantoms.ellipsoid_phantom_3d(8, 0.25, spins_per_voxel=2, b0_max=50.0, sigma_vox=1.0)
    n = len(p.pd)
    g = torch.Generator().manual_seed(21)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=torch.float64)
    bound = physics.BoundPool(0.1 + 0.05 * rnd(n), 20 + 20 * rnd(n), torch.ones(n, dtype=torch.float64),
                              (9 + 4 * rnd(n)) * 1e-6, (rnd(n) - 0.5) * 400)
    ph = replace(p, bound=bound)
    seq = sequences.gre((8, 8, 4), 0.25, flip_deg=20.0, tr=8e-3, te=3e-3, dwell=20e-6, rf="sinc", rf_duration=1.2e-3,
                        rf_steps=40, slab_thickness=0.15, n_echoes=2, echo_spacing=0.5e-3, n_dummy=2)
    coils = phantoms.birdcage_sensitivities(p.pos, 4)
    sc = physics.Scanner(field_strength=0.55, concomitant="leading")
    r = bpb.simulate(ph, seq, coils, scanner=sc)
    sig, m, mb = bloch.simulate_with_pool(bloch.case_from(ph, seq, coils, scanner=sc))
    s32, m32, mb32 = bloch.simulate_with_pool(f32_case(ph, seq, coils, None, sc))
    e = {"signal": rel(r.signal, sig), "m": rel(r.m, m),
         "m_bound": float((r.m_bound.double() - mb).abs().max() / m.abs().max()),
         "signal_f32_inputs": rel(r.signal, s32), "m_f32_inputs": rel(r.m, m32)}
    print(f"\n3D slab GRE, {n} spins x {len(seq)} segments, pool + field model: "
          + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert e["signal"] < 1e-4 and e["m"] < 1e-3 and e["m_bound"] < 1e-4, e
    assert e["signal_f32_inputs"] < 1e-5 and e["m_f32_inputs"] < 1e-5, e


@pytest.mark.parametrize("name", ["grad_field_leading", "grad_field_exact"])
def test_field_model_gradients_match_reference_autograd(name):
    """Gradients through the scanner field model (mirrors blochparty ``tests/engines/test_gpu_grad.py:57-75``): a
    random case with gradients x 30 at 0.55 T with a nonlinearity, the fixed linear loss of signal and m, against
    the reference's float64 autograd with respect to the nonlinearity's alpha, the field strength, T1, the positions,
    dB0, the RF waveform and the gradients. Bars: 2e-4 (largest error over the largest value), 1e-4 on B0 (the
    reference's own for its GPU engines)."""
    import numpy as np

    from golden_cases import GOLDEN

    z = np.load(GOLDEN / f"{name}.npz")
    t = lambda k: torch.from_numpy(z[k]).to(F64)
    leaves = {"alpha": t("sc_alpha").requires_grad_(), "b0": torch.tensor(float(z["sc_b0"]), dtype=F64,
                                                                           requires_grad=True),
              "t1": t("t1").requires_grad_(), "pos": t("pos").requires_grad_(), "db0": t("db0").requires_grad_(),
              "rf": t("rf").requires_grad_(), "grad": t("grad").requires_grad_()}
    sc = physics.Scanner(leaves["b0"], str(z["sc_conc"]),
                         nonlinearity=physics.GradientNonlinearity(leaves["alpha"], t("sc_beta"), float(z["sc_r0"])))
    ph = bpb.Phantom(leaves["pos"], t("pd"), leaves["t1"], t("t2"), leaves["db0"], b1=t("b1"))
    seq = bpb.Sequence(t("dt"), leaves["rf"], leaves["grad"], t("adc_phase"), [bool(x) for x in z["is_rf"]],
                       [bool(x) for x in z["adc"]], [bool(x) for x in z["spoil"]], b0_offset=t("b0_offset"))
    coils = torch.complex(t("coils_re"), t("coils_im"))
    r = bpb.simulate(ph, seq, coils, scanner=sc)
    wr, wi, wm = t("w_re"), t("w_im"), t("w_m")
    loss = (r.signal.real.double() * wr).sum() + (r.signal.imag.double() * wi).sum() + (r.m.double() * wm).sum()
    grads = torch.autograd.grad(loss, list(leaves.values()))
    e = {k: rel(g, t(f"grad_{k}")) for k, g in zip(leaves, grads)}
    print(f"\n{name}: " + ", ".join(f"{k} {v:.1e}" for k, v in e.items()))
    assert e["b0"] < 1e-4 and max(e.values()) < 2e-4, e
