"""The bound pool and the field model on the CPU: the oracle (``oracle/physics.py``, ``oracle.bloch``) against the
reference's own float64 core (``tests/golden/mt_*.npz``, ``field_*.npz``), and the product's host restatements
(``blochparty_b200.physics``: the super-Lorentzian table, the RF frequency, the encoding positions and concomitant
coefficients) against the reference's own values and the oracle's."""

import math

import numpy as np
import pytest
import torch

from blochparty_b200 import physics
from golden_cases import GOLDEN, PHYSICS, load_physics
from oracle import bloch
from oracle import physics as ophys


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_super_lorentzian_table_matches_the_reference():
    z = np.load(GOLDEN / "sl_table.npz")
    lx0, step, mine = physics.sl_table()
    assert abs(lx0 - z["lx"][0]) < 1e-15 and abs(step - (z["lx"][1] - z["lx"][0])) < 1e-15
    x = np.exp(z["lx"])
    d = np.abs(mine - z["log_f"])
    assert d[x < 3].max() < 1e-12, d[x < 3].max()  # where the lineshape is not negligible (ln F > -8)
    assert d.max() < 1e-9, d.max()


def test_oracle_super_lorentzian_points():
    """The oracle's adaptive quadrature at a few points of the reference's table."""
    z = np.load(GOLDEN / "sl_table.npz")
    for i in (0, 1000, 2048, 3000, 3600, 4096):
        x = float(np.exp(z["lx"][i]))
        assert abs(ophys._sl_log_point(x) - z["log_f"][i]) < 1e-9, (i, ophys._sl_log_point(x), z["log_f"][i])


def test_lineshape_host_against_oracle():
    n = 200
    g = torch.Generator().manual_seed(3)
    delta = (torch.rand(n, generator=g, dtype=torch.float64) - 0.5) * 4e4
    t2 = (8 + 6 * torch.rand(n, generator=g, dtype=torch.float64)) * 1e-6
    for shape in ("lorentzian", "superlorentzian"):
        pool = ophys.PoolCase(t2, t2, t2, t2, t2, shape, 1e3)
        ref = ophys.lineshape(pool, delta)
        mine = torch.from_numpy(physics.lineshape(delta.numpy(), t2.numpy(), shape, 1e3))
        assert rel(mine, ref) < 1e-12, shape


@pytest.mark.parametrize("name", ["mt_sl", "mt_lor", "mt_field"])
def test_rf_frequency_matches_the_reference(name):
    (ph, seq, coils, m0, sc), _, z = load_physics(name)
    ref = torch.from_numpy(z["ref_rf_freq"])
    mine = torch.from_numpy(physics.rf_frequency(seq.dt, seq.rf, seq.is_rf))
    assert float((mine - ref).abs().max()) <= 1e-9 * float(ref.abs().max())
    orc = ophys.rf_frequency(seq.dt, seq.rf, seq.is_rf)
    assert float((orc - ref).abs().max()) <= 1e-9 * float(ref.abs().max())


@pytest.mark.parametrize("name", ["field_nl", "field_leading", "field_exact", "mt_field"])
def test_spin_fields_match_the_reference(name):
    (ph, seq, coils, m0, sc), _, z = load_physics(name)
    for fn in (physics.spin_fields, ophys.spin_fields):
        enc, conc, mode = fn(sc, ph.pos)
        enc = torch.as_tensor(np.asarray(enc))
        assert mode == int(z["ref_mode"])
        assert float((enc - torch.from_numpy(z["ref_enc"])).abs().max()) < 1e-13
        if mode:
            conc = torch.as_tensor(np.asarray(conc))
            assert rel(conc, torch.from_numpy(z["ref_conc"])) < 1e-13


def test_solid_harmonics_two_ways():
    """The product's Cartesian recurrences against the oracle's scipy Legendre functions, up to degree 7."""
    g = torch.Generator().manual_seed(5)
    pos = ((torch.rand(300, 3, generator=g, dtype=torch.float64) - 0.5) * 0.4).numpy()
    a = [t.numpy() for t in physics.solid_harmonics(torch.from_numpy(pos), 7, 0.25)]
    b = ophys._solid(pos, 7, 0.25)
    for x, y in zip(a, b):
        assert np.abs(x - y).max() < 1e-13 * max(1.0, np.abs(y).max())


@pytest.mark.parametrize("name", PHYSICS)
def test_oracle_against_the_reference_core(name):
    (ph, seq, coils, m0, sc), (sig, m, mb), z = load_physics(name)
    sig_o, m_o, mb_o = bloch.simulate_with_pool(bloch.case_from(ph, seq, coils, m0, sc))
    assert rel(sig_o, sig) < 1e-11, rel(sig_o, sig)
    assert rel(m_o, m) < 1e-11
    if mb is not None:
        assert rel(mb_o, mb) < 1e-11
    else:
        assert mb_o is None


def test_field_model_host_functions_are_differentiable():
    """The encoding positions and concomitant coefficients (``physics.spin_fields_torch``) carry gradients to the
    nonlinearity's coefficients, the field strength and the positions: autograd against central differences."""
    g = torch.Generator().manual_seed(7)
    pos = ((torch.rand(40, 3, generator=g, dtype=torch.float64) - 0.5) * 0.3).requires_grad_()
    alpha = (torch.randn(3, 4, 4, generator=g, dtype=torch.float64) * 0.3).requires_grad_()
    beta = torch.randn(3, 4, 4, generator=g, dtype=torch.float64) * 0.3
    b0 = torch.tensor(0.55, dtype=torch.float64, requires_grad=True)
    wa, wb = torch.randn(40, 3, generator=g, dtype=torch.float64), torch.randn(40, 7, generator=g, dtype=torch.float64)

    def f(pos, alpha, b0, mode):
        sc = physics.Scanner(b0, mode, nonlinearity=physics.GradientNonlinearity(alpha, beta, 0.25))
        enc, conc, _ = physics.spin_fields_torch(sc, pos)
        # (each coefficient scaled to order one: the quadratic form's are ~1e-10, the transverse rows ~0.1 m, f0
        # 2.3e7 Hz)
        scale = 1e6 if mode == "leading" else torch.tensor([1.0] * 6 + [1e-7], dtype=torch.float64)
        return (enc * wa).sum() + (conc * wb[:, : conc.shape[1]] * scale).sum()

    for mode in ("leading", "exact"):
        ga, gb, gp = torch.autograd.grad(f(pos, alpha, b0, mode), [alpha, b0, pos])
        h = 1e-6
        d = torch.zeros_like(alpha)
        d[0, 3, 1] = 1.0
        fd = (f(pos, alpha + h * d, b0, mode) - f(pos, alpha - h * d, b0, mode)) / (2 * h)
        assert abs(float(ga[0, 3, 1]) - float(fd)) <= 1e-6 * max(1.0, abs(float(fd)))
        fd = (f(pos, alpha, b0 + h, mode) - f(pos, alpha, b0 - h, mode)) / (2 * h)
        assert abs(float(gb) - float(fd)) <= 1e-6 * max(1.0, abs(float(fd)))
        dp = torch.zeros_like(pos)
        dp[5, 2] = 1.0
        fd = (f(pos + h * dp, alpha, b0, mode) - f(pos - h * dp, alpha, b0, mode)) / (2 * h)
        assert abs(float(gp[5, 2]) - float(fd)) <= 1e-5 * max(1.0, abs(float(fd)))
