"""The CPU oracle against the reference's own float64 outputs and gradients (the golden fixtures), and against
closed forms (blochparty tests/physics/test_analytic.py covers the same physics for its core)."""

import math

import pytest
import torch

from golden_cases import NAMES, load
from oracle import bloch

F64 = torch.float64


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("merge", [True, False])
def test_oracle_matches_reference_core(name, merge):
    case, sig, m, _ = load(name)
    s, mm = bloch.simulate(case, merge=merge)
    assert s.shape == sig.shape
    assert rel(s, sig) < 1e-11
    assert rel(mm, m) < 1e-11


@pytest.mark.parametrize("name", ["grad_rand", "grad_busy"])
def test_oracle_gradients_match_reference_autograd(name):
    case, _, _, z = load(name)
    wr, wi, wm = (torch.from_numpy(z[k]).to(F64) for k in ("w_re", "w_im", "w_m"))
    loss = lambda s, m: (s.real * wr).sum() + (s.imag * wi).sum() + (m * wm).sum()
    _, g = bloch.gradients(case, loss)
    checked = 0
    for k, v in g.items():
        if v is None:
            continue
        if v.is_complex():
            ref = torch.complex(torch.from_numpy(z[f"grad_{k}_re"]), torch.from_numpy(z[f"grad_{k}_im"]))
        else:
            ref = torch.from_numpy(z[f"grad_{k}"])
        assert rel(v, ref) < 1e-9, k
        checked += 1
    assert checked >= 11


def _one_spin(**kw):
    base = dict(pos=torch.zeros(1, 3, dtype=F64), pd=torch.ones(1, dtype=F64), t1=torch.full((1,), 1e9, dtype=F64),
                t2=torch.full((1,), 1e9, dtype=F64), db0=torch.zeros(1, dtype=F64), b1=None,
                coils=torch.ones(1, 1, dtype=torch.complex128))
    base.update(kw)
    return base


def test_flip_angle_and_phase_convention():
    """A hard pulse of flip a about x leaves Mxy = i sin(a) (blochparty's convention Mxy = i e^{i phase})."""
    for deg, ph in ((30.0, 0.0), (90.0, 0.7), (150.0, -2.0)):
        dur = 1e-4
        amp = deg / 360.0 / dur
        case = bloch.Case(**_one_spin(), dt=torch.tensor([dur, 1e-6], dtype=F64),
                          rf=torch.tensor([[amp * math.cos(ph), amp * math.sin(ph)], [0, 0]], dtype=F64),
                          grad=torch.zeros(2, 3, dtype=F64), adc_phase=torch.zeros(2, dtype=F64), b0_offset=None,
                          is_rf=[True, False], adc=[False, True], spoil=[False, False])
        sig, m = bloch.simulate(case)
        a = math.radians(deg)
        expect = 1j * math.sin(a) * complex(math.cos(ph), math.sin(ph))
        assert abs(complex(sig[0, 0]) - expect) < 1e-12
        assert abs(float(m[0, 2]) - math.cos(a)) < 1e-12


def test_fid_decay_and_precession():
    t2, f = 0.05, 37.0
    n = 20
    dts = [1e-4] + [1e-3] * n
    case = bloch.Case(**_one_spin(t2=torch.tensor([t2], dtype=F64), db0=torch.tensor([f], dtype=F64)),
                      dt=torch.tensor(dts, dtype=F64),
                      rf=torch.tensor([[2500.0, 0.0]] + [[0.0, 0.0]] * n, dtype=F64),
                      grad=torch.zeros(n + 1, 3, dtype=F64), adc_phase=torch.zeros(n + 1, dtype=F64),
                      b0_offset=None, is_rf=[True] + [False] * n, adc=[False] + [True] * n, spoil=[False] * (n + 1))
    sig, _ = bloch.simulate(case)
    # 90-degree pulse (2500 Hz x 100 us); relaxation over the pulse is split around it
    m0 = complex(bloch.simulate(bloch.Case(**{**case.__dict__, "dt": case.dt[:1], "rf": case.rf[:1],
                                               "grad": case.grad[:1], "adc_phase": case.adc_phase[:1],
                                               "is_rf": [True], "adc": [True], "spoil": [False]}))[0][0, 0])
    for j in range(n):
        t = (j + 1) * 1e-3
        expect = m0 * math.exp(-t / t2) * complex(math.cos(-2 * math.pi * f * t), math.sin(-2 * math.pi * f * t))
        assert abs(complex(sig[0, j]) - expect) < 1e-12


def test_spoiled_gre_steady_state():
    """Ideal spoiling: the steady state after many TRs is the Ernst signal
    M0 sin(a) (1 - E1) / (1 - cos(a) E1) (blochparty reference.py: spoiled_gre_signal)."""
    t1, t2, tr, deg = 0.8, 0.05, 10e-3, 20.0
    amp = deg / 360.0 / 1e-6
    k = 600
    dts, rfs, adc, spoil, isrf = [], [], [], [], []
    for _ in range(k):
        dts += [1e-6, 1e-6, tr - 2e-6]
        rfs += [[amp, 0.0], [0.0, 0.0], [0.0, 0.0]]
        isrf += [True, False, False]
        adc += [False, True, False]
        spoil += [False, False, True]
    case = bloch.Case(**_one_spin(t1=torch.tensor([t1], dtype=F64), t2=torch.tensor([t2], dtype=F64)),
                      dt=torch.tensor(dts, dtype=F64), rf=torch.tensor(rfs, dtype=F64),
                      grad=torch.zeros(3 * k, 3, dtype=F64), adc_phase=torch.zeros(3 * k, dtype=F64),
                      b0_offset=None, is_rf=isrf, adc=adc, spoil=spoil)
    sig, _ = bloch.simulate(case)
    a, e1 = math.radians(deg), math.exp(-tr / t1)
    ernst = math.sin(a) * (1 - e1) / (1 - math.cos(a) * e1)
    assert abs(abs(complex(sig[0, -1])) - ernst) < 1e-4


@pytest.mark.parametrize("name", NAMES)
def test_c_oracle_matches_reference_core(name):
    """The C restatement (``oracle/bloch_c.c``, for the workloads' long sequences) against the reference's float64
    outputs, with one thread and with chunks of 3 samples (every chunk boundary case), and against the Python
    restatement."""
    from oracle import fast

    case, sig, m, _ = load(name)
    ref_s, ref_m = bloch.simulate(case)
    for threads, chunk in ((0, 0), (1, 3)):
        s, mm = fast.simulate(case, threads=threads, chunk=chunk)
        assert s.shape == sig.shape
        assert rel(s, sig) < 1e-11 and rel(mm, m) < 1e-11
        assert rel(s, ref_s) < 1e-11 and rel(mm, ref_m) < 1e-11


def test_c_oracle_matches_python_oracle_on_a_2d_gre():
    """Both restatements on a 16^2 GRE with 20 dummy TRs and radial B1 (many runs and samples), 3-sample chunks."""
    from blochparty_b200 import phantoms, sequences
    from oracle import fast

    ph = phantoms.ellipse_phantom_2d(16, 0.25, seed=2)
    ph.b1 = phantoms.radial_b1(ph.pos)
    seq = sequences.gre((16, 16), 0.25, flip_deg=25.0, tr=6e-3, te=3e-3, n_dummy=20, dwell=20e-6)
    case = bloch.case_from(ph, seq, phantoms.birdcage_sensitivities(ph.pos, 3))
    s0, m0 = bloch.simulate(case)
    s1, m1 = fast.simulate(case, chunk=3)
    assert rel(s1, s0) < 1e-11 and rel(m1, m0) < 1e-11


def test_adjoint128_golden_is_this_packages_case_and_the_oracle_follows_it():
    """The 128^2 flip-train golden (the reference's float64 core and autograd at the case's own size): this
    package's builders still make the inputs it was written from, and the oracle's loss and gradients follow it."""
    from golden_cases import load_adjoint128

    z, (ph, seq, coils, flips, t1_target), same = load_adjoint128()
    assert all(same.values()), same
    s_t = torch.complex(torch.from_numpy(z["s_t_re"]).to(F64), torch.from_numpy(z["s_t_im"]).to(F64))
    case = bloch.case_from(ph, seq, coils)
    loss, g = bloch.gradients(case, lambda s, m: ((s - s_t).abs() ** 2).sum(), names=("t1", "t2", "pd", "db0", "b1"))
    assert abs(loss - float(z["loss"])) < 1e-5 * float(z["loss"])
    for k in ("t1", "t2", "pd", "db0", "b1"):
        ref = torch.from_numpy(z[f"grad_{k}"]).to(F64)
        assert rel(g[k], ref) < 1e-5, k
