"""Gradients through the hand-written adjoint on the GPU (``simulate`` with inputs that require grad).

Mirrors blochparty ``tests/engines/test_gpu_grad.py``: every input's gradient of a fixed random-weight linear loss
against the float64 core's autograd (golden fixtures written by the reference itself, and the float64 oracle),
the per-TR flip train of the 2D 128^2 adjoint workload against central finite differences, and bit-identical
gradients for any ``checkpoint_every`` and across runs (blochparty test_gpu_grad.py:95-102).
Tolerances: largest relative error (max-norm) per input 2e-4, the reference engines' gradient tolerance
(blochparty tests/engines/test_engines.py:47 GRAD_TOL).
"""

from dataclasses import replace

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import workloads
from golden_cases import load, objects
from oracle import bloch

pytestmark = pytest.mark.gpu
F64 = torch.float64
GRAD_TOL = 2e-4

NAMES = ("pos", "pd", "t1", "t2", "db0", "b1", "coils", "dt", "rf", "grad", "adc_phase", "b0_offset", "m_init")


def rel(a, b):
    a = a.to(b.dtype)
    s = b.abs().max()
    return float((a - b).abs().max() / s) if s > 0 else float((a - b).abs().max())


def gpu_gradients(ph, seq, coils, m_init, loss_fn, names=NAMES, **kw):
    leaves = {}

    def leaf(k, t):
        if t is None or k not in names:
            return t
        t = t.detach().clone().requires_grad_()
        leaves[k] = t
        return t

    gph = bpb.Phantom(leaf("pos", ph.pos), leaf("pd", ph.pd), leaf("t1", ph.t1), leaf("t2", ph.t2),
                      leaf("db0", ph.db0), b1=leaf("b1", ph.b1))
    gseq = bpb.Sequence(leaf("dt", seq.dt), leaf("rf", seq.rf), leaf("grad", seq.grad),
                        leaf("adc_phase", seq.adc_phase), list(seq.is_rf), list(seq.adc), list(seq.spoil),
                        b0_offset=leaf("b0_offset", seq.b0_offset))
    r = bpb.simulate(gph, gseq, leaf("coils", coils), m_init=leaf("m_init", m_init), **kw)
    loss = loss_fn(r.signal, r.m)
    grads = torch.autograd.grad(loss, list(leaves.values()), allow_unused=True)
    return float(loss.detach()), {k: g for k, g in zip(leaves, grads)}


@pytest.mark.parametrize("name", ["grad_rand", "grad_busy"])
def test_gradients_match_reference_autograd(name):
    case, _, _, z = load(name)
    ph, seq, coils, m_init = objects(case)
    wr, wi, wm = (torch.from_numpy(z[k]) for k in ("w_re", "w_im", "w_m"))
    loss = lambda s, m: (s.real.double() * wr).sum() + (s.imag.double() * wi).sum() + (m.double() * wm).sum()
    _, g = gpu_gradients(ph, seq, coils, m_init, loss)
    errors = {}
    for k, v in g.items():
        if v is None:
            continue
        ref = (torch.complex(torch.from_numpy(z[f"grad_{k}_re"]), torch.from_numpy(z[f"grad_{k}_im"]))
               if k == "coils" else torch.from_numpy(z[f"grad_{k}"]))
        errors[k] = rel(v, ref)
    assert len(errors) >= 11, errors
    assert max(errors.values()) < GRAD_TOL, errors


@pytest.mark.parametrize("name", ["grad_rand", "grad_busy"])
def test_rf_gradient_alone_matches_reference_autograd(name):
    """The RF waveform's gradient alone runs the sweep without per-spin gradients; the busy case's windows that
    mix RF and free segments (an ADC at the end of an RF segment) and the spoils after runs take its recompute
    from the window start. Against the reference's float64 autograd (the same fixtures)."""
    case, _, _, z = load(name)
    ph, seq, coils, m_init = objects(case)
    wr, wi, wm = (torch.from_numpy(z[k]) for k in ("w_re", "w_im", "w_m"))
    loss = lambda s, m: (s.real.double() * wr).sum() + (s.imag.double() * wi).sum() + (m.double() * wm).sum()
    _, g = gpu_gradients(ph, seq, coils, m_init, loss, names=("rf",))
    err = rel(g["rf"], torch.from_numpy(z["grad_rf"]))
    print(f"\n{name}: RF gradient alone {err:.1e}")
    assert err < GRAD_TOL, err


def _adjoint_case(n=32):
    ph, seq, coils, flips, t1_target = workloads.adjoint_2d_128(n)
    return ph, seq, coils, flips, t1_target


def _target(ph, seq, coils, t1_target):
    with torch.no_grad():
        return bpb.simulate(replace(ph, t1=t1_target), seq, coils).signal.to(torch.complex128)


def test_adjoint_workload_vjp_against_oracle():
    """The 2D adjoint workload (32^2 here) with its cotangent fixed: d/dtheta of Re sum conj(w) s, where w is the
    GPU's own residual 2 (s - s_target) (so both sides differentiate the same linear form), w.r.t. T1, T2, PD, B0,
    B1, the coils and the RF train, against the float64 oracle's autograd; the bar is the engines' 2e-4."""
    ph, seq, coils, flips, t1_target = _adjoint_case(32)
    target = _target(ph, seq, coils, t1_target)
    with torch.no_grad():
        w = 2 * (bpb.simulate(ph, seq, coils).signal.to(torch.complex128) - target)
    loss = lambda s, m: (s.to(torch.complex128) * w.conj()).real.sum()
    names = ("pd", "t1", "t2", "db0", "b1", "coils", "rf")
    _, g = gpu_gradients(ph, seq, coils, None, loss, names, checkpoint_every=8 * 32)
    _, ref = bloch.gradients(bloch.case_from(ph, seq, coils), loss, names=names)
    errors = {k: rel(g[k], ref[k]) for k in names}
    print("\nadjoint 32^2 fixed-cotangent relative errors:", {k: f"{v:.1e}" for k, v in errors.items()})
    assert max(errors.values()) < GRAD_TOL, errors


def test_adjoint_workload_loss_against_oracle_autograd():
    """The workload's own loss, ||s - s_target||^2 with s_target from T1 (1 + 5% noise): both sides use their own
    forward, so the float32 forward's ~1e-6 relative error enters the small residual (a few % of s) and is
    amplified ~30x in every gradient; bounded at 2e-3 here (the reference's integration test allows 3e-3 on
    flip and B1 gradients, blochparty tests/engines/test_integration.py:38-53)."""
    ph, seq, coils, flips, t1_target = _adjoint_case(32)
    target = _target(ph, seq, coils, t1_target)
    names = ("pd", "t1", "t2", "db0", "b1", "coils", "rf")
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum()
    _, g = gpu_gradients(ph, seq, coils, None, loss, names, checkpoint_every=8 * 32)
    _, ref = bloch.gradients(bloch.case_from(ph, seq, coils), loss, names=names)
    errors = {k: rel(g[k], ref[k]) for k in names}
    print("\nadjoint 32^2 workload-loss relative errors:", {k: f"{v:.1e}" for k, v in errors.items()})
    assert max(errors.values()) < 2e-3, errors


def test_flip_train_against_central_differences():
    """d loss / d flip_j through the per-TR RF amplitudes, against central differences of the GPU forward
    (h = 1e-3 relative); the float32 forward limits the agreement to ~1e-3."""
    ph, seq, coils, flips, t1_target = _adjoint_case(16)
    target = _target(ph, seq, coils, t1_target)
    rf_idx = np.flatnonzero(np.asarray(seq.is_rf))
    assert len(rf_idx) == len(flips)

    def with_flips(f):
        rf = seq.rf.clone()
        rf[rf_idx] = seq.rf[rf_idx] * (f / flips)[:, None]
        return replace(seq, rf=rf)

    def loss_of(f):
        with torch.no_grad():
            s = bpb.simulate(ph, with_flips(f), coils).signal.to(torch.complex128)
        return float(((s - target).abs() ** 2).sum())

    f = flips.clone().requires_grad_()
    r = bpb.simulate(ph, with_flips(f), coils)
    loss = ((r.signal.to(torch.complex128) - target).abs() ** 2).sum()
    (g,) = torch.autograd.grad(loss, [f])
    for j in (0, 3, len(flips) // 2, len(flips) - 1):
        h = 1e-3 * float(flips[j])
        fp, fm = flips.clone(), flips.clone()
        fp[j] += h
        fm[j] -= h
        fd = (loss_of(fp) - loss_of(fm)) / (2 * h)
        assert abs(float(g[j]) - fd) <= 2e-3 * abs(fd) + 1e-6 * float(loss), (j, float(g[j]), fd)


def test_gradients_do_not_depend_on_checkpoint_interval():
    ph, seq, coils, flips, t1_target = _adjoint_case(16)
    target = _target(ph, seq, coils, t1_target)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    names = ("pd", "t1", "t2", "db0", "b1", "coils", "rf", "dt", "grad")
    _, a = gpu_gradients(ph, seq, coils, None, loss, names, checkpoint_every=64)
    _, b = gpu_gradients(ph, seq, coils, None, loss, names, checkpoint_every=32 * 50)
    _, c = gpu_gradients(ph, seq, coils, None, loss, names, checkpoint_every=32 * 50)
    for k in names:
        assert torch.equal(a[k], b[k]), k
        assert torch.equal(b[k], c[k]), k


def test_outer_checkpoint_level_keeps_the_gradients(monkeypatch):
    """Three checkpoint levels (the forward stores every third interval start, the backward rebuilds the others
    from it) give the two-level gradients bit for bit: the rebuilt interval starts are the forward's own states."""
    from blochparty_b200 import adjoint

    ph, seq, coils, flips, t1_target = _adjoint_case(16)
    target = _target(ph, seq, coils, t1_target)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    names = ("pd", "t1", "t2", "db0", "b1", "coils", "rf", "dt", "grad")
    monkeypatch.setattr(adjoint, "choose_checkpoints", lambda S, n: (64, 0))
    _, a = gpu_gradients(ph, seq, coils, None, loss, names)
    monkeypatch.setattr(adjoint, "choose_checkpoints", lambda S, n: (64, 3))
    _, b = gpu_gradients(ph, seq, coils, None, loss, names)
    for k in names:
        assert torch.equal(a[k], b[k]), k


def test_sweep_without_offset_gradients_matches_the_full_sweep():
    """Asking for T1, T2, PD and the RF alone takes the sweep variant that skips the offsets' gradients (position,
    dB0, segment dt, moments, b0_offset): its gradients are the full sweep's, bit for bit."""
    ph, seq, coils, flips, t1_target = _adjoint_case(16)
    target = _target(ph, seq, coils, t1_target)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    lean = ("pd", "t1", "t2", "rf")
    _, a = gpu_gradients(ph, seq, coils, None, loss, lean)
    _, b = gpu_gradients(ph, seq, coils, None, loss, lean + ("pos", "db0"))
    for k in lean:
        assert torch.equal(a[k], b[k]), k


@pytest.mark.parametrize("case", ["adjoint", "head"])
def test_sweep_without_spin_gradients_matches_the_full_sweep(case):
    """Asking for the RF waveform alone takes the sweep variant without per-spin gradients: its windows of free
    segments carry lambda back without recomputing states, and its windows of RF segments integrate the states
    backward from the state after them instead of recomputing them forward (on these sequences from the states the
    forward saved after each RF run: the whole slab pulse, 200 steps, is integrated backward). Its RF gradients are
    the full sweep's within 3e-5 (largest error over the largest value: the two sweeps' float32 states differ by
    their roundings, which accumulate over a pulse integrated backward; 3.7e-6 with one 32-step window at a time),
    on the 2D flip-train case and on the 4-echo head workload at 16^3 with its readout runs; and the variant's own
    gradients are the same bits for every checkpoint interval."""
    if case == "adjoint":
        ph, seq, coils, flips, t1_target = _adjoint_case(16)
        target = _target(ph, seq, coils, t1_target)
    else:
        ph, seq, coils = workloads.gre3d_128_4echo(16)
        seq = workloads.first_n_trs(seq, 12)
        target = torch.zeros(coils.shape[1], int(sum(seq.adc)), dtype=torch.complex128)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    lean = ("rf",)
    _, a = gpu_gradients(ph, seq, coils, None, loss, lean, checkpoint_every=64)
    _, c = gpu_gradients(ph, seq, coils, None, loss, lean, checkpoint_every=32 * 40)
    _, b = gpu_gradients(ph, seq, coils, None, loss, lean + ("t1",))
    assert torch.equal(a["rf"], c["rf"])
    err = rel(a["rf"], b["rf"])
    print(f"\n{case}: RF gradient without per-spin gradients against the full sweep {err:.1e}")
    assert err < 3e-5, err


@pytest.mark.parametrize("case", ["adjoint", "head"])
def test_backward_from_saved_states(case, monkeypatch):
    """The RF waveform's gradient alone on a sequence whose adjoint windows are all runs of RF segments (one dt and
    offset, no sample, no spoil) or of free segments takes the backward from saved states: the forward saves the
    state after every RF run, the sweep integrates each run's windows backward from it (the chain carried across
    the intervals) and replays nothing. Against the same sweep with a replay of every interval: RF gradient within
    3e-5 (the chain's states are integrated over a whole pulse instead of one 32-step window), the forward's signal
    and m the same bits (the forward's extra window starts fall after RF segments), and the same bits for any
    checkpoint_every."""
    from blochparty_b200 import adjoint

    if case == "adjoint":
        ph, seq, coils, flips, t1_target = _adjoint_case(16)
        target = _target(ph, seq, coils, t1_target)
    else:
        ph, seq, coils = workloads.gre3d_128_4echo(16)
        seq = workloads.first_n_trs(seq, 12)
        target = torch.zeros(coils.shape[1], int(sum(seq.adc)), dtype=torch.complex128)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    modes = []
    init = adjoint.Checkpointed.__init__

    def spy(self, *a, **k):
        init(self, *a, **k)
        modes.append(None if self.saved is None else self.saved.n_slots)

    monkeypatch.setattr(adjoint.Checkpointed, "__init__", spy)
    la, a = gpu_gradients(ph, seq, coils, None, loss, ("rf",), checkpoint_every=64)
    lc, c = gpu_gradients(ph, seq, coils, None, loss, ("rf",), checkpoint_every=32 * 40)
    monkeypatch.setattr(adjoint.SavedStates, "of", classmethod(lambda cls, flags, awin: None))
    lb, b = gpu_gradients(ph, seq, coils, None, loss, ("rf",), checkpoint_every=64)
    print(f"\n{case}: {modes[0]} saved states (one per TR)")
    assert modes == [seq.meta["n_tr"], seq.meta["n_tr"], None], modes
    assert la == lb == lc
    assert torch.equal(a["rf"], c["rf"])
    err = rel(a["rf"], b["rf"])
    print(f"{case}: RF gradient from saved states against the replay's {err:.1e}")
    assert err < 3e-5, err


def test_checkpoint_every_must_be_window_multiple():
    ph, seq, coils, _, _ = _adjoint_case(8)
    with pytest.raises(ValueError, match="multiple of 32"):
        bpb.simulate(replace(ph, t1=ph.t1.clone().requires_grad_()), seq, coils, checkpoint_every=48)


def test_saved_states_in_blocks_keep_the_bits(monkeypatch):
    """When the states saved after the RF runs do not fit (here: a budget of 9 states for 12), the forward stores
    the starts of blocks of intervals and the backward rebuilds each block's saved states by one forward of the
    block before its sweep: the rebuilt states are the forward's own, so the RF gradient is the one-block run's bit
    for bit (4-echo head workload at 16^3, 12 TRs)."""
    from blochparty_b200 import adjoint

    ph, seq, coils = workloads.gre3d_128_4echo(16)
    seq = workloads.first_n_trs(seq, 12)
    target = torch.zeros(coils.shape[1], int(sum(seq.adc)), dtype=torch.complex128)
    loss = lambda s, m: ((s.to(torch.complex128) - target).abs() ** 2).sum() + m.double().sum()
    blocks = []
    init = adjoint.Checkpointed.__init__

    def spy(self, *a, **k):
        init(self, *a, **k)
        blocks.append(len(self.blocks()) if self.saved is not None else None)

    monkeypatch.setattr(adjoint.Checkpointed, "__init__", spy)
    la, a = gpu_gradients(ph, seq, coils, None, loss, ("rf",), checkpoint_every=64)
    layout = adjoint.saved_layout
    monkeypatch.setattr(adjoint, "saved_layout", lambda plan, sb, budget: layout(plan, sb, 9 * sb))
    lb, b = gpu_gradients(ph, seq, coils, None, loss, ("rf",), checkpoint_every=64)
    print(f"\nblocks: {blocks}")
    assert blocks[0] == 1 and blocks[1] > 1, blocks
    assert la == lb
    assert torch.equal(a["rf"], b["rf"])
