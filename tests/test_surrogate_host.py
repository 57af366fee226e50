"""Host-side checks of the learned RF surrogate (no GPU): the float64 rotation oracle against closed forms, the
frame relations the surrogate relies on, the network oracle's gradient, and the matching of pulse occurrences."""

import math

import numpy as np
import torch

from blochparty_b200 import api, sequences, surrogate, workloads
from oracle import surrogate as S

F64 = torch.float64


def test_hard_pulse_quaternion_is_a_rotation_about_x():
    """A constant RF of amplitude a for time T on resonance is the rotation by -2 pi a T about x."""
    a, n, dt = 500.0, 50, 1e-5
    rf = np.tile([[a, 0.0]], (n, 1))
    q, qr = S.pulse_quaternions(rf, dt, 0.0, torch.zeros(1), torch.zeros(1), torch.ones(1))
    angle = -2 * math.pi * a * n * dt
    expect = torch.tensor([[math.cos(angle / 2), math.sin(angle / 2), 0.0, 0.0]], dtype=F64)
    assert torch.allclose(q, expect, atol=1e-12) and torch.allclose(qr, expect, atol=1e-12)


def test_reduced_rotation_without_rf_is_the_identity():
    rf = np.zeros((30, 2))
    z, df = torch.tensor([0.01, -0.02]), torch.tensor([30.0, -150.0])
    q, qr = S.pulse_quaternions(rf, 1e-5, 2e5, z, df, torch.ones(2))
    assert torch.allclose(qr, torch.tensor([[1.0, 0, 0, 0]] * 2, dtype=F64), atol=1e-12)
    assert float((S.rotmat(q)[:, 2, 2] - 1).abs().max()) < 1e-12  # a pure z rotation


def test_rf_phase_conjugates_the_reduced_rotation():
    """RF x exp(i phi0): R = Rz(wz/2 + phi0) R~ Rz(wz/2 - phi0) with R~ the unshifted pulse's, exactly."""
    base, dt, gz, _ = sequences.sinc_pulse(90.0, 3e-3, 300, slice_thickness=5e-3)
    shifted, *_ = sequences.sinc_pulse(90.0, 3e-3, 300, slice_thickness=5e-3, phase=1.1)
    z = torch.tensor([-0.004, 0.0, 0.002], dtype=F64)
    df, b1 = torch.tensor([20.0, -80.0, 150.0], dtype=F64), torch.tensor([0.8, 1.0, 1.25], dtype=F64)
    q, _ = S.pulse_quaternions(shifted, dt, gz, z, df, b1)
    _, qr = S.pulse_quaternions(base, dt, gz, z, df, b1)
    a = -2 * math.pi * (gz * z + df) * 300 * dt
    cand = S.qmul(S.qmul(S.qz(0.5 * a + 1.1), qr), S.qz(0.5 * a - 1.1))
    assert float((S.rotmat(q) - S.rotmat(cand)).abs().max()) < 1e-12


def test_network_oracle_gradient_against_central_differences():
    g = torch.Generator().manual_seed(0)
    p = torch.randn(S.N_PARAMS, generator=g, dtype=F64) * 0.1
    x = torch.rand(16, 2, generator=g, dtype=F64) * 2 - 1
    t = torch.cat([torch.nn.functional.normalize(torch.randn(16, 4, generator=g, dtype=F64), dim=-1),
                   0.1 * torch.randn(16, 12, generator=g, dtype=F64)], -1)
    loss, grad = S.loss_and_grad(p, x, t, vweight=30.0, cweight=0.5)
    for i in (0, 100, 900, 5000, 9300, 10310):
        e = torch.zeros_like(p)
        e[i] = 1e-6
        fd = (S.loss_and_grad(p + e, x, t, 30.0, 0.5)[0] - S.loss_and_grad(p - e, x, t, 30.0, 0.5)[0]) / 2e-6
        assert abs(fd - float(grad[i])) < 1e-6 * max(1.0, abs(fd))


def test_occurrences_of_the_tse_pulses_are_found():
    ph, seq, coils = workloads.tse_3slice_128(16)
    sur = []
    for z0 in (-5e-3, 0.0, 5e-3):
        for flip, phase in ((90.0, 0.0), (180.0, 0.5 * math.pi)):
            w, dt, gz, _ = sequences.sinc_pulse(flip, 3e-3, 300, slice_thickness=5e-3, slice_offset=z0, phase=phase)
            sur.append(surrogate.RFSurrogate(w, dt, gz, 5e-3, device="cpu"))
    assert [round(s.z0 * 1e3, 6) for s in sur] == [-5.0, -5.0, 0.0, 0.0, 5.0, 5.0]
    inp = api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase,
                     None, list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    occ = surrogate.find_occurrences(sur, inp)
    assert len(occ) == sum(seq.is_rf) // 300
    starts = [o[0] for o in occ]
    assert all(seq.is_rf[s] and (s == 0 or not seq.is_rf[s - 1]) for s in starts)
    assert all(abs(o[3]) < 1e-9 for o in occ)  # every occurrence is one of the trained waveforms itself
    # the same pulses cut into two pieces each: twice the occurrences, back to back within every pulse
    halves = [h for z0 in (-5e-3, 0.0, 5e-3) for flip, phase in ((90.0, 0.0), (180.0, 0.5 * math.pi))
              for h in surrogate.pulse_pieces(sequences.sinc_pulse(flip, 3e-3, 300, slice_thickness=5e-3,
                                                                   slice_offset=z0, phase=phase)[0],
                                              1e-5, sur[0].gz, 5e-3, pieces=2, device="cpu")]
    occ2 = surrogate.find_occurrences(halves, inp)
    assert len(occ2) == 2 * len(occ) and all(o[1] == 150 for o in occ2)


def _tse_through_maps(n, first_order):
    """The 3-slice TSE (n^2 x 8 spins per slice) in float64 with every pulse occurrence replaced by the surrogate's
    map (``S.pulse_map``) built from EXACT targets (``S.pulse_targets``), the rest stepped by the oracle: the
    accuracy the map's form allows, before any network error."""
    from oracle import bloch

    ph, seq, coils = workloads.tse_3slice_128(n)
    c = bloch.case_from(ph, seq, coils)
    sgs = []
    for z0 in (-5e-3, 0.0, 5e-3):
        for flip, phase in ((90.0, 0.0), (180.0, 0.5 * math.pi)):
            w, dt, gz, _ = sequences.sinc_pulse(flip, 3e-3, 300, slice_thickness=5e-3, slice_offset=z0, phase=phase)
            sgs.append(surrogate.RFSurrogate(w, dt, gz, 5e-3, domain=(200.0, 0.3, 2.5), device="cpu"))
    inp = api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase, None,
                     list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    occ = {s: (k, i, phi) for s, k, i, phi, _ in surrogate.find_occurrences(sgs, inp)}
    z = c.pos[:, 2]
    targets = {}
    mx, my, mz = torch.zeros_like(c.pd), torch.zeros_like(c.pd), c.pd.clone()
    cols, skip = [], -1
    for a, b in bloch._steps(c.is_rf, c.spoil, True):
        if a < skip:
            continue
        if a in occ:
            k, i, phi = occ[a]
            sg = sgs[i]
            if i not in targets:
                targets[i] = S.pulse_targets(sg.rf, sg.dt, sg.gz, z, c.db0, torch.ones_like(z))[1]
            half = -math.pi * (sg.gz * z + c.db0) * sg.T
            m = S.pulse_map(targets[i], sg.T, half, phi, 1 / c.t1, 1 / c.t2, c.pd, torch.stack([mx, my, mz], -1),
                            first_order)
            mx, my, mz = m.unbind(-1)
            skip = a + k
            continue
        if c.is_rf[a]:
            mx, my, mz, _ = bloch._rf_step(mx, my, mz, a, c, None)
            if c.adc[a]:
                cols.append(bloch._sample(mx, my, c.adc_phase[a], c)[:, None])
        else:
            mx, my, mz, _, smp = bloch._free_run(mx, my, mz, a, b, c, None)
            cols += smp
        if c.spoil[b - 1]:
            mx, my = torch.zeros_like(mx), torch.zeros_like(my)
    sig64, _ = bloch.simulate(c)
    sig = torch.cat(cols, 1)
    return len(occ), float(torch.linalg.vector_norm(sig - sig64) / torch.linalg.vector_norm(sig64))


def test_first_order_pulse_map_reaches_the_stepped_signal():
    """With exact targets, the first-order map puts the TSE within 2e-4 of the stepped float64 signal, while the
    relax / rotate / relax splitting alone is off by more than 1e-2 (the 16 refocusing pulses of each echo train
    compound it): the first-order terms are what lets the surrogate reach 1e-3 at all."""
    n_occ, e_first = _tse_through_maps(16, True)
    _, e_split = _tse_through_maps(16, False)
    print(f"\nTSE 16^2 x 3 slices, {n_occ} occurrences: first-order map {e_first:.2e}, splitting alone {e_split:.2e}")
    assert n_occ > 0
    assert e_first < 2e-4
    assert e_split > 1e-2
