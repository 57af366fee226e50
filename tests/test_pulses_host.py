"""Finding reused pulses on the host (``blochparty_b200.pulses.find_reused``): the groups, their occurrences and
phases on the workloads' sequences, and the rules kept from blochparty ``engines/gpu/driver.py:112-164`` (runs of
two or more RF segments without samples, cut after a spoil; equal up to a global RF phase)."""

import math

import numpy as np
import torch

from blochparty_b200 import pulses, sequences, workloads
from blochparty_b200.api import Inputs

F64 = torch.float64


def _inputs(ph, seq, coils):
    return Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase,
                  getattr(seq, "b0_offset", None), list(seq.is_rf), list(seq.adc), list(seq.spoil), None)


def _phase_of(seq, a, s, k):
    z = (seq.rf[:, 0] + 1j * seq.rf[:, 1]).numpy()
    c = np.vdot(z[a:a + k], z[s:s + k])
    return float(np.angle(c))


def test_rf_spoiled_gre_is_one_pulse_with_the_spoiling_phases():
    ph, seq, coils = workloads.gre3d_64(8)
    groups = pulses.find_reused(_inputs(ph, seq, coils))
    assert len(groups) == 1
    a, k, occ = groups[0]
    assert k == 200 and len(occ) == seq.meta["n_tr"] + seq.meta.get("n_dummy", 0)
    assert occ[0] == (a, 0.0)
    for s, p in occ[1:50]:
        assert abs(math.remainder(p - _phase_of(seq, a, s, k), 2 * math.pi)) < 1e-9


def test_tse_pulses_group_by_slice_and_kind():
    ph, seq, coils = workloads.tse_3slice_128(32)  # ETL 16: two shots per slice
    groups = pulses.find_reused(_inputs(ph, seq, coils))
    assert len(groups) == 6  # 3 slices x (excitation, refocusing)
    counts = sorted(len(o) for _, _, o in groups)
    assert counts == [2] * 3 + [32] * 3
    assert all(k == 300 for _, k, _ in groups)
    # most saved segments first
    saved = [(len(o) - 1) * k for _, k, o in groups]
    assert saved == sorted(saved, reverse=True)


def test_runs_skip_samples_and_cut_after_spoil():
    b = sequences.SequenceBuilder()
    w = np.ones((4, 2)) * 100.0
    for rep in range(3):
        b.rf_waveform(w, 1e-5)
        b.delay(1e-3)
    b.rf_waveform(w, 1e-5)
    seq = b.build()
    n = 4
    ph = workloads.Phantom(torch.zeros(n, 3, dtype=F64), torch.ones(n, dtype=F64), torch.ones(n, dtype=F64),
                           torch.full((n,), 0.1, dtype=F64), torch.zeros(n, dtype=F64))
    inp = _inputs(ph, seq, torch.ones(n, 1, dtype=torch.complex128))
    groups = pulses.find_reused(inp)
    assert len(groups) == 1 and len(groups[0][2]) == 4 and groups[0][1] == 4
    # a spoil inside a run cuts it after the spoiled segment
    spoil = list(inp.spoil)
    spoil[1] = True
    inp.spoil = spoil
    groups = pulses.find_reused(inp)
    lens = sorted({k for _, k, _ in groups})
    assert 4 in lens  # the three runs without the spoil still recur
    starts, lens = pulses._runs(np.asarray(inp.is_rf), np.asarray(inp.adc), np.asarray(spoil))
    assert (starts[0], lens[0]) == (0, 2) and (starts[1], lens[1]) == (2, 2)
