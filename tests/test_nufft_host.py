"""The NUFFT readout's host side (``blochparty_b200.nufft``) on the CPU: the runs it finds, the windows it plans,
and its tables, by a float64 emulation of the spreading and of the grid's DFT (the arithmetic of
``bp_forward_nufft`` and ``bp_nufft_finish``) against the direct sum over spins of every run sample."""

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import _lib, engine, nufft, phantoms, sequences

F64 = torch.float64


def _case(n_spins=6000, nx=64, seed=0):
    g = torch.Generator().manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    ph = bpb.Phantom(pos=(rnd(n_spins, 3) - 0.5) * 0.24, pd=rnd(n_spins), t1=0.3 + rnd(n_spins),
                     t2=0.02 + 0.1 * rnd(n_spins), db0=(rnd(n_spins) - 0.5) * 200)
    seq = sequences.gre((4, 4, nx), 0.25, flip_deg=20.0, tr=6e-3, te=2.5e-3, dwell=10e-6, n_echoes=2,
                        echo_spacing=1.5e-3)
    coils = phantoms.birdcage_sensitivities(ph.pos, 4)
    inp = bpb.api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase,
                         None, list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    return inp, seq


def test_runs_are_the_dwell_samples_of_every_readout():
    inp, seq = _case()
    pk = engine.pack(inp, "cpu")
    runs = nufft.find_runs(pk.flags)
    # every readout: a half-dwell sample, then nx - 1 dwell samples with one factor set (the run)
    assert len(runs) == 16 * 2 and all(k == 63 for _, k in runs)
    adc = np.asarray(seq.adc)
    for a, k in runs:
        assert adc[a:a + k].all() and not adc[a - 2] if a >= 2 else True


def test_windows_hold_each_run_alone_and_keep_the_rows():
    inp, _ = _case()
    pk = engine.pack(inp, "cpu")
    p = nufft.plan(pk.spins.numpy(), pk.segs.numpy(), pk.seg64.numpy(), pk.flags)
    win, run_of, rows = nufft.windows_for(p, pk.flags, _lib.lib().bp_forward_samp_max(pk.n_coils))
    assert win[0, 0] == 0 and win[-1, 1] == pk.flags.shape[0] and (win[1:, 0] == win[:-1, 1]).all()
    adc = (pk.flags & engine.ADC) != 0
    before = np.concatenate([[0], np.cumsum(adc)])
    for w, (s0, s1, z, cnt) in enumerate(win):
        assert z == before[s0]
        if run_of[w] >= 0:
            a, k = p.runs[run_of[w]]
            assert (s0, s1 - s0, cnt) == (a, k, 0) and rows[run_of[w]] == z
        else:
            assert cnt == adc[s0:s1].sum() and cnt <= _lib.lib().bp_forward_samp_max(pk.n_coils)
    assert sorted(run_of[run_of >= 0].tolist()) == list(range(len(p.runs)))


def test_tables_reproduce_the_direct_sum():
    """One run: the spins (sorted by the plan) spread z1 exp(-2 pi i x h) decay_m psi onto the grid, the grid's DFT
    times the weights, against sum_j z1_j q_j^p in float64: within 2e-7 (the float32 tables)."""
    inp, _ = _case()
    pk0 = engine.pack(inp, "cpu")
    p = nufft.plan(pk0.spins.numpy(), pk0.segs.numpy(), pk0.seg64.numpy(), pk0.flags)
    pk = engine.pack(nufft.sorted_inputs(inp, p.order), "cpu")
    spins, segs, seg64 = pk.spins.numpy(), pk.segs.numpy(), pk.seg64.numpy()
    base, frac, shift, decay, tiles = nufft.spin_tables(p, spins, segs, seg64)
    # sorted: a tile of 128 spins reaches its W cells plus the few its x range spans; they fit the accumulator
    assert ((tiles[:, 1] - tiles[:, 0]) * p.M <= 64).all() and (tiles[:, 1] - tiles[:, 0]).min() >= p.W
    a0 = int(p.runs[0, 0])
    x = nufft.run_phase(spins, segs[a0], seg64[a0])
    assert (np.diff(x) >= 0).all()
    g = np.random.default_rng(1)
    n = spins.shape[1]
    z1 = g.normal(size=n) + 1j * g.normal(size=n)
    r2 = spins[5].astype(np.float64)
    dt = float(segs[a0, 0])
    pidx = np.arange(p.L)
    direct = (z1[None, :] * np.exp(-2j * np.pi * np.outer(pidx, x) - np.outer(pidx * dt, r2))).sum(1)
    grid = np.zeros((p.G, p.M), complex)
    w0 = z1 * (shift[:, 0] + 1j * shift[:, 1])
    for w in range(p.W):
        z = 2.0 / p.W * (w - (p.W // 2 - 1) - frac.astype(np.float64))
        psi = np.exp(p.beta * (np.sqrt(np.maximum(0.0, 1.0 - z * z)) - 1.0))
        for m in range(p.M):
            np.add.at(grid[:, m], (base + w) % p.G, w0 * psi * decay[m])
    kap = pidx - p.L // 2
    gi = np.arange(p.G)
    dft = np.exp(-2j * np.pi * np.outer(kap, gi) / p.G)
    out = (p.weights.T * (dft @ grid)).sum(1)
    err = np.linalg.norm(out - direct) / np.linalg.norm(direct)
    assert err < 2e-7, err


def test_refusals():
    with pytest.raises(ValueError, match="too few spins"):
        inp, _ = _case(n_spins=300)
        pk = engine.pack(inp, "cpu")
        p = nufft.plan(pk.spins.numpy(), pk.segs.numpy(), pk.seg64.numpy(), pk.flags)
        nufft.spin_tables(p, pk.spins[:, torch.from_numpy(p.order)].numpy(), pk.segs.numpy(), pk.seg64.numpy())
    with pytest.raises(ValueError, match="more than"):
        nufft.terms_for(1e4, 1.27e-3)
    assert nufft.terms_for(1.0 / 0.02, 1.26e-3) == 4 and nufft.terms_for(1.0 / 0.07, 1.26e-3) == 3


def test_device_preparation_matches_the_host_tables():
    """``nufft.prepare`` (one packing, the sort and the tables in torch on the target device; here the CPU) gives
    the order and the tables of the host restatement (``plan``, ``spin_tables``): the same order, cells and decay
    terms, and fractions and shifts within a float32 ulp."""
    inp, _ = _case()
    pk0 = engine.pack(inp, "cpu")
    p = nufft.plan(pk0.spins.numpy(), pk0.segs.numpy(), pk0.seg64.numpy(), pk0.flags)
    pk_h = engine.pack(nufft.sorted_inputs(inp, p.order), "cpu")
    base, frac, shift, decay, tiles = nufft.spin_tables(p, pk_h.spins.numpy(), pk_h.segs.numpy(), pk_h.seg64.numpy())
    pk, nr, order = nufft.prepare(inp, torch.device("cpu"))
    assert np.array_equal(order.numpy(), p.order)
    assert torch.equal(pk.spins, pk_h.spins) and torch.equal(pk.sens, pk_h.sens)
    assert np.array_equal(nr.base.numpy(), base) and np.array_equal(nr.tiles.numpy(), tiles)
    assert np.abs(nr.frac.numpy() - frac).max() <= 1e-6
    assert np.abs(nr.shift.numpy() - shift).max() <= 2e-7
    assert np.abs(nr.decay.numpy() - decay).max() <= 1e-7
    assert (nr.plan.M, nr.plan.L, nr.plan.G) == (p.M, p.L, p.G) and np.array_equal(nr.plan.runs, p.runs)
