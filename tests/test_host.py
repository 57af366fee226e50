"""Host-side checks that need no GPU: the C ABI library loads and exports what the header declares, the native
window planner, the packing of segments and state, the capability refusals and argument errors of ``simulate``."""

import ctypes
import re
from dataclasses import replace
from pathlib import Path

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import _lib, capabilities, engine, physics, sequences

ROOT = Path(__file__).resolve().parents[1]
F64 = torch.float64


def declared_functions():
    text = (ROOT / "include" / "blochparty_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(bp_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load_library()
    names = declared_functions()
    assert len(names) >= 4
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_planner_windows_cover_the_sequence():
    g = np.random.default_rng(0)
    flags = (g.random(5000) < 0.3).astype(np.int32) | ((g.random(5000) < 0.4).astype(np.int32) << 1)
    for samp in (1, 7, 64):
        w = engine.plan_windows(flags, samp, seg_max=100)
        assert w[0, 0] == 0 and w[-1, 1] == 5000
        assert (w[1:, 0] == w[:-1, 1]).all()
        assert ((w[:, 1] - w[:, 0]) <= 100).all() and (w[:, 3] <= samp).all()
        # cuts by a limit fall on multiples of BP_ADJ_WIN segments whenever the window keeps one
        limited = w[:-1, 1]
        assert all(e % _lib.BP_ADJ_WIN == 0 or e - a < _lib.BP_ADJ_WIN or e // _lib.BP_ADJ_WIN * _lib.BP_ADJ_WIN <= a
                   for a, e in zip(w[:-1, 0], limited))
        adc = (flags & 2) != 0
        counts = np.array([adc[a:b].sum() for a, b in w[:, :2]])
        assert (counts == w[:, 3]).all()
        assert (w[:, 2] == np.concatenate([[0], np.cumsum(counts)[:-1]])).all()


def test_planner_breaks_and_errors():
    flags = np.zeros(10, np.int32)
    br = np.zeros(10, np.uint8)
    br[[3, 7]] = 1
    w = engine.plan_windows(flags, 4, seg_max=_lib.BP_SEG_MAX, breaks=br)
    assert w[:, 0].tolist() == [0, 3, 7]
    lib = _lib.lib()
    out = np.zeros((1, 4), np.int32)
    nw = np.zeros(1, np.int64)
    assert lib.bp_plan_windows(flags.ctypes.data, 10, 4, 4, None, out.ctypes.data, 1, nw.ctypes.data) == _lib.BP_E_SIZE
    assert lib.bp_plan_windows(flags.ctypes.data, 10, _lib.BP_SEG_MAX + 1, 4, None, out.ctypes.data, 9,
                               nw.ctypes.data) == _lib.BP_E_ARG
    assert lib.bp_forward_samp_max(8) > 0 and lib.bp_forward_samp_max(33) == 0 and lib.bp_forward_samp_max(0) == 0


def test_segment_records():
    b = sequences.SequenceBuilder().rf(1e-4, flip_deg=30.0, phase=0.5, n_steps=2, grad=(0, 0, 100.0))
    b.readout(4, 1e-5, grad=(1000.0, 0.0, 0.0)).delay(1e-3).spoil()
    seq = b.build()
    seq.b0_offset = torch.full((len(seq),), 3.0, dtype=F64)
    rec, seg64, psi, flags, n_adc = engine.pack_segments(seq.dt, seq.rf, seq.grad, seq.b0_offset, seq.adc_phase,
                                                         seq.is_rf, seq.adc, seq.spoil, "cpu")
    assert rec.shape == (len(seq), 8) and rec.dtype == torch.float32 and n_adc == 4
    # the second RF step has the first's dt and offset; the first sample is half a dwell: not "same"
    assert flags.tolist() == [1, 1 | 16 | 32, 2, 2, 2 | 8, 2 | 8, 0, 4]
    assert abs(float(rec[0, 1]) - (-2 * np.pi * 5e-5 * float(seq.rf[0, 0]))) < 1e-6
    assert float(seg64[3, 0]) == 1000.0 * 1e-5 and float(seg64[3, 3]) == 3.0 * 1e-5
    assert rec.view(torch.int32)[:, 7].tolist() == flags.tolist()


def test_small_rf_marks_follow_the_rotation_bound():
    """SMALL goes on the RF segments whose |w|^2 is below 0.0624 for every spin (b1 and the positions' extents
    bounding it), in the device records and the host flags alike; never on a free segment."""
    b = sequences.SequenceBuilder().rf(1e-4, flip_deg=30.0, n_steps=10, grad=(0, 0, 100.0))
    b.readout(4, 1e-5, grad=(1000.0, 0.0, 0.0))
    seq = b.build()
    rec, _, _, flags, _ = engine.pack_segments(seq.dt, seq.rf, seq.grad, None, seq.adc_phase, seq.is_rf, seq.adc,
                                               seq.spoil, "cpu")

    def marks(z_max, b1):
        pos = torch.zeros(2, 3, dtype=F64)
        pos[1, 2] = z_max
        spins, _ = engine.pack_spins(pos, torch.ones(2, dtype=F64), torch.ones(2, dtype=F64),
                                     torch.full((2,), 0.1, dtype=F64), torch.zeros(2, dtype=F64),
                                     torch.full((2,), b1, dtype=F64), torch.ones(2, 1, dtype=torch.complex128), "cpu")
        r, f = rec.clone(), flags.copy()
        engine.mark_small_rf(spins, r, f)
        assert r.view(torch.int32)[:, 7].tolist() == f.tolist()
        return (f & engine.SMALL) != 0

    rf = np.asarray(seq.is_rf)
    # 30 degrees over 10 steps: 0.052 rad per step, and 2 pi 100 Hz/m 1e-5 s z: small up to z of a few metres
    assert (marks(0.1, 1.0) == rf).all()
    assert not marks(100.0, 1.0).any()     # the off-resonance of a spin far out in the slice gradient
    assert not marks(0.1, 6.0).any()       # B1 scale 6: |w| = 0.31 > 1/4
    assert not (marks(0.1, 1.0) & ~rf).any()


@pytest.mark.parametrize("workload", ["gre3d_16", "head_16"])
def test_adjoint_windows_follow_runs_and_not_intervals(workload):
    """The adjoint's windows (32-segment blocks cut again at every run start): the same for every checkpoint
    interval (a multiple of 32), every window one RF run or one free run (spoiling at most last), and no cut inside
    a readout run of the forward kernel (whose merged arithmetic a cut would change)."""
    from blochparty_b200 import adjoint, workloads

    if workload == "gre3d_16":
        _, seq, _ = workloads.gre3d_64(16)
    else:
        _, seq, _ = workloads.gre3d_128_4echo(16)
    flags = engine.pack_segments(seq.dt, seq.rf, seq.grad, None, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                                 list(seq.spoil), "cpu")[3]
    S, w = len(flags), _lib.BP_ADJ_WIN
    rb = adjoint.run_breaks(flags)
    plans = []
    for every in (w * 2, w * 37, w * 1000):
        br = np.zeros(S, dtype=np.uint8)
        br[::every] = 1
        plans.append(engine.plan_windows(flags, w, seg_max=w, breaks=br | rb))
    assert all(np.array_equal(plans[0], p) for p in plans[1:])
    win = plans[0]
    for s0, s1, _, _ in win.tolist():
        f = flags[s0:s1]
        rf = (f & engine.RF) != 0
        assert rf.all() or (~rf).all(), (s0, s1)
        assert not (f[:-1] & engine.SPOIL).any(), (s0, s1)
        same = engine.SAME_OFF if rf[0] else engine.SAME_FREE
        assert ((f[1:] & same) != 0).all(), (s0, s1)
        if s0 % w and s0 > 0:  # a cut the 32-segment blocks do not make: not inside a readout run
            prev, cur = int(flags[s0 - 1]), int(flags[s0])
            inside = ((cur & ~engine.SPOIL) & 0x3F) == (engine.ADC | engine.SAME_FREE) and (prev & engine.ADC) \
                and not (prev & (engine.SPOIL | engine.RF))
            assert not inside, s0


def test_initial_state_split_is_exact():
    pd = torch.rand(100, dtype=F64)
    m = torch.rand(100, 3, dtype=F64)
    s = engine.initial_state(pd, m, "cpu")
    assert torch.equal(s[0:3].to(F64) + s[3:6].to(F64), m.T) or (
        (s[0:3].to(F64) + s[3:6].to(F64) - m.T).abs().max() < 1e-14)


def _tiny():
    ph = bpb.Phantom(torch.zeros(2, 3, dtype=F64), torch.ones(2, dtype=F64), torch.ones(2, dtype=F64),
                     torch.full((2,), 0.1, dtype=F64), torch.zeros(2, dtype=F64))
    return ph, sequences.SequenceBuilder().rf(1e-4, flip_deg=10.0).readout(4, 1e-5).build()


def test_refusals_use_the_reference_wording():
    ph, seq = _tiny()
    ph.diffusion = torch.ones(2, dtype=F64)
    with pytest.raises(NotImplementedError, match=r"b200 engine: simulating with diffusion \(Phantom.diffusion\) "
                                                  r"is not implemented; use blochparty.simulate \(the core\)"):
        bpb.simulate(ph, seq)
    ph.diffusion = None
    pool = physics.BoundPool(0.1, 30.0, 1.0, 12e-6)
    with pytest.raises(NotImplementedError, match=r"gradients through a bound pool \(Phantom.bound\)"):
        bpb.simulate(replace(ph, t1=ph.t1.clone().requires_grad_(), bound=pool), seq)
    b0 = torch.tensor(0.55, dtype=F64, requires_grad=True)  # a gradient through the scanner alone is one
    assert bpb.api.requires_grad(ph, seq, None, None, physics.Scanner(b0))
    with pytest.raises(NotImplementedError, match=r"simulating with field maps \(FieldMaps\)"):
        bpb.simulate(ph, seq, maps=object())
    gen = replace(ph, bound=physics.BoundPool(0.1, 30.0, 1.0, 12e-6, model="generalized"))
    with pytest.raises(NotImplementedError, match="the generalized Bloch bound pool"):
        bpb.simulate(gen, seq)
    seq.bound_only = [True] + [False] * (len(seq) - 1)
    with pytest.raises(NotImplementedError, match="gradients through .*bound-pool-only"):
        bpb.simulate(replace(ph, t1=ph.t1.clone().requires_grad_()), seq)
    used = capabilities.features(ph, seq, torch.zeros(2, 3))
    assert "m_init" in used and "bound_only" in used
    with pytest.raises(ValueError, match="m_init has a bound-pool column"):
        bpb.simulate(ph, seq, m_init=torch.zeros(2, 4))


def test_argument_errors():
    ph, seq = _tiny()
    with pytest.raises(TypeError, match="unexpected keyword argument"):
        bpb.simulate(ph, seq, spin_chunk=4)
    with pytest.raises(ValueError, match="readouts must be"):
        bpb.simulate(ph, seq, readouts="fast")
    with pytest.raises(ValueError, match="disagree"):
        bpb.simulate(ph, seq, readouts="nufft", readout="fp32")
    from blochparty_b200.api import _reference_options
    assert _reference_options({"readouts": "nufft", "chunk": 4096, "group": 128, "mma": True, "nufft_width": 6,
                               "nufft_terms": 3}) == {"readout": "nufft"}
    assert _reference_options({"readouts": "direct"}) == {"readout": "fp32"}
    with pytest.raises(ValueError, match="merge_free_runs=False"):
        bpb.simulate(ph, seq, merge_free_runs=False)
    with pytest.raises(ValueError, match="engine must be one of"):
        bpb.simulate(ph, seq, engine="metal")
    with pytest.raises(ValueError, match="readout must be"):
        bpb.simulate(ph, seq, readout="tf32")
    with pytest.raises(ValueError, match=r"coils must be \(N, C\)"):
        bpb.simulate(ph, seq, torch.ones(3, 1, dtype=torch.complex64))


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error")
def test_no_gpu_fails_loudly():
    ph, seq = _tiny()
    with pytest.raises(RuntimeError, match="needs a CUDA device"):
        bpb.simulate(ph, seq)


def test_span_descriptor_layout_matches_the_header(tmp_path):
    """The ctypes ``BpSpan`` has the C struct's size and field offsets (compiled against the header with gcc)."""
    import ctypes
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    fields = [f for f, _ in _lib.BpSpan._fields_]
    src = tmp_path / "span.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "blochparty_b200.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof(BpSpan, {f}));\n' for f in fields)
                   + '  printf("%zu\\n", sizeof(BpSpan));\n  return 0;\n}\n')
    exe = tmp_path / "span"
    inc = Path(__file__).resolve().parents[1] / "include"
    subprocess.run(["gcc", f"-I{inc}", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [getattr(_lib.BpSpan, f).offset for f in fields] + [ctypes.sizeof(_lib.BpSpan)]
    assert got == want


def test_workspace_query_matches_the_host_allocations():
    """``bp_forward_workspace_bytes`` / ``bp_adjoint_workspace_bytes`` give the sizes of the buffers the host side
    allocates (``adjoint.sized`` checks every allocation against them); here the same shapes, from a plan of the
    4-echo head workload at 16^3 with a 37-window checkpoint interval, against the query."""
    from blochparty_b200 import adjoint, workloads

    ph, seq, coils = workloads.gre3d_128_4echo(16)
    inp = bpb.api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad,
                         seq.adc_phase, None, list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    pk = engine.pack(inp, "cpu")
    every = 37 * _lib.BP_ADJ_WIN
    plan = adjoint.Plan(pk, every, "cpu")
    n, S, A, C, grid = pk.n, pk.flags.shape[0], pk.n_adc, pk.n_coils, 592
    f = _lib.forward_workspace(n, A, C)
    assert (f.state, f.raw, f.psi, f.signal) == (6 * n * 4, A * 2 * C * 8, pk.psi.numel() * 8, C * A * 8)
    w = _lib.adjoint_workspace(n, S, A, C, every, plan.max_aw, grid)
    assert w.checkpoints == len(plan.starts) * 6 * n * 4
    assert w.wstates == (plan.max_aw + 1) * 6 * n * 4
    assert w.gseg == grid * plan.max_len * 8 * 4
    assert (w.seg, w.lam, w.gs, w.gc, w.h) == (S * 64, 3 * n * 4, 8 * n * 4, 2 * C * n * 4, A * 2 * C * 4)
    assert w.total == sum(getattr(w, k) for k in ("checkpoints", "wstates", "replay_state", "gseg", "seg", "lam",
                                                   "gs", "gc", "h"))
    lib = _lib.lib()
    assert lib.bp_adjoint_workspace_bytes(n, S, A, C, every + 1, plan.max_aw, grid, 0, None) == _lib.BP_E_ARG
    # the outer level: the block starts plus one block's interval starts
    k = len(plan.starts)
    wo = _lib.adjoint_workspace(n, S, A, C, every, plan.max_aw, grid, 2)
    assert wo.checkpoints == ((k + 1) // 2 + min(k, 2)) * 6 * n * 4
    assert lib.bp_forward_workspace_bytes(n, A, 33, None) == _lib.BP_E_ARG


def test_workspace_structs_match_the_header(tmp_path):
    """The ctypes workspace, NUFFT and physics structs have the C structs' sizes and field offsets (compiled with
    gcc)."""
    import ctypes
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    inc = Path(__file__).resolve().parents[1] / "include"
    for struct in (_lib.BpForwardWorkspace, _lib.BpAdjointWorkspace, _lib.BpNufft, _lib.BpPhysics):
        name = struct.__name__
        fields = [f for f, _ in struct._fields_]
        src = tmp_path / f"{name}.c"
        src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "blochparty_b200.h"\nint main(void) {\n'
                       + "".join(f'  printf("%zu\\n", offsetof({name}, {f}));\n' for f in fields)
                       + f'  printf("%zu\\n", sizeof({name}));\n  return 0;\n}}\n')
        exe = tmp_path / name
        subprocess.run(["gcc", f"-I{inc}", str(src), "-o", str(exe)], check=True)
        got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
        assert got == [getattr(struct, f).offset for f in fields] + [ctypes.sizeof(struct)]


def test_checkpoint_choice():
    """Two levels while their states fit the budget, three beyond it (about 3 (S/32)^(1/3) states)."""
    from blochparty_b200 import adjoint

    assert adjoint.choose_checkpoints(1_110_016, 1 << 20, budget_bytes=40 << 30)[1] == 0
    every, outer = adjoint.choose_checkpoints(11_829_248, 8_388_608, budget_bytes=80 << 30)
    assert outer > 1 and every % 32 == 0
    k = -(-11_829_248 // every)
    states = -(-k // outer) + outer + every // 32 + 1
    assert states * 24 * 8_388_608 < 80 << 30


def test_saved_states_plan():
    """The backward from saved states: on the 4-echo head sequence every adjoint window is a run of RF or of free
    segments, one state is saved per TR (after its slab pulse, at the first segment that is not RF), and the
    forward's windows start there too; a window that mixes RF and free segments leaves it to the replay."""
    from blochparty_b200 import adjoint, workloads

    _, seq, _ = workloads.gre3d_128_4echo(16)
    seq = workloads.first_n_trs(seq, 5)
    flags = engine.pack_segments(seq.dt, seq.rf, seq.grad, None, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                                 list(seq.spoil), "cpu")[3]
    S, w = len(flags), _lib.BP_ADJ_WIN
    br = np.zeros(S, dtype=np.uint8)
    br[::64] = 1
    awin = engine.plan_windows(flags, w, seg_max=w, breaks=br | adjoint.run_breaks(flags))
    sv = adjoint.SavedStates.of(flags, awin)
    assert sv is not None and sv.n_slots == 5 and not sv.final
    rf = (flags & engine.RF) != 0
    pulse_ends = np.flatnonzero(rf[:-1] & ~rf[1:]) + 1
    assert np.array_equal(sv.points, pulse_ends)
    assert np.array_equal(np.flatnonzero(sv.slot >= 0), np.searchsorted(awin[:, 0], pulse_ends))
    assert (sv.rf == (np.add.reduceat(rf.astype(int), awin[:, 0]) > 0)).all()
    # a sample at the end of an RF segment: that window needs its states recomputed (no saved plan)
    mixed = flags.copy()
    mixed[int(np.flatnonzero(rf)[3])] |= engine.ADC
    assert adjoint.SavedStates.of(mixed, awin) is None
    # a sequence ending in an RF run saves the final state as its last slot
    sub = flags[: pulse_ends[1] - 5]
    sv2 = adjoint.SavedStates.of(sub, engine.plan_windows(sub, w, seg_max=w, breaks=adjoint.run_breaks(sub)))
    assert sv2 is not None and sv2.final and sv2.n_slots == 2 and list(sv2.points) == [pulse_ends[0]]


def test_saved_entry_points_check_their_arguments():
    """bp_forward_saving and bp_adjoint_saved refuse a missing slot map, and the saved sweep refuses any gradient
    but the RF waveform's (argument checks only: no GPU call)."""
    lib = _lib.lib()
    one = ctypes.c_void_p(16)
    assert lib.bp_forward_saving(one, one, 4, 1, one, one, one, 0, 1, one, None, None, one, 0, one, None) \
        == _lib.BP_E_ARG
    args = lambda mask, wslot, chain: (one, one, 4, 1, one, one, one, 0, 1, 0, 32, one, wslot, chain, 0, None, 0,
                                       one, None, mask, 1, one, None)
    rf = _lib.BP_SEG_WX | _lib.BP_SEG_WY | _lib.BP_SPIN_NONE
    assert lib.bp_adjoint_saved(*args(rf, None, one)) == _lib.BP_E_ARG
    assert lib.bp_adjoint_saved(*args(rf, one, None)) == _lib.BP_E_ARG
    assert lib.bp_adjoint_saved(*args(rf | _lib.BP_SEG_DT, one, one)) == _lib.BP_E_ARG
    assert lib.bp_adjoint_saved(*args(_lib.BP_SEG_WX | _lib.BP_SEG_WY, one, one)) == _lib.BP_E_ARG


def test_saved_layout_in_blocks():
    """When the states saved after the RF runs do not fit, blocks of intervals: every block's sweep finds the
    states it needs (its own runs' and the one after its end) in distinct slots (run number mod the slot count),
    and the block starts plus the slots fit the budget."""
    from blochparty_b200 import adjoint, workloads

    _, seq, _ = workloads.gre3d_128_4echo(16)
    seq = workloads.first_n_trs(seq, 12)
    flags = engine.pack_segments(seq.dt, seq.rf, seq.grad, None, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                                 list(seq.spoil), "cpu")[3]

    class P:  # the parts of a Plan that saved_layout reads
        pass

    S, w, every = len(flags), _lib.BP_ADJ_WIN, 64
    plan = P()
    plan.starts = list(range(0, S, every))
    br = np.zeros(S, dtype=np.uint8)
    br[plan.starts] = 1
    plan.awin = engine.plan_windows(flags, w, seg_max=w, breaks=br | adjoint.run_breaks(flags))
    plan.saved = adjoint.SavedStates.of(flags, plan.awin)
    a0 = np.searchsorted(plan.awin[:, 0], plan.starts)
    plan.aranges = list(zip(a0.tolist(), list(a0[1:]) + [len(plan.awin)]))
    k = len(plan.starts)
    assert adjoint.saved_layout(plan, 1, 12) == (k, 12)  # all twelve fit
    K, cap = adjoint.saved_layout(plan, 1, 9)
    blocks = [(b, min(b + K, k)) for b in range(0, k, K)]
    assert len(blocks) > 1 and len(blocks) + cap <= 9
    run_of = np.cumsum(plan.saved.slot >= 0) - 1  # run number of each saved window start
    for ka, kb in blocks:
        lo, hi = plan.aranges[ka][0], plan.aranges[kb - 1][1]
        live = [int(run_of[e]) for e in range(lo, hi + 1) if plan.saved.slot[e] >= 0]
        assert len({r % cap for r in live}) == len(live), (ka, kb, live, cap)
    assert adjoint.saved_layout(plan, 1, 2) is None


@pytest.mark.parametrize("budget", [7, 9, 12, 40])
def test_saved_slots_protocol_in_blocks(budget):
    """The host's plan of the backward from saved states, replayed on the host with the slots as a dictionary: the
    forward writes every run's state into slot run mod cap (the block starts aside), each block but the last is
    rebuilt before its sweep, and every window of RF segments whose next window is not one reads the slot of the
    next window's start: it must hold that run's state, for every layout the budget allows (4-echo head sequence,
    12 TRs, intervals of 64 segments)."""
    from blochparty_b200 import adjoint, workloads

    _, seq, _ = workloads.gre3d_128_4echo(16)
    seq = workloads.first_n_trs(seq, 12)
    flags = engine.pack_segments(seq.dt, seq.rf, seq.grad, None, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                                 list(seq.spoil), "cpu")[3]
    S, w, every = len(flags), _lib.BP_ADJ_WIN, 64
    starts = list(range(0, S, every))
    br = np.zeros(S, dtype=np.uint8)
    br[starts] = 1
    awin = engine.plan_windows(flags, w, seg_max=w, breaks=br | adjoint.run_breaks(flags))
    sv = adjoint.SavedStates.of(flags, awin)

    class P:
        pass

    plan = P()
    plan.starts, plan.awin, plan.saved = starts, awin, sv
    a0 = np.searchsorted(awin[:, 0], starts)
    plan.aranges = list(zip(a0.tolist(), list(a0[1:]) + [len(awin)]))
    K, cap = adjoint.saved_layout(plan, 1, budget)
    k, W = len(starts), len(awin)
    run_of = {int(e): r for r, e in enumerate(np.flatnonzero(sv.slot >= 0))}  # window start -> run number
    slots = {}

    def write_block(ka, kb):  # the forward over intervals [ka, kb) saves the runs whose window starts lie there
        lo, hi = plan.aranges[ka][0], plan.aranges[kb - 1][1]
        for e in range(lo, hi):
            if e in run_of:
                slots[run_of[e] % cap] = run_of[e]

    blocks = [(b, min(b + K, k)) for b in range(0, k, K)]
    for ka, kb in blocks:
        write_block(ka, kb)
    if sv.final:
        slots[run_of[W] % cap] = run_of[W]
    for bi, (ka, kb) in reversed(list(enumerate(blocks))):
        if bi + 1 < len(blocks):
            write_block(ka, kb)
        for kk in reversed(range(ka, kb)):
            aa, ab = plan.aranges[kk]
            for win in range(ab - 1, aa - 1, -1):
                e = win + 1
                if sv.rf[win] and (e == W or not sv.rf[e]):  # the end of an RF run: its state is read
                    assert slots.get(run_of[e] % cap) == run_of[e], (budget, K, cap, win)
