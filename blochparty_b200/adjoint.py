"""Gradients: the forward with checkpoints and the hand-written adjoint behind a ``torch.autograd.Function``.

Replaces blochparty ``engines/gpu/adjoint.py`` (``_GPUSimulate`` :45-261, ``_simulate_grad`` :264-323) for static
spins. The forward stores the state at the start of every checkpoint interval (``checkpoint_every`` segments, a
multiple of ``BP_ADJ_WIN`` = 32). The backward walks the intervals in reverse: it replays an interval with the
forward kernel, storing the state at every 32-segment window start, then runs ``bp_adjoint`` over it (each window
recomputed into shared memory and swept backward) and ``bp_seg_reduce`` (segment gradients summed over CTAs in
fixed order, float64). Windows fall on multiples of 32 segments whatever the interval, so the gradients are the
same bits for every ``checkpoint_every`` and every run.

For the RF waveform's gradient alone, on sequences whose adjoint windows are all runs of RF segments or of free
segments (every GRE here), the forward saves instead the state after each RF run (``bp_forward_saving``) and the
backward sweeps every interval from those states with no replay (``bp_adjoint_saved``): its RF windows integrate
their states backward from the state after the pulse, its free windows carry lambda alone (``SavedStates``,
``saved_layout``; in blocks, each block's states rebuilt by one forward of the block, when they do not all fit).

Chain rules on the host (float64), from the kernels' raw gradients: r1 = 1/T1 -> dL/dT1 = -dL/dr1 / T1^2; the
segment record (dt, w_x = -2 pi dt rf_x, w_y, k = g dt, beta = b0_offset dt) -> dL/d(dt, rf, grad, b0_offset);
the receiver phase: signal = raw exp(-i psi), so dL/dpsi = gr Im(signal) - gi Re(signal) (blochparty
``adjoint.py:241-245``).
"""

from __future__ import annotations

import math

import numpy as np
import torch
from torch.autograd.function import once_differentiable

from . import _lib, engine
from ._lib import ptr
from .types import SimResult

F32, F64 = torch.float32, torch.float64
TWO_PI = 2.0 * math.pi


def sized(nbytes: int, shape, dtype, device, zero: bool = False) -> torch.Tensor:
    """A device buffer of ``shape`` whose size is the C ABI's workspace figure ``nbytes`` (checked)."""
    t = (torch.zeros if zero else torch.empty)(*shape, dtype=dtype, device=device)
    if t.numel() * t.element_size() != nbytes:
        raise RuntimeError(f"buffer {tuple(shape)} {dtype}: {t.numel() * t.element_size()} bytes, the workspace "
                           f"query says {nbytes}")
    return t


def default_checkpoint_every(n_segments: int) -> int:
    """About sqrt(32 x segments), a multiple of the 32-segment adjoint window: the interval that minimises the
    stored states, S / every checkpoints plus every / 32 window starts of one replayed interval (each segment is
    replayed once whatever the interval)."""
    w = _lib.BP_ADJ_WIN
    return w * max(1, math.ceil(math.sqrt(w * max(n_segments, 1)) / w))


def choose_checkpoints(n_segments: int, n_spins: int, budget_bytes: int | None = None) -> tuple[int, int]:
    """(checkpoint_every, outer_every) for a sequence of ``n_segments`` on ``n_spins``: the two-level scheme of
    ``default_checkpoint_every`` (outer_every 0) when its stored states (interval starts plus one interval's window
    starts, 24 bytes per spin each) fit ``budget_bytes`` (default: half the device's free memory), else three
    levels with the cube root of the window count for each (intervals of that many windows, blocks of that many
    intervals): about 3 (S / 32)^(1/3) states instead of 2 (S / 32)^(1/2), for one more forward."""
    w = _lib.BP_ADJ_WIN
    every = default_checkpoint_every(n_segments)
    per_state = 24 * max(n_spins, 1)
    two = (math.ceil(max(n_segments, 1) / every) + every // w + 1) * per_state
    if budget_bytes is None:
        budget_bytes = torch.cuda.mem_get_info()[0] // 2 if torch.cuda.is_available() else 1 << 62
    if two <= budget_bytes:
        return every, 0
    root = max(2, math.ceil((max(n_segments, 1) / w) ** (1.0 / 3.0)))
    return w * root, root


def run_breaks(flags: np.ndarray) -> np.ndarray:
    """Window breaks for the adjoint at the start of every run of like segments: where RF and free segments
    alternate, where an RF segment changes dt or offset, where a free segment changes its factors, and after every
    spoiling segment, and at every multiple of 32 segments. The sweep runs a window whose segments are all one RF
    run, or all one free run (spoiling at most in its last segment), without per-segment tests. The windows are
    the 32-segment blocks cut at these breaks: the checkpoint intervals (multiples of 32) add no cut, so every
    window, its recompute and the gradients keep the same bits for every interval. No break falls inside a
    readout run of the forward kernel (samples with one segment's factors, the last of which may spoil, cut at
    32-segment blocks), whose arithmetic would change with a cut: the replayed states keep their bits too."""
    S = flags.shape[0]
    out = np.zeros(S, dtype=np.uint8)
    if S < 2:
        return out
    rf = (flags & engine.RF) != 0
    spoil = (flags & engine.SPOIL) != 0
    same_off = (flags & engine.SAME_OFF) != 0
    same_free = (flags & engine.SAME_FREE) != 0
    cut = (rf[1:] != rf[:-1]) | (rf[1:] & ~same_off[1:]) | (~rf[1:] & ~same_free[1:]) | spoil[:-1]
    out[1:] = cut
    out[::_lib.BP_ADJ_WIN] = 1
    return out


class SavedStates:
    """Where the backward without a replay (``bp_adjoint_saved``) needs states: for adjoint windows ``awin`` whose
    every window is either RF segments with one dt and offset, no sample and no spoil (``rf[w]``: integrated backward
    from the state after it), or free segments with one set of factors spoiling at most in its last segment (lambda
    alone), the state after each run of RF windows. ``slot`` [W + 1] int32: the slot of the state at window w's start
    (-1: none); ``points``: the segments whose start states are saved, slots 0, 1, ... in order, and ``final``
    whether the state after the last segment is saved too (the last slot). ``of(flags, awin)`` is None when some
    window is of neither kind."""

    def __init__(self, rf, slot, points, final):
        self.rf, self.slot, self.points, self.final = rf, slot, points, final
        self.n_slots = len(points) + int(final)

    @classmethod
    def of(cls, flags: np.ndarray, awin: np.ndarray):
        W = awin.shape[0]
        if W == 0:
            return None
        s0, s1 = awin[:, 0].astype(np.int64), awin[:, 1].astype(np.int64)
        if (s1 <= s0).any():
            return None
        count = lambda b: np.add.reduceat(b.astype(np.int64), s0)  # per window
        is_rf = (flags & engine.RF) != 0
        spoil = (flags & engine.SPOIL) != 0
        no_off = (flags & engine.SAME_OFF) == 0
        no_free = (flags & engine.SAME_FREE) == 0
        rf = ((count(~is_rf) == 0) & (count((flags & (engine.ADC | engine.SPOIL)) != 0) == 0)
              & (count(no_off) - no_off[s0] == 0))
        free = (count(is_rf) == 0) & (count(spoil) - spoil[s1 - 1] == 0) & (count(no_free) - no_free[s0] == 0)
        if not (rf | free).all():
            return None
        nxt = np.append(rf[1:], False)
        ends = np.flatnonzero(rf & ~nxt) + 1  # windows (or W: the end) whose start follows a run of RF windows
        slot = np.full(W + 1, -1, dtype=np.int32)
        slot[ends] = np.arange(len(ends), dtype=np.int32)
        final = bool(len(ends) and ends[-1] == W)
        points = awin[ends[:-1] if final else ends, 0].astype(np.int64)
        return cls(rf, slot, points, final)


def rf_relaxation_invertible(pk: engine.Packed) -> bool:
    """Whether every spin's half-step relaxation over every RF segment keeps 1 + expm1(-dt r / 2) >= 1/2 (the
    backward integration divides by it) with a margin: dt r <= 1.35 (2 ln 2 = 1.386) for the longest RF segment."""
    rf = (pk.flags & engine.RF) != 0
    if not rf.any():
        return True
    dt = float(pk.segs[torch.from_numpy(np.flatnonzero(rf)).to(pk.segs.device), 0].max())
    r = float(torch.maximum(pk.spins[4], pk.spins[5]).max())
    return dt * r <= 1.35


def saved_layout(plan, state_bytes: int, budget_bytes: int):
    """(intervals per block, slots) of the backward from saved states for ``plan`` (a ``Plan`` with its
    ``saved``), or None when no layout fits ``budget_bytes`` (``state_bytes`` per stored state): every interval in
    one block with one slot per saved state when they fit; else blocks of K intervals whose starts the forward
    stores, the saved states of one block at a time in slots taken modulo the largest count one block's sweep
    needs (its own runs' and the one after its end: consecutive runs never share a slot), K minimising the states
    held."""
    sv, k = plan.saved, len(plan.starts)
    if sv.n_slots * state_bytes <= budget_bytes:
        return k, sv.n_slots
    ends = np.flatnonzero(sv.slot >= 0)  # the windows whose start state is saved, in slot order
    lo = np.array([a for a, _ in plan.aranges])
    hi = np.array([b for _, b in plan.aranges])
    best = None
    for K in np.unique(np.geomspace(1, k, 256).astype(int)):
        first = np.arange(0, k, K)
        last = np.minimum(first + K, k) - 1
        need = np.searchsorted(ends, hi[last], "right") - np.searchsorted(ends, lo[first], "left")
        cap = max(int(need.max()), 1)
        held = len(first) + cap
        if held * state_bytes <= budget_bytes and (best is None or held < best[0]):
            best = (held, int(K), cap)
    return None if best is None else best[1:]


class Plan:
    """Windows and intervals of one gradient-carrying simulation. ``saved``: plan the states of the backward
    without a replay (``self.saved``, a ``SavedStates``, or None where it does not apply); the forward's windows
    then also start at every saved point."""

    def __init__(self, pk: engine.Packed, every: int, device, saved: bool = False):
        S = pk.flags.shape[0]
        self.every = every
        self.starts = list(range(0, S, every))
        breaks = np.zeros(S, dtype=np.uint8)
        breaks[self.starts] = 1
        samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
        w = _lib.BP_ADJ_WIN
        self.awin = engine.plan_windows(pk.flags, w, seg_max=w, breaks=breaks | run_breaks(pk.flags))
        self.saved = SavedStates.of(pk.flags, self.awin) if saved else None
        fbreaks = breaks.copy()
        if self.saved is not None:
            # (a cut after an RF segment: no readout run of the forward is split, its states keep their bits)
            fbreaks[self.saved.points] = 1
        self.fwin = engine.plan_windows(pk.flags, samp, breaks=fbreaks)
        self.fwin_dev = torch.from_numpy(self.fwin).to(device)
        self.awin_dev = torch.from_numpy(self.awin).to(device)
        if self.saved is not None:
            fslot = np.full(self.fwin.shape[0], -1, dtype=np.int32)
            at = np.searchsorted(self.fwin[:, 0], self.saved.points)
            if not (self.fwin[at, 0] == self.saved.points).all():
                raise RuntimeError("the forward's windows do not start at the saved points")
            fslot[at] = np.arange(len(at), dtype=np.int32)
            self.fslot = fslot  # the slot (run number) of each forward window's start state, -1: none
        # window ranges of every interval
        fstart, astart = self.fwin[:, 0], self.awin[:, 0]
        self.franges, self.aranges, self.seg_ranges = [], [], []
        for k, s0 in enumerate(self.starts):
            s1 = self.starts[k + 1] if k + 1 < len(self.starts) else S
            fa, fb = np.searchsorted(fstart, s0), np.searchsorted(fstart, s1)
            aa, ab = np.searchsorted(astart, s0), np.searchsorted(astart, s1)
            self.franges.append((int(fa), int(fb)))
            self.aranges.append((int(aa), int(ab)))
            self.seg_ranges.append((s0, s1))
        self.max_aw = max(b - a for a, b in self.aranges)
        self.max_len = max(b - a for a, b in self.seg_ranges)


class Checkpointed:
    """The device side of a simulation with gradients on a packed case: the forward that stores the state at every
    interval start, and the backward (per interval in reverse: replay, reverse sweep, segment-gradient reduction);
    or, with ``saved``, the forward that saves the states after the RF runs and the backward without a replay.
    With ``outer`` > 1 intervals per block, the forward stores the state at every block start only, and the
    backward first re-runs each block's forward (no readout) to store its intervals' starts. Every buffer is sized
    by the C ABI's workspace query (``bp_forward_workspace_bytes``, ``bp_adjoint_workspace_bytes``); the backward's
    buffers are allocated on its first call and reused."""

    def __init__(self, pk: engine.Packed, every: int, device, outer: int = 0, phys=None, saved: bool = False,
                 budget_bytes: int | None = None):
        self.pk, self.dev = pk, device
        self.phys = phys  # the field model (``PhysGrad``): the forward, replay and sweep take its variants
        # saved: the caller wants the RF waveform's gradient alone; then, where the sequence's windows allow it, the
        # forward saves the states after every run of RF windows and the backward needs no replay
        # (bp_forward_saving, bp_adjoint_saved). When those states do not fit half the free memory (or
        # ``budget_bytes``), the forward stores the state at every start of a block of intervals instead, and the
        # backward rebuilds each block's saved states by one forward of the block (no readout) before its sweep.
        # Its intervals are at most 2048 segments (the sweep sums an interval's RF gradient in shared memory).
        want = saved and phys is None and rf_relaxation_invertible(pk)
        plan = Plan(pk, min(every, 2048), device, saved=True) if want else None
        self.layout = None  # saved: (intervals per block, slots)
        if plan is not None and plan.saved is not None:
            if budget_bytes is None:
                budget_bytes = torch.cuda.mem_get_info(device)[0] // 2 if torch.cuda.is_available() else 1 << 62
            self.layout = saved_layout(plan, 24 * pk.n, budget_bytes)
        if self.layout is None:
            plan = Plan(pk, every, device)
        self.plan = plan
        self.saved = plan.saved
        k = len(plan.starts)
        self.outer = outer if outer > 1 and k > outer and self.saved is None else 0
        fws = _lib.forward_workspace(pk.n, pk.n_adc, pk.n_coils)
        self.grid = _lib.lib().bp_adjoint_grid(pk.n, pk.n_coils)
        if self.grid < 1:
            raise RuntimeError("bp_adjoint_grid failed")
        self.ws = _lib.adjoint_workspace(pk.n, pk.flags.shape[0], pk.n_adc, pk.n_coils, plan.every, plan.max_aw,
                                         self.grid, self.outer)
        if self.saved is None:
            # interval starts (two levels), or block starts followed by one block's interval starts (three)
            n_states = k if not self.outer else (k + self.outer - 1) // self.outer + self.outer
            self.ckpts = sized(self.ws.checkpoints, (n_states, 6, pk.n), F32, device)
        else:
            # the block starts (none with one block), then the saved states by slot: the state after run r of RF
            # windows in slot r mod `cap` (not in the workspace query: their count is the sequence's)
            per_block, cap = self.layout
            self.n_block_states = 0 if per_block >= k else -(-k // per_block)
            self.ckpts = torch.empty(self.n_block_states + cap, 6, pk.n, dtype=F32, device=device)
            self.slots = self.ckpts[self.n_block_states:]
            mod = lambda m: torch.from_numpy(np.where(m >= 0, m % cap, -1).astype(np.int32)).to(device)
            self.fslot_dev, self.aslot_dev = mod(plan.fslot), mod(plan.saved.slot)
            self.final_slot = (self.saved.n_slots - 1) % cap
        self.raw = sized(fws.raw, (max(pk.n_adc, 1), 2 * pk.n_coils), F64, device, zero=True)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self._bufs = None

    def blocks(self):
        """[(first interval, end interval)] of the outer blocks (one block of every interval on two levels), or of
        the blocks of the backward from saved states."""
        k = len(self.plan.starts)
        step = self.layout[0] if self.saved is not None else (self.outer or k)
        return [(b, min(b + step, k)) for b in range(0, k, step)]

    def _fwd_saving(self, state, ka, kb, raw):
        """The forward over intervals [ka, kb), saving the states after the RF runs in them into their slots."""
        pk, plan = self.pk, self.plan
        fa, fb = plan.franges[ka][0], plan.franges[kb - 1][1]
        code = _lib.lib().bp_forward_saving(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs),
                                            ptr(pk.seg64), ptr(plan.fwin_dev), fa, fb, ptr(state), ptr(raw),
                                            ptr(self.fslot_dev), ptr(self.slots), 0, ptr(self.status),
                                            _lib.stream_ptr())
        _lib.check(code, "bp_forward_saving")

    def forward(self, state: torch.Tensor) -> None:
        """All intervals from ``state`` ([6][n], advanced in place), the raw coil sums into ``raw`` (zeroed first),
        the state at every interval start (at every block start with an outer level) into the checkpoints."""
        pk, plan = self.pk, self.plan
        self.raw.zero_()
        if self.saved is not None:  # one launch per block, saving the states the backward needs (slots mod cap:
            # the last block's are there at the end)
            for bi, (ka, kb) in enumerate(self.blocks()):
                if self.n_block_states:
                    self.ckpts[bi].copy_(state)
                self._fwd_saving(state, ka, kb, self.raw if pk.n_adc else None)
            if self.saved.final:
                self.slots[self.final_slot].copy_(state)
            return
        for k, (fa, fb) in enumerate(plan.franges):
            if not self.outer:
                self.ckpts[k].copy_(state)
            elif k % self.outer == 0:
                self.ckpts[k // self.outer].copy_(state)
            self._fwd(state, plan.fwin_dev, fa, fb, self.raw if pk.n_adc else None)

    def _fwd(self, state, wdev, wa, wb, raw, wstates=None):
        """The forward kernel over windows [wa, wb) (the physics variant with the field model)."""
        pk = self.pk
        if self.phys is None:
            engine.run_forward(pk, state, wdev, wa, wb, raw, self.status, wstates=wstates, wstate_stride=1)
            return
        import ctypes

        ph = self.phys.ph
        ph.wstates, ph.wstate_stride = ptr(wstates), 1
        code = _lib.lib().bp_forward_physics(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs),
                                             ptr(pk.seg64), ptr(wdev), wa, wb, ptr(state), ptr(raw), 0,
                                             ctypes.byref(ph), ptr(self.status), _lib.stream_ptr())
        ph.wstates, ph.wstate_stride = None, 0
        _lib.check(code, "bp_forward_physics")

    def buffers(self, need_seg: bool, want_gc: bool):
        pk, plan, ws, dev = self.pk, self.plan, self.ws, self.dev
        if self._bufs is None:
            self._bufs = {"gs": sized(ws.gs, (8, pk.n), F32, dev), "seg": sized(ws.seg, (pk.flags.shape[0], 8), F64, dev)}
            if self.saved is None:
                self._bufs["wstates"] = sized(ws.wstates, (plan.max_aw + 1, 6, pk.n), F32, dev)
                self._bufs["state"] = sized(ws.replay_state, (6, pk.n), F32, dev)
            else:  # the chain's state between intervals, the rebuild's state
                self._bufs["chain"] = torch.zeros(3, pk.n, dtype=F32, device=dev)
                if self.n_block_states:
                    self._bufs["state"] = sized(ws.replay_state, (6, pk.n), F32, dev)
        b = self._bufs
        if need_seg and "gseg" not in b:
            b["gseg"] = sized(ws.gseg, (self.grid, plan.max_len, 8), F32, dev)
        if want_gc and "gc" not in b:
            b["gc"] = sized(ws.gc, (2 * pk.n_coils, pk.n), F32, dev)
        return b

    def backward(self, h: torch.Tensor | None, lam: torch.Tensor, seg_mask: int, want_gc: bool, need_seg: bool):
        """dL/d(per-spin inputs) ``gs`` [8][n], dL/d(coils) ``gc`` [2C][n] (or None) and the segment gradients
        ``seg`` [S][8] (float64), from the cotangent ``h`` of the raw coil sums ([A][2C] float32, or None) and
        ``lam`` = dL/dm at the end ([3][n], turned into dL/dm at the start in place). Asynchronous: the status word
        is checked by ``check``."""
        pk, plan = self.pk, self.plan
        b = self.buffers(need_seg, want_gc)
        gs, seg, wstates, state = b["gs"], b["seg"], b.get("wstates"), b.get("state")
        gc, gseg = (b["gc"] if want_gc else None), (b["gseg"] if need_seg else None)
        gs.zero_()
        seg.zero_()
        if gc is not None:
            gc.zero_()
        if self.phys is not None and self.phys.gconc is not None:
            self.phys.gconc.zero_()
        if self.saved is not None:
            self._saved_backward(h, lam, gseg if need_seg else None, seg, seg_mask, want_gc, b["chain"], state)
            return gs, gc, seg
        n_blocks = len(self.blocks())
        for bi, (ka, kb) in reversed(list(enumerate(self.blocks()))):
            if self.outer:  # this block's interval starts, from its start (no readout)
                state.copy_(self.ckpts[bi])
                for k in range(ka, kb):
                    self.ckpts[n_blocks + k - ka].copy_(state)
                    if k + 1 < kb:
                        fa, fb = plan.franges[k]
                        self._fwd(state, plan.fwin_dev, fa, fb, None)
            for k in reversed(range(ka, kb)):
                self._interval(k, n_blocks + k - ka if self.outer else k, h, lam, gs, gc, gseg, seg, seg_mask,
                               need_seg, wstates, state)
        return gs, gc, seg

    def _interval(self, k, ck, h, lam, gs, gc, gseg, seg, seg_mask, need_seg, wstates, state):
        """Interval k from checkpoint ``ck``: replay with window states, the reverse sweep, the segment reduction."""
        pk, plan = self.pk, self.plan
        lib, stream, n, C, A = _lib.lib(), _lib.stream_ptr(), pk.n, pk.n_coils, pk.n_adc
        aa, ab = plan.aranges[k]
        s0, s1 = plan.seg_ranges[k]
        state.copy_(self.ckpts[ck])
        self._fwd(state, plan.awin_dev, aa, ab, None, wstates=wstates)
        wstates[ab - aa].copy_(state)  # the state after the interval's last window
        if self.phys is None:
            code = lib.bp_adjoint(ptr(pk.spins), ptr(pk.sens), n, C, ptr(pk.segs), ptr(pk.seg64), ptr(plan.awin_dev),
                                  aa, ab, s0, s1 - s0, ptr(wstates), ptr(h), A, ptr(lam), ptr(gs), ptr(gc), ptr(gseg),
                                  seg_mask, self.grid, ptr(self.status), stream)
        else:
            import ctypes

            code = lib.bp_adjoint_physics(ptr(pk.spins), ptr(pk.sens), n, C, ptr(pk.segs), ptr(pk.seg64),
                                          ptr(plan.awin_dev), aa, ab, s0, s1 - s0, ptr(wstates), ptr(h), A, ptr(lam),
                                          ptr(gs), ptr(gc), ptr(gseg), seg_mask, self.grid,
                                          ctypes.byref(self.phys.ph), ptr(self.phys.gconc), ptr(self.status), stream)
        _lib.check(code, "bp_adjoint")
        if need_seg:
            _lib.check(lib.bp_seg_reduce(ptr(gseg), self.grid, s1 - s0, s0, ptr(seg), stream), "bp_seg_reduce")

    def _saved_backward(self, h, lam, gseg, seg, seg_mask, want_gc, chain, state):
        """The backward without a replay: per block in reverse, its saved states (rebuilt by one forward of the
        block from its start, except the last block's, which the forward left), then per interval in reverse the
        sweep from the saved states, carrying the chain of RF windows integrated backward across the intervals,
        and the segment reduction."""
        pk, plan, sv = self.pk, self.plan, self.saved
        lib, stream, W = _lib.lib(), _lib.stream_ptr(), plan.awin.shape[0]
        if want_gc or not rf_only(seg_mask):
            raise ValueError("the backward from saved states forms the RF waveform's gradient alone")
        blocks = self.blocks()
        for bi, (ka, kb) in reversed(list(enumerate(blocks))):
            if bi + 1 < len(blocks):
                state.copy_(self.ckpts[bi])
                self._fwd_saving(state, ka, kb, None)
            for k in reversed(range(ka, kb)):
                aa, ab = plan.aranges[k]
                s0, s1 = plan.seg_ranges[k]
                chain_in = int(ab < W and bool(sv.rf[ab]))
                code = lib.bp_adjoint_saved(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs),
                                            ptr(pk.seg64), ptr(plan.awin_dev), aa, ab, s0, s1 - s0, ptr(self.slots),
                                            ptr(self.aslot_dev), ptr(chain), chain_in, ptr(h), pk.n_adc, ptr(lam),
                                            ptr(gseg), seg_mask, self.grid, ptr(self.status), stream)
                _lib.check(code, "bp_adjoint_saved")
                if gseg is not None:
                    _lib.check(lib.bp_seg_reduce(ptr(gseg), self.grid, s1 - s0, s0, ptr(seg), stream),
                               "bp_seg_reduce")

    def launches(self, need_seg: bool) -> tuple[int, int]:
        """(forward, backward) kernel launches of one call each."""
        k = len(self.plan.starts)
        if self.saved is not None:
            nb = len(self.blocks())
            return nb, nb - 1 + k * (2 if need_seg else 1)
        rebuild = sum(kb - ka - 1 for ka, kb in self.blocks()) if self.outer else 0
        return k, k * (3 if need_seg else 2) + rebuild

    def check(self, what: str = "bp_forward / bp_adjoint") -> None:
        torch.cuda.synchronize(self.dev)
        _lib.check_status(self.status, what)

    def cotangent(self, g_sig: torch.Tensor) -> torch.Tensor:
        """h = dL/d(raw coil sums) [A][2C] float32 on the device from dL/dsignal (C, A) (complex, or (C, A, 2)
        real pairs): dL/draw = dL/dsignal e^{+i psi}."""
        pk = self.pk
        g = g_sig if g_sig.is_complex() else torch.complex(g_sig[..., 0].to(F64), g_sig[..., 1].to(F64))
        hr = g.to(torch.complex128).to(self.dev) * torch.exp(1j * pk.psi)[None, :]
        h = sized(self.ws.h, (pk.n_adc, 2 * pk.n_coils), F32, self.dev)
        h.copy_(torch.view_as_real(hr.T.contiguous()).reshape(pk.n_adc, 2 * pk.n_coils))
        return h


class PhysGrad:
    """The field model's device buffers for a gradient-carrying simulation: the concomitant coefficients ([7][n]
    float32, rows of the mode's coefficients), the segments' dt-weighted gradient monomials ([S][6] float64, mode
    1), the ``BpPhysics`` descriptor, and the coefficients' gradient ([7][n], when wanted)."""

    def __init__(self, conc: torch.Tensor, mode: int, dt, grad, device, want_grad: bool):
        from .physics import gradient_moments2

        n = conc.shape[0]
        cc = torch.zeros(7, n, dtype=F32)
        cc[: conc.shape[1]] = conc.detach().to(F64).cpu().T.to(F32)
        self.conc = cc.to(device).contiguous()
        self.segq = (torch.from_numpy(np.ascontiguousarray(gradient_moments2(dt, grad))).to(device)
                     if mode == 1 else None)
        self.gconc = torch.zeros(7, n, dtype=F32, device=device) if want_grad else None
        self.ph = _lib.BpPhysics()
        self.ph.conc_mode, self.ph.conc, self.ph.segq = mode, ptr(self.conc), ptr(self.segq)
        self.width = conc.shape[1]


def rf_only(seg_mask: int) -> bool:
    """Whether ``seg_mask`` asks for the RF waveform's gradient alone (no per-spin, coil or offset gradient): the
    sweep that ``bp_adjoint_saved`` runs."""
    return bool(seg_mask & _lib.BP_SPIN_NONE) and not seg_mask & _lib.BP_SEG_ALL & ~(_lib.BP_SEG_WX | _lib.BP_SEG_WY)


def seg_mask_for(need) -> int:
    """The segment gradients the chain rules use (``need``: ``_Simulate``'s needs_input_grad): dt needs all of
    them (the record's every field scales with dt), the RF its two components, the gradient the moments,
    b0_offset its phase; ``BP_SPIN_NO_OFFSETS`` unless the positions' or dB0's gradients are wanted, and
    ``BP_SPIN_NONE`` when no per-spin input (position, PD, T1, T2, dB0, B1, coils) needs one."""
    conc = len(need) > 14 and need[14]  # the concomitant coefficients (their gradient is an offsets' gradient)
    spin_none = not any(need[i] for i in range(1, 8)) and not conc
    return (_lib.BP_SEG_ALL if need[8] else 0) | ((_lib.BP_SEG_WX | _lib.BP_SEG_WY) if need[9] else 0) | (
        (_lib.BP_SEG_KX | _lib.BP_SEG_KY | _lib.BP_SEG_KZ) if need[10] else 0) | (
        _lib.BP_SEG_BETA if need[12] else 0) | (0 if (need[1] or need[5] or conc) else _lib.BP_SPIN_NO_OFFSETS) | (
        _lib.BP_SPIN_NONE if spin_none else 0)


class _Simulate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, opts, pos, pd, t1, t2, db0, b1, coils_ri, dt, rf, grad, adc_phase, b0_offset, m0, conc=None):
        from .api import Inputs

        dev, every, flags_in = opts["device"], opts["every"], opts["flags"]
        coils = torch.view_as_complex(coils_ri.detach().contiguous())
        d = lambda t: None if t is None else t.detach()
        inp = Inputs(d(pos), d(pd), d(t1), d(t2), d(db0), d(b1), coils, d(dt), d(rf), d(grad), d(adc_phase),
                     d(b0_offset), *flags_in, d(m0))
        pk = engine.pack(inp, dev)
        phys = None
        if conc is not None:  # the field model's concomitant coefficients (positions: the encoding ones)
            phys = PhysGrad(conc, opts["conc_mode"], inp.dt, inp.grad, dev, ctx.needs_input_grad[14])
        # the RF waveform's gradient alone: the backward from saved states where the sequence allows it
        run = Checkpointed(pk, every, dev, opts.get("outer", 0), phys,
                           saved=opts.get("saved", True) and rf_only(seg_mask_for(ctx.needs_input_grad)))
        state = engine.initial_state(inp.pd, inp.m_init, dev)
        run.forward(state)
        sig = engine.finish_signal(pk, run.raw)
        run.check("bp_forward")
        ctx.run, ctx.dev = run, dev
        ctx.like = [None if t is None else (t.dtype, t.device) for t in
                    (pos, pd, t1, t2, db0, b1, coils_ri, dt, rf, grad, adc_phase, b0_offset, m0, conc)]
        ctx.raw_mode = bool(opts.get("raw"))
        ctx.set_materialize_grads(False)
        if ctx.raw_mode:  # the float64 raw coil sums on the device, not demodulated (the caller demodulates)
            ctx.save_for_backward(t1, t2, dt, rf, grad, b0_offset, adc_phase, None)
            return run.raw[: pk.n_adc].clone(), engine.final_m(state)
        sig_ri = torch.view_as_real(sig).cpu().contiguous()  # (C, A, 2)
        ctx.save_for_backward(t1, t2, dt, rf, grad, b0_offset, adc_phase, sig_ri)
        return sig_ri, engine.final_m(state)

    @staticmethod
    @once_differentiable
    def backward(ctx, g_sig, g_m):
        t1, t2, dt, rf, grad, b0_offset, adc_phase, sig_ri = ctx.saved_tensors
        run, dev = ctx.run, ctx.dev
        pk = run.pk
        # inputs: opts, pos, pd, t1, t2, db0, b1, coils_ri, dt, rf, grad, adc_phase, b0_offset, m0, conc
        need = ctx.needs_input_grad
        if g_sig is None and g_m is None:
            return (None,) * 15
        n, C, A, S = pk.n, pk.n_coils, pk.n_adc, len(dt)
        if ctx.raw_mode:  # dL/d(raw coil sums) directly
            h = sized(run.ws.h, (A, 2 * C), F32, dev).copy_(g_sig) if (g_sig is not None and A) else None
        else:
            h = run.cotangent(g_sig) if (g_sig is not None and A) else None
        lam = sized(run.ws.lam, (3, n), F32, dev, zero=True)
        if g_m is not None:
            lam.copy_(g_m.T.to(F32))
        need_seg = any(need[i] for i in (8, 9, 10, 12))
        gs, gc, seg = run.backward(h, lam, seg_mask_for(need), need[7] and h is not None, need_seg)
        run.check("bp_forward (replay) / bp_adjoint")
        gs64, lam64 = gs.to(F64).cpu(), lam.to(F64).cpu()
        out = [None] * 14
        if need[1]:
            out[0] = gs64[0:3].T.contiguous()
        if need[2]:
            out[1] = gs64[4]
        if need[3]:
            out[2] = -gs64[5] / t1.detach().to(F64).cpu() ** 2
        if need[4]:
            out[3] = -gs64[6] / t2.detach().to(F64).cpu() ** 2
        if need[5]:
            out[4] = gs64[3]
        if need[6]:
            out[5] = gs64[7]
        if need[7] and gc is not None:
            g = gc.to(F64).cpu()
            out[6] = torch.stack([g[0::2].T, g[1::2].T], -1)
        if need_seg:
            sg = seg.cpu()
            dt64, rf64, gr64 = dt.detach().to(F64).cpu(), rf.detach().to(F64).cpu(), grad.detach().to(F64).cpu()
            b064 = torch.zeros(S, dtype=F64) if b0_offset is None else b0_offset.detach().to(F64).cpu()
            w = -TWO_PI * dt64
            if need[8]:
                out[7] = (sg[:, 0] + sg[:, 1] * (-TWO_PI * rf64[:, 0]) + sg[:, 2] * (-TWO_PI * rf64[:, 1])
                          + (sg[:, 3:6] * gr64).sum(1) + sg[:, 6] * b064)
            if need[9]:
                out[8] = torch.stack([sg[:, 1] * w, sg[:, 2] * w], -1)
            if need[10]:
                out[9] = sg[:, 3:6] * dt64[:, None]
            if need[12]:
                out[11] = sg[:, 6] * dt64
        if need[11] and g_sig is not None and A and not ctx.raw_mode:
            adc_idx = torch.tensor(np.flatnonzero(pk.flags & engine.ADC))
            sr, si_ = sig_ri[..., 0].to(F64), sig_ri[..., 1].to(F64)
            gr, gi = g_sig[..., 0].to(F64), g_sig[..., 1].to(F64)
            gp = torch.zeros(S, dtype=F64)
            gp[adc_idx] = (gr * si_ - gi * sr).sum(0)
            out[10] = gp
        if need[13]:
            out[12] = lam64.T.contiguous()
        if need[14] and run.phys is not None and run.phys.gconc is not None:
            out[13] = run.phys.gconc.to(F64).cpu()[: run.phys.width].T.contiguous()
        return (None, *[None if v is None or not need[i + 1] else v.to(dtype=ctx.like[i][0], device=ctx.like[i][1])
                        for i, v in enumerate(out)])


def _check_grad_options(options):
    """With gradients, readout "nufft" and pulses "reuse" (forward-only accelerations) take the float32 readout and
    stepped pulses, as blochparty's GPU engines do (engines/gpu/__init__.py:78-80 hand neither to their gradient
    path); the split-BF16 readout and the learned surrogate are refused."""
    if options.get("readout", "fp32") not in ("fp32", "nufft"):
        raise NotImplementedError(f"b200 engine: gradients through readout={options['readout']!r} are not "
                                  "implemented; use the default float32 readout (or torch.no_grad())")
    if options.get("pulses", "step") not in ("step", "reuse"):
        raise NotImplementedError("b200 engine: gradients through pulses='surrogate' are not implemented; use "
                                  "pulses='step' (or torch.no_grad())")


def _apply(inp, dev, checkpoint_every, raw: bool, scanner=None):
    S = len(inp.dt)
    conc, mode = None, 0
    if scanner is not None:  # encoding positions and concomitant coefficients, differentiable (physics)
        from dataclasses import replace

        from .physics import spin_fields_torch

        enc, conc, mode = spin_fields_torch(scanner, inp.pos)
        inp = replace(inp, pos=enc)
    every, outer = (checkpoint_every, 0) if checkpoint_every else choose_checkpoints(S, inp.pd.shape[0])
    if every % _lib.BP_ADJ_WIN:
        raise ValueError(f"checkpoint_every must be a multiple of {_lib.BP_ADJ_WIN}, got {every}")
    n = inp.pd.shape[0]
    m0 = inp.m_init
    if m0 is None:
        z = torch.zeros_like(inp.pd)
        m0 = torch.stack([z, z, inp.pd], -1)
    coils_ri = torch.view_as_real(inp.coils if inp.coils.is_complex() else inp.coils.to(torch.complex64))
    opts = {"device": dev, "every": every, "outer": outer, "flags": (inp.is_rf, inp.adc, inp.spoil), "raw": raw,
            "conc_mode": mode}
    return _Simulate.apply(opts, inp.pos, inp.pd, inp.t1, inp.t2, inp.db0, inp.b1, coils_ri, inp.dt, inp.rf, inp.grad,
                           inp.adc_phase, inp.b0_offset, m0, conc)


def simulate_grad(inp, dev, checkpoint_every, options, scanner=None) -> SimResult:
    """``simulate`` with gradients: the inputs as tensors of ``_Simulate`` (with a scanner field model, the encoding
    positions and concomitant coefficients from its differentiable host functions)."""
    _check_grad_options(options)
    sig_ri, m = _apply(inp, dev, checkpoint_every, raw=False, scanner=scanner)
    return SimResult(torch.view_as_complex(sig_ri.contiguous()), m)


def simulate_raw(inp, dev, checkpoint_every=None):
    """The differentiable float64 raw coil sums (A, 2 C) on the device (coil c's real part in column 2 c, its
    imaginary part in 2 c + 1; not demodulated) and m (N, 3) float32 on the CPU, gradients by the adjoint: the
    per-rank part of a sharded simulation, whose ranks sum their raw sums before demodulating
    (``parallel.simulate``)."""
    return _apply(inp, dev, checkpoint_every, raw=True)


def demodulate(total: torch.Tensor, adc_phase: torch.Tensor, adc) -> torch.Tensor:
    """The (C, A) complex signal from raw coil sums (A, 2 C): coil c is (total[:, 2c] + i total[:, 2c + 1])
    exp(-i adc_phase) at the ADC segments (differentiable in both, float64)."""
    idx = torch.tensor(np.flatnonzero(np.asarray([bool(x) for x in adc])), dtype=torch.long)
    psi = adc_phase.to(F64)[idx.to(adc_phase.device)].to(total.device)
    z = torch.complex(total[:, 0::2].to(F64), total[:, 1::2].to(F64))
    return (z * torch.exp(-1j * psi)[:, None]).T
