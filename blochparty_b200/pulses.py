"""Reused pulses (``simulate(..., pulses="reuse")``, forward only): a pulse of two or more RF segments that recurs
up to a global RF phase is composed once per spin into its exact affine map (``bp_pulse_maps``, float64) and
applied at every occurrence turned about z by the occurrence's phase (``bp_pulse_apply``).

The reference's form is blochparty ``engines/gpu/driver.py:112-164`` (finding the pulses) with
``engines/gpu/cuda/pulse.cu.in:3-32`` (the maps); its rules are kept: a pulse is a run of at least two consecutive
RF segments without a sample (a spoil only on its last segment); an occurrence has the flags, dt, gradient and
b0_offset of the pulse's first occurrence (to ``tol`` of their largest magnitude) and its RF times e^{i phase}
(the phase by least squares); pulses that save the most stepped segments come first, as many as fit in
``memory`` bytes of maps (96 bytes per spin and pulse). Pulses that do not fit are stepped.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib, engine
from ._lib import ptr

F64 = torch.float64
PULSE_MEMORY = 16 << 30  # bytes of per-spin maps at most


def _runs(is_rf, adc, spoil):
    """(start, length) of every maximal run of RF segments without a sample, cut after a spoiled segment."""
    live = is_rf & ~adc
    S = live.shape[0]
    prev_live = np.concatenate([[False], live[:-1]])
    prev_spoil = np.concatenate([[False], spoil[:-1]])
    starts = np.flatnonzero(live & (~prev_live | prev_spoil))
    next_live = np.concatenate([live[1:], [False]])
    ends = np.flatnonzero(live & (~next_live | spoil)) + 1
    return starts, ends - starts


def find_reused(inp, tol: float = 1e-6):
    """[(first segment, length, [(segment, phase), ...])] of every pulse that recurs (at least two occurrences,
    the first with phase 0), most stepped segments saved first."""
    d = lambda t: t.detach().to(F64).cpu().numpy()
    dt, rf, grad = d(inp.dt), d(inp.rf), d(inp.grad)
    S = dt.shape[0]
    b0 = np.zeros(S) if inp.b0_offset is None else d(inp.b0_offset)
    is_rf, adc, spoil = (np.fromiter(f, dtype=bool, count=S) for f in (inp.is_rf, inp.adc, inp.spoil))
    z = rf[:, 0] + 1j * rf[:, 1]
    starts, lens = _runs(is_rf, adc, spoil)
    keep = lens >= 2
    starts, lens = starts[keep], lens[keep]
    if starts.size == 0:
        return []
    # buckets of equal length and duration (ns); within one, runs are compared with a representative at once
    csum = np.concatenate([[0.0], np.cumsum(dt)])
    dur = np.round((csum[starts + lens] - csum[starts]) * 1e9).astype(np.int64)
    groups = []
    for key in sorted(set(zip(lens.tolist(), dur.tolist()))):
        sel = starts[(lens == key[0]) & (dur == key[1])]
        k = key[0]
        idx = sel[:, None] + np.arange(k)
        D, G, B, W, P = dt[idx], grad[idx], b0[idx], z[idx], spoil[idx]
        left = np.arange(sel.size)
        while left.size:
            r = left[0]
            same = ((P[left] == P[r][None]).all(1) & _close_tol(D[left], D[r], tol) & _close_tol(G[left], G[r], tol)
                    & _close_tol(B[left], B[r], tol))
            c = W[left] @ np.conj(W[r])
            ph = np.where(c != 0, np.angle(c), 0.0)
            same &= _close_tol(W[left], W[r], tol, rot=np.exp(1j * ph))
            same[0] = True
            members = left[same]
            occ = [(int(sel[m]), 0.0 if m == r else float(p)) for m, p in zip(members, ph[same])]
            if len(occ) > 1:
                groups.append((int(sel[r]), k, occ))
            left = left[~same]
    return sorted(groups, key=lambda g: (-(len(g[2]) - 1) * g[1], g[0]))


def _close_tol(x, y, tol, rot=None):
    """Rows of x within tol (relative to the larger peak magnitude) of y, or of y times rot[row] when given."""
    ref = y[None] if rot is None else y[None] * rot.reshape((-1,) + (1,) * (x.ndim - 1))
    scale = np.maximum(np.abs(x).reshape(x.shape[0], -1).max(1), float(np.abs(y).max()) if y.size else 0.0)
    return np.abs(x - ref).reshape(x.shape[0], -1).max(1) <= tol * np.maximum(scale, 1e-300)


class Reuse:
    """The reused pulses of one packed case: the pulses kept under the ``memory`` cap, their occurrences in order,
    the window plan around them, and room for the maps (filled by ``make_maps``)."""

    def __init__(self, inp, pk, memory: int = PULSE_MEMORY):
        per_pulse = _lib.BP_PULSE_MAP_BYTES * pk.n
        self.pulses = find_reused(inp)[: max(0, memory // per_pulse)]
        self.occ = sorted((s, k, pid, ph) for pid, (_, k, lst) in enumerate(self.pulses) for s, ph in lst)
        self.spans = [(s, k) for s, k, _, _ in self.occ]
        self.plan = engine.plan_replacing(pk, self.spans)
        self.maps = torch.empty(len(self.pulses), 12, pk.n, dtype=F64, device=pk.device)

    def make_maps(self, pk):
        lib, st = _lib.lib(), _lib.stream_ptr()
        for pid, (a, k, _) in enumerate(self.pulses):
            _lib.check(lib.bp_pulse_maps(ptr(pk.spins), pk.n, ptr(pk.segs), ptr(pk.seg64), a, k, ptr(self.maps[pid]),
                                         st), "bp_pulse_maps")

    def descriptors(self):
        """The occurrences as ``BpSpan`` descriptors for ``bp_forward_spans`` (map pointers into ``self.maps``)."""
        arr = (_lib.BpSpan * max(1, len(self.occ)))()
        for i, (s, k, pid, ph) in enumerate(self.occ):
            arr[i] = _lib.BpSpan(kind=_lib.BP_SPAN_MAP, seg0=s, k_steps=k, phase=ph, map=ptr(self.maps[pid]))
        return arr

    def run(self, pk, state, raw, status, max_ctas: int = 0, events=None):
        """The forward with every occurrence through its pulse's map (``make_maps`` first): one native call, or the
        launches one by one from Python when ``events`` collects the forward launches' CUDA events."""
        if events is None:
            if not hasattr(self, "_desc"):
                self._desc = self.descriptors()
            engine.forward_spans(pk, state, self.plan, self._desc, raw, status, max_ctas)
            return
        lib, st = _lib.lib(), _lib.stream_ptr()

        def apply(i):
            _, _, pid, ph = self.occ[i]
            _lib.check(lib.bp_pulse_apply(ptr(self.maps[pid]), pk.n, ptr(state), ph, st), "bp_pulse_apply")

        engine.forward_replacing(pk, state, self.spans, apply, raw, status, max_ctas=max_ctas, plan=self.plan,
                                 events=events)


def forward_with_reuse(inp, device, max_ctas: int = 0, memory: int = PULSE_MEMORY):
    """``simulate(..., pulses="reuse")``: signal (C, A) complex64 and m (N, 3) float32 on the CPU."""
    pk = engine.pack(inp, device)
    reuse = Reuse(inp, pk, memory)
    reuse.make_maps(pk)
    state = engine.initial_state(inp.pd, inp.m_init, device)
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    reuse.run(pk, state, raw if pk.n_adc else None, status, max_ctas)
    sig = engine.finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward")
    return sig.cpu(), engine.final_m(state)
