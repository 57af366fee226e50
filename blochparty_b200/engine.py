"""Host driver of the b200 engine: inputs into device buffers, the window plan, the launches, the results.

Replaces blochparty's GPU driver for static spins (``engines/gpu/driver.py:_forward``, :197-756): the same
float64-on-host preparation (positions, rates 1/T1 and 1/T2, per-segment quantities, the state split into a
float32 high part and its float32 remainder) feeding the C ABI of ``libblochparty_b200.so``.

Device buffers (float32 unless stated; N spins, S segments, C coils, A ADC samples):

* ``spins`` [8][N]: x, y, z, pd, r1, r2, dB0, b1 (structure of arrays: one coalesced row per field);
* ``sens`` [16 ceil(C/8)][N]: coil c real at row 2c, imaginary at 2c+1, zero padding rows;
* ``segs`` [S] 32-byte records: dt, -2 pi dt rf_x, -2 pi dt rf_y, g dt (3), b0_offset dt, flags (int32);
* ``seg64`` [S][4] float64: g dt (3), b0_offset dt: the free segments' phase is evaluated in float64;
* ``windows`` [W][4] int32: first segment, end segment, first ADC row, samples (``bp_plan_windows``);
* ``state`` [6][N]: mx, my, mz and their compensation parts;
* ``raw`` [A][2C] float64: the coil sums before demodulation; ``signal`` (C, A) complex64.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import ptr

TWO_PI = 2.0 * math.pi
F32, F64 = torch.float32, torch.float64

RF, ADC, SPOIL, SAME_FREE, SAME_RFDT, SAME_OFF, SMALL = 1, 2, 4, 8, 16, 32, 64


@dataclass
class Packed:
    """A case's device buffers (see module docstring) and sizes."""

    n: int
    n_coils: int
    n_adc: int
    spins: torch.Tensor
    sens: torch.Tensor
    segs: torch.Tensor  # (S, 8) float32 view of the records (the flags column holds int32 bits)
    seg64: torch.Tensor
    psi: torch.Tensor  # (A,) float64 receiver phase of every sample
    flags: np.ndarray  # (S,) int32 on the host
    device: torch.device


def _bools(flags, n: int) -> np.ndarray:
    """A sequence of n truth values (Python bools or ints, as blochparty's Sequence holds them) as a bool array:
    through bytes() when every item is a small int (four times faster on a million items), else item by item."""
    if isinstance(flags, (list, tuple)):
        try:
            out = np.frombuffer(bytes(flags), dtype=np.uint8).astype(bool)
            if out.shape[0] == n:
                return out
        except (TypeError, ValueError):
            pass
    return np.fromiter((bool(x) for x in flags), dtype=bool, count=n)


def _np64(t) -> np.ndarray:
    return t.detach().to(F64).cpu().numpy()


def pack_spins(pos, pd, t1, t2, db0, b1, coils, device):
    """spins [8][N] and sens [16 ceil(C/8)][N] float32 on ``device``: every value rounded once to float32 from its
    float64 value (the rates 1/T1, 1/T2 formed in float64), written row by row into the float32 buffers."""
    n = pd.shape[0]
    d64 = lambda t: t.detach().cpu().to(F64)
    spins = torch.empty(8, n, dtype=F32)
    spins[0:3] = d64(pos).T
    spins[3] = d64(pd)
    spins[4] = 1.0 / d64(t1)
    spins[5] = 1.0 / d64(t2)
    spins[6] = d64(db0)
    if b1 is None:
        spins[7] = 1.0
    else:
        spins[7] = d64(b1)
    n_coils = coils.shape[1]
    ncg = (n_coils + 7) // 8
    # (N, 2C) float32 rounded on the host, moved as it lies, transposed on the device (a host-side transpose of the
    # spin-major coil array costs more than the copy)
    c = torch.view_as_real(coils.detach().cpu().to(torch.complex128).contiguous()).reshape(n, 2 * n_coils).to(F32)
    sens = torch.zeros(16 * ncg, n, dtype=F32, device=device)
    sens[0:2 * n_coils] = c.to(device).T
    return spins.to(device).contiguous(), sens.contiguous()


def pack_segments(dt, rf, grad, b0_offset, adc_phase, is_rf, adc, spoil, device):
    """Segment records (float64 arithmetic, one rounding to float32), the float64 moments, flags and psi. The
    fields are filled and compared as contiguous rows of a field-major array, then transposed once into records."""
    dt, rf, grad = _np64(dt), _np64(rf), _np64(grad)
    S = dt.shape[0]
    b0 = np.zeros(S) if b0_offset is None else _np64(b0_offset)
    w = -TWO_PI * dt
    k = grad.T * dt  # (3, S)
    beta = b0 * dt
    cols = np.empty((8, S), dtype=np.float32)  # the record's fields, one row each
    cols[0] = dt
    cols[1] = w * rf[:, 0]
    cols[2] = w * rf[:, 1]
    cols[3:6] = k
    cols[6] = beta
    k64 = np.empty((4, S), dtype=np.float64)
    k64[0:3] = k
    k64[3] = beta
    is_rf, adc_b, spoil_b = (_bools(f, S) for f in (is_rf, adc, spoil))
    flags = is_rf.astype(np.int32) | (adc_b.astype(np.int32) << 1) | (spoil_b.astype(np.int32) << 2)
    if S > 1:
        free = ~is_rf
        same_dt = cols[0, 1:] == cols[0, :-1]
        same_k = same_dt.copy()  # the moments and the offset phase
        for c in range(4):
            same_k &= k64[c, 1:] == k64[c, :-1]
        same_free = free[1:] & free[:-1] & same_k
        same_rf = is_rf[1:] & is_rf[:-1] & same_dt
        same_off = same_rf.copy()  # the same G.r + dt dB0 + beta per spin
        for c in range(3, 7):
            same_off &= cols[c, 1:] == cols[c, :-1]
        flags[1:] |= ((same_free.astype(np.int32) << 3) | (same_rf.astype(np.int32) << 4)
                      | (same_off.astype(np.int32) << 5))
    cols.view(np.int32)[7] = flags
    rec, seg64 = np.ascontiguousarray(cols.T), np.ascontiguousarray(k64.T)
    psi = np.remainder(_np64(adc_phase)[adc_b], TWO_PI)
    return (torch.from_numpy(rec).to(device).contiguous(), torch.from_numpy(seg64).to(device).contiguous(),
            torch.from_numpy(psi).to(device).contiguous(), flags, int(adc_b.sum()))


def plan_windows(flags: np.ndarray, samp_max: int, seg_max: int = _lib.BP_SEG_MAX, breaks: np.ndarray | None = None):
    """(W, 4) int32 windows from the native planner (``bp_plan_windows``)."""
    S = flags.shape[0]
    n_adc = int(((flags & ADC) != 0).sum())
    n_breaks = 0 if breaks is None else int(breaks.sum())
    cap = 2 * (S // seg_max + n_adc // samp_max + n_breaks) + 2  # (grown below if the aligned cuts need more)
    nw = np.zeros(1, dtype=np.int64)
    fl = np.ascontiguousarray(flags, dtype=np.int32)
    br = None if breaks is None else np.ascontiguousarray(breaks, dtype=np.uint8)
    while True:
        out = np.zeros((cap, 4), dtype=np.int32)
        code = _lib.lib().bp_plan_windows(fl.ctypes.data, S, seg_max, samp_max,
                                          None if br is None else br.ctypes.data, out.ctypes.data, cap, nw.ctypes.data)
        if code != _lib.BP_E_SIZE or cap >= S + 1:
            break
        cap = min(2 * cap, S + 1)
    _lib.check(code, "bp_plan_windows")
    return out[: int(nw[0])].copy()


def initial_state(pd, m_init, device):
    """[6][N] float32: m0 split exactly from float64 into a float32 high part and its float32 remainder."""
    n = pd.shape[0]
    out = torch.zeros(6, n, dtype=F32)
    if m_init is None:  # (0, 0, pd): only the z rows are nonzero
        z = pd.detach().cpu().to(F64)
        out[2] = z
        out[5] = z - out[2].to(F64)
    else:
        m64 = m_init.detach().cpu().to(F64).T
        out[0:3] = m64
        out[3:6] = m64 - out[0:3].to(F64)
    return out.to(device).contiguous()


def final_m(state: torch.Tensor) -> torch.Tensor:
    s = state.to(F64)
    return (s[0:3] + s[3:6]).to(F32).T.contiguous().cpu()


def mark_small_rf(spins: torch.Tensor, segs: torch.Tensor, flags: np.ndarray) -> None:
    """Set SMALL on the RF segments whose rotation |w|^2 = b1^2 (wx0^2 + wy0^2) + wz^2 stays below 0.0624 (under
    the first tier's 1/16) for every spin, bounding |wz| = 2 pi |k.r + dt dB0 + beta| by the spins' extents (in the
    device records and the host flags). The kernels then take the first-tier factors without tests: the same
    arithmetic the tests would choose. (The reference tests phi per spin and step, switching to its two-term
    series below phi = 1e-3: blochparty ``engines/gpu/shaders/common.metal:57-72``.)"""
    if spins.shape[1] == 0 or segs.shape[0] == 0:
        return
    ext = spins.abs().amax(dim=1).to(F64)  # |x|, |y|, |z|, pd, r1, r2, |dB0|, |b1| maxima
    rec = segs.to(F64)
    wz = TWO_PI * (rec[:, 3].abs() * ext[0] + rec[:, 4].abs() * ext[1] + rec[:, 5].abs() * ext[2]
                   + rec[:, 0].abs() * ext[6] + rec[:, 6].abs())
    p2 = ext[7] ** 2 * (rec[:, 1] ** 2 + rec[:, 2] ** 2) + wz ** 2
    bits = segs.view(torch.int32)[:, 7]
    small = ((bits & RF) != 0) & (p2 < 0.0624)
    bits |= small.to(torch.int32) * SMALL
    flags |= small.cpu().numpy().astype(np.int32) * SMALL


def pack(case, device) -> Packed:
    spins, sens = pack_spins(case.pos, case.pd, case.t1, case.t2, case.db0, case.b1, case.coils, device)
    segs, seg64, psi, flags, n_adc = pack_segments(case.dt, case.rf, case.grad, case.b0_offset, case.adc_phase,
                                                   case.is_rf, case.adc, case.spoil, device)
    mark_small_rf(spins, segs, flags)
    return Packed(case.pd.shape[0], case.coils.shape[1], n_adc, spins, sens, segs, seg64, psi, flags, device)


def run_forward(pk: Packed, state: torch.Tensor, windows_dev: torch.Tensor, w_begin: int, w_end: int,
                raw: torch.Tensor | None, status: torch.Tensor, wstates: torch.Tensor | None = None,
                wstate_stride: int = 1, max_ctas: int = 0) -> None:
    code = _lib.lib().bp_forward(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                 ptr(windows_dev), w_begin, w_end, ptr(state), ptr(raw), ptr(wstates),
                                 wstate_stride, max_ctas, ptr(status), _lib.stream_ptr())
    _lib.check(code, "bp_forward")


def finish_signal(pk: Packed, raw: torch.Tensor) -> torch.Tensor:
    """(C, A) complex64 on the device: the float64 sums demodulated by exp(-i psi)."""
    out = torch.empty(pk.n_coils, max(pk.n_adc, 1), dtype=torch.complex64, device=pk.device)
    code = _lib.lib().bp_signal_finish(ptr(raw), ptr(pk.psi), pk.n_adc, pk.n_coils, ptr(out), _lib.stream_ptr())
    _lib.check(code, "bp_signal_finish")
    return out[:, : pk.n_adc]


def plan_replacing(pk: Packed, spans):
    """Windows (host array and device copy) with breaks at every span's start and end, and the window ranges
    [(w_begin, w_end)] stepped before each span and after the last, for ``forward_replacing``."""
    S = pk.flags.shape[0]
    breaks = np.zeros(S, dtype=np.uint8)
    for s, k in spans:
        breaks[s] = 1
        if s + k < S:
            breaks[s + k] = 1
    samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
    windows = plan_windows(pk.flags, samp, breaks=breaks)
    starts = windows[:, 0]
    ranges, w = [], 0
    for s, k in spans:
        wa = int(np.searchsorted(starts, s))
        ranges.append((w, wa))
        w = int(np.searchsorted(starts, s + k))
    ranges.append((w, windows.shape[0]))
    return windows, torch.from_numpy(windows).to(pk.device), ranges


def forward_replacing(pk: Packed, state: torch.Tensor, spans, apply, raw: torch.Tensor | None,
                      status: torch.Tensor, max_ctas: int = 0, plan=None, events=None) -> None:
    """The forward over all segments, where each span ``(start, length)`` of ``spans`` (sorted, disjoint, no ADC
    inside) is not stepped but replaced by ``apply(i)`` (launching the replacement of span i on the state).
    Windows are planned with breaks at every span's start and end (``plan_replacing``, or ``plan`` when given), so
    a span is a whole run of windows. ``events``: a list that receives a (start, end) pair of recorded CUDA events
    around every forward launch (the stepped part's device time)."""
    _, wdev, ranges = plan or plan_replacing(pk, spans)

    def step(wa, wb):
        if wb <= wa:
            return
        if events is not None:
            e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            e[0].record()
        run_forward(pk, state, wdev, wa, wb, raw, status, max_ctas=max_ctas)
        if events is not None:
            e[1].record()
            events.append(e)

    for i in range(len(spans)):
        step(*ranges[i])
        apply(i)
    step(*ranges[-1])


def forward_spans(pk: Packed, state: torch.Tensor, plan, spans, raw: torch.Tensor | None, status: torch.Tensor,
                  max_ctas: int = 0) -> None:
    """``forward_replacing`` in one native call: ``spans`` is a ctypes array of ``_lib.BpSpan`` (one per span of
    ``plan``, from ``plan_replacing``), launched in order by ``bp_forward_spans``."""
    _, wdev, ranges = plan
    rng = np.ascontiguousarray(np.asarray(ranges, dtype=np.int32).reshape(-1, 2))
    n_spans = rng.shape[0] - 1
    code = _lib.lib().bp_forward_spans(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                       ptr(wdev), rng.ctypes.data, n_spans, ctypes.addressof(spans) if n_spans else None,
                                       ptr(state), ptr(raw), max_ctas, ptr(status), _lib.stream_ptr())
    _lib.check(code, "bp_forward_spans")


def forward(case, device, max_ctas: int = 0):
    """Signal (C, A) complex64 and m (N, 3) float32, both on the CPU, of a case (``oracle.bloch.Case``-like)."""
    pk = pack(case, device)
    samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
    if samp <= 0:
        raise ValueError(f"at most {_lib.BP_MAX_COILS} coils, got {pk.n_coils}")
    windows = plan_windows(pk.flags, samp)
    wdev = torch.from_numpy(windows).to(device).contiguous()
    state = initial_state(case.pd, case.m_init, device)
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    run_forward(pk, state, wdev, 0, windows.shape[0], raw if pk.n_adc else None, status, max_ctas=max_ctas)
    sig = finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward")
    return sig.cpu(), final_m(state)
