"""Readout runs through a nonuniform FFT (``simulate(..., readout="nufft")``, forward only).

Replaces blochparty's NUFFT readouts (``engines/gpu/cuda/kernels.cu.in:91-140``, planned in
``engines/gpu/driver.py:236-266``; the design notes are ``docs/PERFORMANCE.md:98-148``). A readout run is L
consecutive samples with one free segment's factors, so spin j contributes z1_j q_j^p to sample p < L, with
q_j = exp(-dt r2_j) exp(-2 pi i x_j) and x_j the segment's phase in cycles, modulo 1. The sum over spins is a type-1
nonuniform DFT in x with a slowly varying decay:

* decay: exp(-p dt r2) ~ sum_m a_m(p) exp(-tau_m r2), Lagrange interpolation at M Chebyshev nodes tau_m on the run
  (time segmentation; M from the largest r2: the interpolation bound (r2 T)^M / (M! 2^(2M-1)) below 5e-8);
* phase: centred modes k = p - floor(L/2), exp(-2 pi i x p) = exp(-2 pi i x floor(L/2)) exp(-2 pi i x k);
* type-1 NUFFT (Dutt and Rokhlin; Greengard and Lee; the kernel of Barnett et al., FINUFFT): every spin spreads its
  weight onto an oversampled grid of G >= 2L cells with psi(z) = exp(beta (sqrt(1 - z^2) - 1)) over W = 8 cells
  (beta = 2.30 W), the grid's DFT at the L modes divided by G times the kernel's Fourier transform gives the sum.

The spins are sorted by x (of the dominant run class) before packing, so a tile of 128 spins reaches about W cells
and a CTA's accumulator holds its tiles' cells (``bp_forward_nufft``); the grid's DFT runs in float64
(``bp_nufft_finish``). The float64 prototype of this arithmetic is within 1.1e-7 (relative L2) of the direct sum
for W = 8, M = 3 and T2 down to 20 ms over a 127-sample run.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, engine
from ._lib import ptr

F32, F64 = torch.float32, torch.float64
W_DEFAULT = 8
BETA_PER_W = 2.30
MIN_RUN = 16
TILE = 128


def find_runs(flags: np.ndarray, min_len: int = MIN_RUN, max_len: int = _lib.BP_SEG_MAX):
    """[(first segment, length)] of the readout runs: consecutive free ADC segments each with the factors of the
    one before (``SAME_FREE``), a spoil only on the last, at least ``min_len`` long (longer runs are cut into
    pieces of at most ``max_len``, one window each)."""
    S = flags.shape[0]
    f = flags.astype(np.int64)
    is_sample = ((f & engine.ADC) != 0) & ((f & engine.RF) == 0)
    cont = np.zeros(S, dtype=bool)
    cont[1:] = is_sample[1:] & is_sample[:-1] & ((f[1:] & engine.SAME_FREE) != 0) & ((f[:-1] & engine.SPOIL) == 0)
    runs, s = [], 0
    while s < S:
        if not is_sample[s]:
            s += 1
            continue
        e = s + 1
        while e < S and cont[e]:
            e += 1
        a = s
        while e - a >= min_len:
            k = min(max_len, e - a)
            if k < min_len:
                break
            runs.append((a, k))
            a += k
        s = e
    return runs


def kernel_ft(kappa: np.ndarray, W: int, beta: float, G: int, n: int = 400) -> np.ndarray:
    """The Fourier transform of psi(u) = exp(beta (sqrt(1 - (2 G u / W)^2) - 1)) (|u| <= W / (2 G)) at the
    integer modes ``kappa`` (Gauss-Legendre quadrature in float64; psi is even)."""
    t, wt = np.polynomial.legendre.leggauss(n)
    u = t * W / (2.0 * G)
    val = np.exp(beta * (np.sqrt(1.0 - t * t) - 1.0)) * wt * W / (2.0 * G)
    return (val[None, :] * np.cos(2.0 * np.pi * np.outer(kappa, u))).sum(1)


def terms_for(r2_max: float, T: float, tol: float = 5e-8) -> int:
    """The time-segmentation terms M: the smallest with (r2 T)^M / (M! 2^(2M-1)) below ``tol``."""
    x = r2_max * T
    for M in range(1, _lib.BP_NUF_MAX_TERMS + 1):
        if x ** M / (math.factorial(M) * 2.0 ** (2 * M - 1)) < tol:
            return M
    raise ValueError(f"readout='nufft': the decay over a run (T/T2 = {x:.2f}) needs more than "
                     f"{_lib.BP_NUF_MAX_TERMS} terms; use readout='fp32'")


def segmentation(L: int, dt: float, M: int):
    """(nodes tau_m, coefficients a[m][p]): Lagrange interpolation of exp(-t r2) at t = p dt from M Chebyshev
    nodes on [0, (L - 1) dt]."""
    T = (L - 1) * dt
    nodes = 0.5 * T * (1.0 - np.cos((2.0 * np.arange(M) + 1.0) * np.pi / (2.0 * M)))
    tp = np.arange(L) * dt
    a = np.ones((M, L))
    for m in range(M):
        for q in range(M):
            if q != m:
                a[m] *= (tp - nodes[q]) / (nodes[m] - nodes[q])
    return nodes, a


def run_phase(spins32: np.ndarray, rec: np.ndarray, k64: np.ndarray) -> np.ndarray:
    """x_j = (k . r_j + dt dB0_j + beta) mod 1 [cycles] in float64 from the packed float32 spins (rows x, y, z, dB0
    of [8][n]) and one segment's record (dt, float32) and float64 moments (kx, ky, kz, beta): the phase the forward
    kernel's free factors use."""
    px, py, pz, db0 = (spins32[i].astype(np.float64) for i in (0, 1, 2, 6))
    cyc = k64[0] * px + k64[1] * py + k64[2] * pz + float(np.float32(rec[0])) * db0 + k64[3]
    return cyc - np.floor(cyc)


@dataclass
class NufftPlan:
    runs: np.ndarray  # (R, 2): first segment, length (all L of one class)
    L: int
    G: int
    W: int
    M: int
    beta: float
    nodes: np.ndarray
    weights: np.ndarray  # [M][L] float64: a_m(p) / (G psi^(p - floor(L/2)))
    order: np.ndarray  # spin order (sorted by x of the class)


def run_class(segs: np.ndarray, seg64: np.ndarray, flags: np.ndarray) -> np.ndarray:
    """(R, 2) the runs (first segment, length) of the class with the most samples: one segment's factors."""
    runs = find_runs(flags)
    if not runs:
        raise ValueError("readout='nufft': the sequence has no readout run of at least "
                         f"{MIN_RUN} samples with one segment's factors")
    classes: dict = {}
    for a, k in runs:
        key = (segs[a, :7].tobytes(), seg64[a].tobytes(), k)
        classes.setdefault(key, []).append((a, k))
    key = max(classes, key=lambda c: len(classes[c]) * c[2])
    return np.asarray(classes[key], dtype=np.int64)


def plan(spins32: np.ndarray, segs: np.ndarray, seg64: np.ndarray, flags: np.ndarray, W: int = W_DEFAULT) -> NufftPlan:
    """The NUFFT plan of a case: the runs of the class with the most samples, the spin order sorting them by x,
    the grid and kernel parameters, the decay terms and the output weights. ``spins32`` [8][n] float32 (packed
    order), ``segs`` (S, 8) float32 records, ``seg64`` (S, 4) float64, ``flags`` (S,) int32."""
    sel = run_class(segs, seg64, flags)
    a0 = int(sel[0, 0])
    x = run_phase(spins32, segs[a0], seg64[a0])
    order = np.argsort(x, kind="stable")
    r2max = float(np.max(spins32[5].astype(np.float64))) if spins32.shape[1] else 0.0
    return plan_of(sel, float(segs[a0, 0]), r2max, order, W)


def plan_of(sel: np.ndarray, dt: float, r2max: float, order, W: int = W_DEFAULT) -> NufftPlan:
    """The plan from the run class, its segment's dt, the largest 1/T2 and the spin order."""
    L = int(sel[0, 1])
    M = terms_for(r2max, (L - 1) * dt)
    G = 1 << int(math.ceil(math.log2(2 * L)))
    beta = BETA_PER_W * W
    nodes, acoef = segmentation(L, dt, M)
    kappa = np.arange(L) - L // 2
    weights = acoef / (G * kernel_ft(kappa, W, beta, G))[None, :]
    return NufftPlan(sel, L, G, W, M, beta, nodes, weights, order)


def spin_tables(p: NufftPlan, spins32: np.ndarray, segs: np.ndarray, seg64: np.ndarray):
    """Per spin (in the packed, sorted order): first cell, fraction, centring shift (float32 pairs), decay terms
    [M][n]; per 128-spin tile: the cells [lo, hi) its spins reach."""
    a0 = int(p.runs[0, 0])
    x = run_phase(spins32, segs[a0], seg64[a0])
    u = x * p.G
    fl = np.floor(u)
    base = (fl - p.W // 2 + 1).astype(np.int64)
    frac = (u - fl).astype(np.float32)
    h = p.L // 2
    ang = -2.0 * np.pi * ((x * h) - np.floor(x * h))
    shift = np.stack([np.cos(ang), np.sin(ang)], -1).astype(np.float32)
    r2 = spins32[5].astype(np.float64)
    decay = np.exp(-np.outer(p.nodes, r2)).astype(np.float32)
    n = spins32.shape[1]
    n_tiles = (n + TILE - 1) // TILE
    pad = n_tiles * TILE - n
    bt = np.concatenate([base, np.full(pad, base[-1] if n else 0)]).reshape(n_tiles, TILE)
    tiles = np.stack([bt.min(1), bt.max(1) + p.W], -1).astype(np.int32)
    span = int((tiles[:, 1] - tiles[:, 0]).max()) if n_tiles else 0
    if span * p.M > 64:
        raise ValueError(f"readout='nufft': a tile of {TILE} sorted spins spans {span} of {p.G} grid cells (too "
                         f"few spins for the grid: at most {64 // p.M}); use readout='fp32'")
    return base.astype(np.int32), frac, shift, decay, tiles


def windows_for(p: NufftPlan, flags: np.ndarray, samp_max: int):
    """(windows (W, 4) int32, run_of (W,) int32, run_rows (R,) int32): the forward's windows with every NUFFT run
    alone in one window (samples field 0: its rows are the run's, filled by ``bp_nufft_finish``), the other
    windows' first rows and sample counts from the true ADC flags."""
    S = flags.shape[0]
    pf = flags.copy()
    breaks = np.zeros(S, dtype=np.uint8)
    for a, k in p.runs:
        pf[a:a + k] &= ~np.int32(engine.ADC)
        breaks[a] = 1
        if a + k < S:
            breaks[a + k] = 1
    win = engine.plan_windows(pf, samp_max, breaks=breaks)
    adc = (flags & engine.ADC) != 0
    before = np.concatenate([[0], np.cumsum(adc)])
    win[:, 2] = before[win[:, 0]]
    win[:, 3] = before[win[:, 1]] - before[win[:, 0]]
    run_start = {int(a): r for r, (a, _) in enumerate(p.runs)}
    run_of = np.full(win.shape[0], -1, dtype=np.int32)
    rows = np.zeros(len(p.runs), dtype=np.int32)
    for w, (s0, s1, z, cnt) in enumerate(win):
        r = run_start.get(int(s0))
        if r is not None and s1 - s0 == p.runs[r][1]:
            run_of[w] = r
            rows[r] = z
            win[w, 3] = 0
    assert (run_of >= 0).sum() == len(p.runs)
    return np.ascontiguousarray(win), run_of, rows


def spin_tables_dev(p: NufftPlan, spins: torch.Tensor, rec: np.ndarray, k64: np.ndarray):
    """``spin_tables`` on the device from the packed (sorted) float32 spins [8][n]: the same float64 arithmetic
    in torch."""
    F64_ = torch.float64
    px, py, pz, db0 = (spins[i].to(F64_) for i in (0, 1, 2, 6))
    cyc = k64[0] * px + k64[1] * py + k64[2] * pz + float(np.float32(rec[0])) * db0 + k64[3]
    x = cyc - torch.floor(cyc)
    u = x * p.G
    fl = torch.floor(u)
    base = (fl - p.W // 2 + 1).to(torch.int64)
    frac = (u - fl).to(torch.float32)
    h = p.L // 2
    ang = -2.0 * math.pi * ((x * h) - torch.floor(x * h))
    shift = torch.stack([torch.cos(ang), torch.sin(ang)], -1).to(torch.float32)
    nodes = torch.as_tensor(p.nodes, dtype=F64_, device=spins.device)
    decay = torch.exp(-nodes[:, None] * spins[5].to(F64_)[None, :]).to(torch.float32)
    n = spins.shape[1]
    n_tiles = (n + TILE - 1) // TILE
    pad = n_tiles * TILE - n
    bt = torch.cat([base, base[-1:].expand(pad)]).reshape(n_tiles, TILE)
    tiles = torch.stack([bt.amin(1), bt.amax(1) + p.W], -1).to(torch.int32)
    span = int((tiles[:, 1] - tiles[:, 0]).max()) if n_tiles else 0
    if span * p.M > 64:
        raise ValueError(f"readout='nufft': a tile of {TILE} sorted spins spans {span} of {p.G} grid cells (too "
                         f"few spins for the grid: at most {64 // p.M}); use readout='fp32'")
    return (base.to(torch.int32).contiguous(), frac.contiguous(), shift.contiguous(), decay.contiguous(),
            tiles.contiguous())


class NufftRun:
    """The device side of a forward with NUFFT readout runs on a packed case (spins already in ``plan.order``).
    ``rec``, ``k64``: the class's segment record and float64 moments (host)."""

    def __init__(self, pk: engine.Packed, p: NufftPlan, rec: np.ndarray | None = None, k64: np.ndarray | None = None):
        dev = pk.device
        a0 = int(p.runs[0, 0])
        if rec is None:
            rec, k64 = pk.segs[a0].cpu().numpy(), pk.seg64[a0].cpu().numpy()
        base, frac, shift, decay, tiles = spin_tables_dev(p, pk.spins, rec, k64)
        samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
        win, run_of, rows = windows_for(p, pk.flags, samp)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.plan, self.pk = p, pk
        self.windows, self.wdev = win, t(win)
        self.run_of, self.base, self.frac = t(run_of), base, frac
        self.shift, self.decay, self.tiles = shift, decay, tiles
        self.rows, self.weights = t(rows), t(p.weights.astype(np.float64))
        self.grid = torch.zeros(len(p.runs), p.G, p.M, 2 * pk.n_coils, dtype=F64, device=dev)
        self.desc = _lib.BpNufft(ptr(self.run_of), ptr(self.base), ptr(self.frac), ptr(self.shift), ptr(self.decay),
                                 ptr(self.tiles), ptr(self.grid), p.G, p.W, p.M, p.beta)

    def run(self, state: torch.Tensor, raw: torch.Tensor, status: torch.Tensor, max_ctas: int = 0) -> None:
        """The whole forward from ``state``: the windows (runs spread onto the grid), then the runs' samples."""
        import ctypes

        pk, p = self.pk, self.plan
        self.grid.zero_()
        lib, st = _lib.lib(), _lib.stream_ptr()
        code = lib.bp_forward_nufft(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                    ptr(self.wdev), 0, self.windows.shape[0], ptr(state), ptr(raw), max_ctas,
                                    ctypes.byref(self.desc), ptr(status), st)
        _lib.check(code, "bp_forward_nufft")
        _lib.check(lib.bp_nufft_finish(ptr(self.grid), ptr(self.rows), len(p.runs), p.G, p.M, p.L, pk.n_coils,
                                       ptr(self.weights), ptr(raw), st), "bp_nufft_finish")


def sorted_inputs(inp, order: np.ndarray):
    """The inputs with every per-spin tensor in ``order``."""
    from dataclasses import replace

    idx = order if isinstance(order, torch.Tensor) else torch.from_numpy(order)
    take = lambda t: None if t is None else t[idx.to(t.device)]
    return replace(inp, pos=take(inp.pos), pd=take(inp.pd), t1=take(inp.t1), t2=take(inp.t2), db0=take(inp.db0),
                   b1=take(inp.b1), coils=take(inp.coils), m_init=take(inp.m_init))


def prepare(inp, device):
    """(packed case in the sorted order, NufftRun, order (a device tensor)): the case packed once onto the device,
    x of the run class from its float32 spins (float64 arithmetic on the device), the spins and coil sensitivities
    gathered into the order of x there, and the tables from them."""
    if inp.coils.shape[1] > 16:
        raise ValueError(f"readout='nufft' takes at most 16 coils, got {inp.coils.shape[1]}")
    spins, sens = engine.pack_spins(inp.pos, inp.pd, inp.t1, inp.t2, inp.db0, inp.b1, inp.coils, device)
    segs, seg64, psi, flags, n_adc = engine.pack_segments(inp.dt, inp.rf, inp.grad, inp.b0_offset, inp.adc_phase,
                                                          inp.is_rf, inp.adc, inp.spoil, "cpu")
    sel = run_class(segs.numpy(), seg64.numpy(), flags)
    a0 = int(sel[0, 0])
    rec, k64 = segs[a0].numpy(), seg64[a0].numpy()
    px, py, pz, db0 = (spins[i].to(torch.float64) for i in (0, 1, 2, 6))
    cyc = k64[0] * px + k64[1] * py + k64[2] * pz + float(np.float32(rec[0])) * db0 + k64[3]
    order = torch.argsort(cyc - torch.floor(cyc), stable=True)
    r2max = float(spins[5].max()) if spins.shape[1] else 0.0
    p = plan_of(sel, float(rec[0]), r2max, order)
    spins, sens = spins[:, order].contiguous(), sens[:, order].contiguous()
    segs_d, seg64_d, psi = segs.to(device).contiguous(), seg64.to(device).contiguous(), psi.to(device)
    engine.mark_small_rf(spins, segs_d, flags)
    pk = engine.Packed(spins.shape[1], inp.coils.shape[1], n_adc, spins, sens, segs_d, seg64_d, psi, flags, device)
    return pk, NufftRun(pk, p, rec, k64), order


def forward_nufft(inp, device, max_ctas: int = 0):
    """Signal (C, A) complex64 and m (N, 3) float32 on the CPU, with the readout runs through the NUFFT."""
    pk, nr, order = prepare(inp, device)
    state = engine.initial_state(inp.pd, inp.m_init, device)[:, order].contiguous()
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    nr.run(state, raw, status, max_ctas)
    sig = engine.finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward_nufft")
    inv = torch.empty_like(order)
    inv[order] = torch.arange(order.shape[0], device=order.device)
    return sig.cpu(), engine.final_m(state[:, inv])
