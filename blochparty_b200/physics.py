"""The bound pool (magnetization transfer, rate model) and the scanner field model: their types and the host side of
the physics variant of the forward kernel (``bp_forward_physics``).

Types, names and units follow blochparty, so its own objects are accepted as they are (read by attribute):

* ``BoundPool`` (blochparty ``exchange.py:59-104``): per spin f = M0b / M0, k the exchange rate from the bound to
  the free pool [Hz], T1 and T2 of the bound pool [s], its resonance shift dw [Hz], the lineshape ("lorentzian" or
  "superlorentzian") and the super-Lorentzian's cutoff [Hz]. The rate model only: the generalized Bloch model and
  the uncut lineshape (``cutoff=None``, a lineshape from fitted Green's-function modes) are refused.
* ``Scanner`` and ``GradientNonlinearity`` (blochparty ``fields.py:93-187``): concomitant fields at field strength
  B0 ("leading" order or "exact" |B|), the z coil's asymmetry, and a solid-harmonic gradient nonlinearity.

What the host derives, in float64 (then rounded once to float32 for the device):

* the super-Lorentzian's integral F(x) = sqrt(2 pi) int_0^1 exp(-2 x^2 / s^2) / s du, s = |3u^2 - 1| (Morrison and
  Henkelman's lineshape, blochparty ``exchange.py:106-134``), tabulated in ln F at 4,097 points uniform in
  ln x over [1e-4, 30] (the reference's grid), computed here by composite 16-point Gauss-Legendre on panels
  graded geometrically towards the magic angle u0 = 1/sqrt(3) and towards u = 0 and 1 (``sl_integral``);
* the RF's instantaneous frequency per segment (blochparty ``exchange.rf_frequency``, :182-212): minus the phase
  step between consecutive RF segments over their mean duration, averaged over both neighbours that carry RF;
* the field model's per-spin inputs (blochparty ``fields.spin_fields``, :248-260): encoding positions r + d(r),
  d the solid-harmonic expansion, and the concomitant coefficients at the true positions.
"""

from __future__ import annotations

import ctypes
import functools
import math
from dataclasses import dataclass

import numpy as np
import torch
from torch import Tensor

GAMMA_BAR = 42.577478518e6  # 1H gyromagnetic ratio / 2 pi [Hz/T]
SL_CUTOFF = 1e3  # [Hz] the super-Lorentzian's default cutoff
LINESHAPES = ("superlorentzian", "lorentzian")
CONCOMITANT_MODES = ("leading", "exact")
SL_XMIN, SL_XMAX, SL_N = 1e-4, 30.0, 4097
LINE_HEADER = 6  # floats before the table in the device lineshape buffer


@dataclass
class BoundPool:
    """Bound-pool parameters per spin (tensors (N,) or scalars), blochparty ``exchange.BoundPool``."""

    f: Tensor | float
    k: Tensor | float
    t1: Tensor | float
    t2: Tensor | float
    dw: Tensor | float = 0.0
    lineshape: str = "superlorentzian"
    cutoff: float | None = SL_CUTOFF
    model: str = "rate"
    memory: float = 300.0

    def __post_init__(self):
        if self.lineshape not in LINESHAPES:
            raise ValueError(f"lineshape must be one of {LINESHAPES}, got {self.lineshape!r}")
        if self.model not in ("rate", "generalized"):
            raise ValueError(f"model must be 'rate' or 'generalized', got {self.model!r}")
        if self.cutoff is not None and not self.cutoff > 0:
            raise ValueError(f"cutoff must be positive or None, got {self.cutoff!r}")


@dataclass
class GradientNonlinearity:
    """Solid-harmonic deviation of each gradient coil from linearity (blochparty ``fields.GradientNonlinearity``):
    alpha, beta (3, L, L) coefficients A_nm, B_nm of the x, y, z coils (entries with m > n ignored), r0 [m]."""

    alpha: Tensor
    beta: Tensor
    r0: float


@dataclass
class Scanner:
    """Hardware field model (blochparty ``fields.Scanner``): B0 [T] (concomitant fields are modelled when given),
    ``concomitant`` "leading", "exact" or None, the z coil's asymmetry a, and a gradient nonlinearity."""

    field_strength: float | Tensor | None = None
    concomitant: str | None = "leading"
    z_asymmetry: float | Tensor = 0.5
    nonlinearity: GradientNonlinearity | None = None

    def __post_init__(self):
        if self.concomitant is not None and self.concomitant not in CONCOMITANT_MODES:
            raise ValueError(f"concomitant must be one of {CONCOMITANT_MODES} or None, got {self.concomitant!r}")


def _f64(v) -> np.ndarray:
    if isinstance(v, Tensor):
        return v.detach().to(torch.float64).cpu().numpy()
    return np.asarray(v, dtype=np.float64)


# ---------------------------------------------------------------- the super-Lorentzian


def sl_integral(x: np.ndarray) -> np.ndarray:
    """F(x) = sqrt(2 pi) int_0^1 exp(-2 x^2 / s^2) / s du, s = |3u^2 - 1|, for x >= SL_XMIN (float64).

    With v the distance from u0 = 1/sqrt(3), s = 3 v (2 u0 -/+ v) on either side. Below v_lo = SL_XMIN / (32 sqrt 3)
    (s < x / 16) the integrand is below e^-512 of its scale and is left out. The rest of each side is split at its
    middle, and each half cut into panels that grow geometrically (ratio 1.25) away from its outer end: towards
    u0, where the integrand goes as 1/s until exp(-2 x^2 / s^2) cuts it off, and towards u = 0 or 1, where for large
    x it is a steep exponential. Every panel takes 16 Gauss-Legendre nodes."""
    x = np.atleast_1d(np.asarray(x, dtype=np.float64))
    u0 = 1.0 / math.sqrt(3.0)
    t, w = np.polynomial.legendre.leggauss(16)
    vlo = SL_XMIN / (32.0 * math.sqrt(3.0))
    out = np.zeros_like(x)

    def graded(a, b, towards_a):
        """Panel ends on [a, b], geometric from the end named by towards_a (first panel 1e-7 of the length)."""
        length = b - a
        d = 1e-7 * length * 1.25 ** np.arange(int(np.ceil(np.log(1e7) / np.log(1.25))) + 1)
        d = np.concatenate([[0.0], d[d < length], [length]])
        return a + d if towards_a else b - d[::-1]

    for side, vmax in ((-1.0, u0), (1.0, 1.0 - u0)):
        mid = 0.5 * (vlo + vmax)
        edges = np.concatenate([graded(vlo, mid, True), graded(mid, vmax, False)[1:]])
        a, b = edges[:-1], edges[1:]
        v = 0.5 * (a + b)[:, None] + 0.5 * (b - a)[:, None] * t  # (P, 16)
        wt = 0.5 * (b - a)[:, None] * w
        s = (3.0 * v * (2.0 * u0 + side * v)).ravel()
        wt = wt.ravel()
        for i in range(0, x.shape[0], 256):
            xb = x[i:i + 256, None]
            out[i:i + 256] += (np.exp(-2.0 * (xb / s) ** 2) / s * wt).sum(1)
    return math.sqrt(2.0 * math.pi) * out


@functools.lru_cache(maxsize=1)
def sl_table() -> tuple[float, float, np.ndarray]:
    """(ln x0, step, ln F (SL_N,)) float64: ln F at ln x uniform over [ln SL_XMIN, ln SL_XMAX] (ln F floored at
    ln 1e-300, finite in float32)."""
    lx = np.linspace(math.log(SL_XMIN), math.log(SL_XMAX), SL_N)
    log_f = np.log(np.maximum(sl_integral(np.exp(lx)), 1e-300))
    return float(lx[0]), float(lx[1] - lx[0]), log_f


def line_buffer(lineshape: str, cutoff: float) -> np.ndarray:
    """The device lineshape buffer (float32): kind, cutoff, ln x0, step, x_min, size, then the table."""
    if lineshape == "lorentzian":
        return np.array([1.0, 0.0, 0.0, 1.0, 0.0, 0.0], dtype=np.float32)
    lx0, step, log_f = sl_table()
    head = np.array([2.0, cutoff, lx0, step, SL_XMIN, SL_N], dtype=np.float64)
    return np.concatenate([head, log_f]).astype(np.float32)


def lineshape(delta: np.ndarray, t2: np.ndarray, shape: str, cutoff: float = SL_CUTOFF) -> np.ndarray:
    """G(2 pi delta) [s] in float64 (host checks of the device table; blochparty ``exchange.lineshape``)."""
    delta, t2 = np.asarray(delta, dtype=np.float64), np.asarray(t2, dtype=np.float64)
    if shape == "lorentzian":
        x = 2.0 * math.pi * delta * t2
        return t2 / (1.0 + x * x)
    x = 2.0 * math.pi * np.maximum(np.abs(delta), cutoff) * t2
    lx0, step, log_f = sl_table()
    pos = np.clip((np.log(np.maximum(x, SL_XMIN)) - lx0) / step, 0.0, SL_N - 1)
    i = np.minimum(np.floor(pos).astype(np.int64), SL_N - 2)
    a = pos - i
    val = np.exp(log_f[i] * (1.0 - a) + log_f[i + 1] * a)
    return t2 * np.where(x > SL_XMAX, 0.0, val)


# ---------------------------------------------------------------- the RF's frequency


def rf_frequency(dt, rf, is_rf, rf_freq=None) -> np.ndarray:
    """(S,) float64 instantaneous RF frequency [Hz] (blochparty's convention: a pulse turning as exp(-i 2 pi f t)
    is resonant with spins at offset f), or ``rf_freq`` itself when the sequence carries one."""
    dt = _f64(dt)
    if rf_freq is not None:
        f = _f64(rf_freq)
        if f.shape != dt.shape:
            raise ValueError(f"Sequence.rf_freq has shape {f.shape}, expected {dt.shape}")
        return f
    rf = _f64(rf)
    live = np.asarray(is_rf, dtype=bool) & ((rf[:, 0] ** 2 + rf[:, 1] ** 2) > 0)
    if dt.shape[0] < 2:
        return np.zeros_like(dt)
    # the phase step from segment s to s + 1, angle(z_{s+1} conj(z_s)), its real and imaginary parts as two
    # products each: a sign change of a real waveform (a sinc's lobes) is a step of +pi or -pi by the sign of the
    # zero imaginary part, y1 x0 - x1 y0, which this order of operations keeps as blochparty's does
    x, y = rf[:, 0], rf[:, 1]
    re = x[1:] * x[:-1] + y[1:] * y[:-1]
    im = y[1:] * x[:-1] - x[1:] * y[:-1]
    both = live[1:] & live[:-1]
    step = np.where(both, -np.arctan2(np.where(both, im, 0.0), np.where(both, re, 1.0)) / (math.pi * (dt[1:] + dt[:-1])),
                    0.0)
    total = np.concatenate([[0.0], step]) + np.concatenate([step, [0.0]])
    count = np.concatenate([[0.0], both]) + np.concatenate([both, [0.0]])
    return total / np.maximum(count, 1.0)


# ---------------------------------------------------------------- the field model


def _t64(v, like: Tensor) -> Tensor:
    """v as a float64 tensor on like's device, keeping its autograd graph."""
    if isinstance(v, Tensor):
        return v.to(dtype=torch.float64, device=like.device)
    return torch.as_tensor(v, dtype=torch.float64, device=like.device)


def solid_harmonics(pos: Tensor, n_max: int, r0: float) -> tuple[Tensor, Tensor]:
    """(N, n_max + 1, n_max + 1) cosine and sine solid harmonics R0 (r/R0)^n N_nm P_n^m(cos theta) (cos m phi,
    sin m phi) (zero for m > n), N_nm = sqrt((2n + 1) (n - m)! / (2 (n + m)!)) for m > 0 and 1 for m = 0, P_n^m
    without the Condon-Shortley phase, in Cartesian form: (x + i y)^m / R0^m, times r^n P_n^m / rho^m from its
    three-term recurrence in n (Q_m^m = (2m - 1)!!, Q_{m+1}^m = (2m + 1) z Q_m^m,
    (n - m) Q_n^m = (2n - 1) z Q_{n-1}^m - (n + m - 1) r^2 Q_{n-2}^m, in units of R0). float64 torch, differentiable
    in the positions."""
    p = pos / r0
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    r2 = x * x + y * y + z * z
    L = n_max + 1
    zero = torch.zeros_like(x)
    cs = [[zero] * L for _ in range(L)]
    sn = [[zero] * L for _ in range(L)]
    cm, sm = torch.ones_like(x), torch.zeros_like(x)  # (x + i y)^m
    dfact = 1.0  # (2m - 1)!!
    for m in range(L):
        if m > 0:
            cm, sm = x * cm - y * sm, x * sm + y * cm
            dfact *= 2 * m - 1
        q_prev, q = None, torch.full_like(x, dfact)
        for deg in range(m, L):
            if deg == m + 1:
                q_prev, q = q, (2 * m + 1) * z * q
            elif deg > m + 1:
                q_prev, q = q, ((2 * deg - 1) * z * q - (deg + m - 1) * r2 * q_prev) / (deg - m)
            norm = 1.0 if m == 0 else math.sqrt((2 * deg + 1) * math.factorial(deg - m) / (2 * math.factorial(deg + m)))
            cs[deg][m] = r0 * norm * q * cm
            sn[deg][m] = r0 * norm * q * sm
    stack = lambda t: torch.stack([torch.stack(row, -1) for row in t], -2)
    return stack(cs), stack(sn)


def displacement(nl, pos: Tensor) -> Tensor:
    """(N, 3) encoding position minus true position of ``nl`` (alpha, beta (3, L, L), r0), differentiable in the
    positions and the coefficients."""
    alpha, beta = _t64(nl.alpha, pos), _t64(nl.beta, pos)
    L = alpha.shape[-1]
    keep = torch.ones(L, L, dtype=torch.bool, device=pos.device).tril()
    cs, sn = solid_harmonics(pos, L - 1, float(nl.r0))
    return torch.einsum("pnm,anm->pa", cs, alpha * keep) + torch.einsum("pnm,anm->pa", sn, beta * keep)


def transverse_rows(pos: Tensor, a) -> Tensor:
    """(N, 6) rows (ax, ay) of the transverse field (Bx, By) = (ax . g, ay . g) [Hz] of the cylindrical coil set
    (Bx = gx z - a gz x, By = gy z - (1 - a) gz y)."""
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    zero = torch.zeros_like(x)
    return torch.stack([z, zero, -a * x, zero, z, -(1.0 - a) * y], dim=-1)


def concomitant_coefficients(pos: Tensor, f0, a) -> Tensor:
    """(N, 6) c with f_c = c . (gx^2, gy^2, gz^2, gx gy, gx gz, gy gz) = (Bx^2 + By^2) / (2 f0) [Hz]."""
    t = transverse_rows(pos, a)
    ax, ay = t[:, :3], t[:, 3:]
    sq = ax * ax + ay * ay
    cross = lambda i, j: 2.0 * (ax[:, i] * ax[:, j] + ay[:, i] * ay[:, j])
    return torch.stack([sq[:, 0], sq[:, 1], sq[:, 2], cross(0, 1), cross(0, 2), cross(1, 2)], dim=-1) / (2.0 * f0)


def spin_fields_torch(scanner, pos: Tensor) -> tuple[Tensor, Tensor | None, int]:
    """(encoding positions (N, 3), coefficients (N, 6) or (N, 7) or None, mode 0 / 1 / 2) as float64 tensors on
    pos's device for ``scanner`` (None: the ideal scanner) at the true positions ``pos``: differentiable in the
    positions, the nonlinearity's coefficients, the field strength and the z coil's asymmetry."""
    p = pos.to(torch.float64)
    if scanner is None:
        return p, None, 0
    nl = getattr(scanner, "nonlinearity", None)
    enc = p if nl is None else p + displacement(nl, p)
    mode = getattr(scanner, "concomitant", None)
    b0 = getattr(scanner, "field_strength", None)
    if mode is None or b0 is None:
        return enc, None, 0
    f0 = GAMMA_BAR * _t64(b0, p)
    a = _t64(getattr(scanner, "z_asymmetry", 0.5), p)
    if mode == "leading":
        return enc, concomitant_coefficients(p, f0, a), 1
    return enc, torch.cat([transverse_rows(p, a), f0.expand(p.shape[0], 1)], dim=1), 2


def spin_fields(scanner, pos) -> tuple[np.ndarray, np.ndarray | None, int]:
    """``spin_fields_torch`` as float64 numpy arrays (no gradients)."""
    with torch.no_grad():
        enc, conc, mode = spin_fields_torch(scanner, torch.as_tensor(_f64(pos)))
    return enc.numpy(), None if conc is None else conc.numpy(), mode


def gradient_moments2(dt, grad) -> np.ndarray:
    """(S, 6) float64 dt (gx^2, gy^2, gz^2, gx gy, gx gz, gy gz) per segment."""
    dt, g = _f64(dt), _f64(grad)
    gx, gy, gz = g[:, 0], g[:, 1], g[:, 2]
    return np.stack([gx * gx, gy * gy, gz * gz, gx * gy, gx * gz, gy * gz], axis=-1) * dt[:, None]


# ---------------------------------------------------------------- checks


def check_bound(bound) -> None:
    """NotImplementedError for the bound-pool models this engine does not run."""
    if getattr(bound, "model", "rate") == "generalized":
        raise NotImplementedError(
            "b200 engine: simulating with the generalized Bloch bound pool is not implemented; "
            "use blochparty.simulate (the core)")
    if getattr(bound, "lineshape", "superlorentzian") == "superlorentzian" and getattr(bound, "cutoff", SL_CUTOFF) is None:
        raise NotImplementedError(
            "b200 engine: simulating with a bound pool without a lineshape cutoff (cutoff=None) is not implemented; "
            "use blochparty.simulate (the core)")


def pool_rows(bound, n: int) -> np.ndarray:
    """[5][N] float64: f, k, 1/T1b, T2b, dw per spin."""
    rows = np.empty((5, n))
    for i, v in enumerate((bound.f, bound.k, bound.t1, bound.t2, getattr(bound, "dw", 0.0))):
        rows[i] = np.broadcast_to(_f64(v), (n,))
    rows[2] = 1.0 / rows[2]
    return rows


# ---------------------------------------------------------------- the forward


def forward_physics(inp, device, bound=None, scanner=None, bound_only=None, rf_freq=None, max_ctas: int = 0):
    """Signal (C, A) complex64, m (N, 3) float32 and the bound pool's Mz (N,) float32 (None without a pool), on the
    CPU, of a case with a bound pool and/or a scanner field model (``inp``: ``api.Inputs``; ``m_init`` may have a
    fourth column, the bound pool's Mz, default f PD). One launch of ``bp_forward_physics`` over every window."""
    from . import _lib, engine
    from ._lib import ptr

    F32, F64 = torch.float32, torch.float64
    n = inp.pd.shape[0]
    S = inp.dt.shape[0]
    if bound is not None:
        check_bound(bound)
    if inp.m_init is not None and inp.m_init.shape[-1] == 4 and bound is None:
        raise ValueError("m_init has a bound-pool column but the phantom has no bound pool")
    enc, conc, mode = spin_fields(scanner, inp.pos)
    spins, sens = engine.pack_spins(torch.from_numpy(enc), inp.pd, inp.t1, inp.t2, inp.db0, inp.b1, inp.coils,
                                    device)
    is_rf = engine._bools(inp.is_rf, S)
    bo = np.zeros(S, dtype=bool) if bound_only is None else engine._bools(bound_only, S) & is_rf
    if bound is None:  # RF that only a bound pool would feel: free segments for the water alone
        is_rf = is_rf & ~bo
        bo[:] = False
    segs, seg64, psi, flags, n_adc = engine.pack_segments(inp.dt, inp.rf, inp.grad, inp.b0_offset, inp.adc_phase,
                                                          is_rf, inp.adc, inp.spoil, device)
    if bo.any():
        bits = torch.from_numpy(bo.astype(np.int32) * _lib.BP_BOUND_ONLY).to(device)
        segs.view(torch.int32)[:, 7] |= bits
        flags |= bo.astype(np.int32) * _lib.BP_BOUND_ONLY
    n_coils = inp.coils.shape[1]
    samp = _lib.lib().bp_forward_samp_max(n_coils)
    if samp <= 0:
        raise ValueError(f"at most {_lib.BP_MAX_COILS} coils, got {n_coils}")
    windows = engine.plan_windows(flags, samp)
    wdev = torch.from_numpy(windows).to(device).contiguous()
    m3 = None if inp.m_init is None else inp.m_init[:, :3]
    state = engine.initial_state(inp.pd, m3, device)
    keep = []  # device buffers the launch reads
    ph = _lib.BpPhysics()
    bstate = None
    if bound is not None:
        rows = pool_rows(bound, n)
        pool = torch.from_numpy(rows).to(F32).to(device).contiguous()
        if inp.m_init is not None and inp.m_init.shape[-1] == 4:
            mb64 = inp.m_init[:, 3].detach().cpu().to(F64)
        else:
            mb64 = torch.from_numpy(rows[0]) * inp.pd.detach().cpu().to(F64)
        hi = mb64.to(F32)
        bstate = torch.stack([hi, (mb64 - hi.to(F64)).to(F32)]).to(device).contiguous()
        f_rf = torch.from_numpy(rf_frequency(inp.dt, inp.rf, is_rf | bo, rf_freq)).to(F32).to(device).contiguous()
        cutoff = getattr(bound, "cutoff", SL_CUTOFF)
        line = torch.from_numpy(line_buffer(getattr(bound, "lineshape", "superlorentzian"),
                                            0.0 if cutoff is None else float(cutoff))).to(device).contiguous()
        keep += [pool, f_rf, line]
        ph.mt, ph.pool, ph.bstate, ph.rf_freq, ph.line = 1, ptr(pool), ptr(bstate), ptr(f_rf), ptr(line)
    if mode:
        cc = np.zeros((7, n), dtype=np.float32)
        cc[: conc.shape[1]] = conc.T
        conc_dev = torch.from_numpy(cc).to(device).contiguous()
        keep.append(conc_dev)
        ph.conc_mode, ph.conc = mode, ptr(conc_dev)
        if mode == 1:
            segq = torch.from_numpy(np.ascontiguousarray(gradient_moments2(inp.dt, inp.grad))).to(device)
            keep.append(segq)
            ph.segq = ptr(segq)
    raw = torch.zeros(max(n_adc, 1), 2 * n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    code = _lib.lib().bp_forward_physics(ptr(spins), ptr(sens), n, n_coils, ptr(segs), ptr(seg64), ptr(wdev), 0,
                                         windows.shape[0], ptr(state), ptr(raw) if n_adc else None, max_ctas,
                                         ctypes.byref(ph), ptr(status), _lib.stream_ptr())
    _lib.check(code, "bp_forward_physics")
    pk = engine.Packed(n, n_coils, n_adc, spins, sens, segs, seg64, psi, flags, device)
    sig = engine.finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward_physics")
    m_bound = None if bstate is None else (bstate[0].to(F64) + bstate[1].to(F64)).to(F32).cpu()
    return sig.cpu(), engine.final_m(state), m_bound
