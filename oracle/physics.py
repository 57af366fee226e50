"""CPU float64 oracle of blochparty's bound pool and scanner field model — TEST INFRASTRUCTURE ONLY.

Only ``tests/`` (and the oracle's own ``bloch.py``) import this module, as the checker; the product path never does.
Its arithmetic is written independently of the product's host code (``blochparty_b200.physics``) and pinned by the
fixtures ``tests/golden/mt_*.npz``, ``field_*.npz`` and ``sl_table.npz``, written by blochparty itself.

What it restates, in torch float64 (differentiable where the reference is):

* ``sl_table``: the super-Lorentzian integral F(x) = sqrt(2 pi) int_0^1 exp(-2 x^2 / s^2) / s du, s = |3u^2 - 1|
  (blochparty ``exchange.py:106-134``) at the reference's 4,097 points uniform in ln x over [1e-4, 30], by scipy's
  adaptive quadrature in ln |u - u0| on either side of the magic angle u0 = 1/sqrt(3);
* ``lineshape`` (``exchange.py:137-180``), ``z_exchange`` (``:215-244``), ``rf_frequency`` (``:182-212``);
* ``spin_fields`` (``fields.py:55-90``, ``:193-260``): encoding positions through the solid harmonics, here from
  scipy's associated Legendre functions in spherical coordinates (the reference uses Cartesian recurrences), and
  the concomitant coefficients.
"""

from __future__ import annotations

import functools
import math
from dataclasses import dataclass

import numpy as np
import torch

F64 = torch.float64
GAMMA_BAR = 42.577478518e6
SL_XMIN, SL_XMAX, SL_N = 1e-4, 30.0, 4097


@dataclass
class PoolCase:
    """The bound pool per spin (float64 (N,) tensors) and its lineshape."""

    f: torch.Tensor
    k: torch.Tensor
    t1: torch.Tensor
    t2: torch.Tensor
    dw: torch.Tensor
    shape: str = "superlorentzian"
    cutoff: float = 1e3


def pool_case(bound, n: int) -> PoolCase:
    conv = lambda v: torch.as_tensor(v, dtype=F64).detach().cpu().expand(n).clone()
    return PoolCase(conv(bound.f), conv(bound.k), conv(bound.t1), conv(bound.t2), conv(getattr(bound, "dw", 0.0)),
                    getattr(bound, "lineshape", "superlorentzian"), getattr(bound, "cutoff", 1e3))


def _sl_log_point(x: float) -> float:
    """ln F(x). Each side of u0 is integrated in y = ln v (v = |u - u0|), its integrand scaled by
    exp(2 x^2 / s_max^2) (s_max = 1 at u = 0, 2 at u = 1, the side's largest s), so that for large x the quadrature
    sees an integrand of order one at the side's end instead of e^-450; the scales come back in the log."""
    from scipy import integrate

    u0 = 1.0 / math.sqrt(3.0)
    logs = []
    for side, vmax, smax in ((-1.0, u0, 1.0), (1.0, 1.0 - u0, 2.0)):
        def f(y):  # v = e^y, dv = v dy
            v = math.exp(y)
            s = 3.0 * v * (2.0 * u0 + side * v)
            return math.exp(-2.0 * x * x * (1.0 / (s * s) - 1.0 / (smax * smax))) / s * v
        # s <= 3 v (2 u0 + v) < 4.8 v on both sides: below v = x / 77, s < x / 16 and the integrand is under
        # e^-512 of its scale
        lo = math.log(x / 77.0)
        if lo >= math.log(vmax):
            continue
        val, _ = integrate.quad(f, lo, math.log(vmax), limit=400, epsabs=0.0, epsrel=1e-13)
        logs.append(math.log(val) - 2.0 * x * x / (smax * smax))
    top = max(logs)
    return 0.5 * math.log(2.0 * math.pi) + top + math.log(sum(math.exp(v - top) for v in logs))


def _sl_point(x: float) -> float:
    return math.exp(_sl_log_point(x))


@functools.lru_cache(maxsize=1)
def sl_table() -> tuple[torch.Tensor, torch.Tensor]:
    """(ln x, ln F) float64 (SL_N,) each."""
    lx = np.linspace(math.log(SL_XMIN), math.log(SL_XMAX), SL_N)
    lf = np.maximum([_sl_log_point(float(math.exp(v))) for v in lx], math.log(1e-300))
    return torch.from_numpy(lx), torch.from_numpy(lf)


def lineshape(pool: PoolCase, delta: torch.Tensor) -> torch.Tensor:
    """G(2 pi delta) [s] per spin."""
    t2 = pool.t2
    if pool.shape == "lorentzian":
        x = 2 * math.pi * delta * t2
        return t2 / (1 + x * x)
    x = 2 * math.pi * delta.abs().clamp_min(pool.cutoff) * t2
    lx, lf = sl_table()
    pos = ((torch.log(x.clamp_min(SL_XMIN)) - lx[0]) / (lx[1] - lx[0])).clamp(0, SL_N - 1)
    i = pos.detach().floor().long().clamp(max=SL_N - 2)
    a = pos - i
    val = torch.exp(lf[i] * (1 - a) + lf[i + 1] * a)
    return t2 * torch.where(x > SL_XMAX, torch.zeros_like(val), val)


def rf_frequency(dt: torch.Tensor, rf: torch.Tensor, is_rf) -> torch.Tensor:
    """(S,) the RF's instantaneous frequency [Hz]: minus the phase step to each neighbouring RF segment over the
    pair's mean duration, averaged over the neighbours that carry RF; 0 without one."""
    S = dt.shape[0]
    out = torch.zeros(S, dtype=F64)
    live = [bool(is_rf[s]) and float(rf[s, 0] ** 2 + rf[s, 1] ** 2) > 0 for s in range(S)]
    for s in range(S):
        acc, cnt = 0.0, 0
        for nb in (s - 1, s + 1):
            if 0 <= nb < S and live[s] and live[nb]:
                a, b = (nb, s) if nb < s else (s, nb)
                xa, ya, xb, yb = float(rf[a, 0]), float(rf[a, 1]), float(rf[b, 0]), float(rf[b, 1])
                # angle(z_b conj(z_a)); a real waveform's sign change is +pi or -pi by the sign of the zero
                # imaginary part yb xa - xb ya, as blochparty forms it
                ang = math.atan2(yb * xa - xb * ya, xb * xa + yb * ya)
                acc += -ang / (2 * math.pi * 0.5 * float(dt[a] + dt[b]))
                cnt += 1
        out[s] = acc / max(cnt, 1)
    return out


def z_exchange(mz, mb, t, pd, r1, pool: PoolCase, w=None):
    """(Mz, Mzb) after a time t of longitudinal relaxation and exchange with the bound pool (saturation rate w), by
    the 2x2 matrix exponential of the linear system about its steady state."""
    kf, kb, r1b = pool.k * pool.f, pool.k, 1.0 / pool.t1
    a11, a12, a21 = -(r1 + kf), kb, kf
    a22 = -(r1b + kb) if w is None else -(r1b + kb + w)
    c1, c2 = r1 * pd, r1b * pool.f * pd
    det = a11 * a22 - a12 * a21
    z1, z2 = -(a22 * c1 - a12 * c2) / det, -(a11 * c2 - a21 * c1) / det
    tr = 0.5 * (a11 + a22)
    h = 0.5 * (a11 - a22)
    q = torch.sqrt(h * h + a12 * a21)
    # exp(A t) = e^{tr t} (cosh(q t) I + sinh(q t)/q (A - tr I)), written as e^{(tr +- q) t}
    ep, em = torch.exp((tr + q) * t), torch.exp((tr - q) * t)
    ch = 0.5 * (ep + em)
    sh = torch.where(q > 0, 0.5 * (ep - em) / torch.where(q > 0, q, torch.ones_like(q)), t * torch.exp(tr * t))
    d1, d2 = mz - z1, mb - z2
    return z1 + ch * d1 + sh * (h * d1 + a12 * d2), z2 + ch * d2 + sh * (a21 * d1 - h * d2)


def saturation(pool: PoolCase, rf, b1, delta):
    w1sq = (2 * math.pi) ** 2 * (rf[0] ** 2 + rf[1] ** 2)
    if b1 is not None:
        w1sq = w1sq * b1 * b1
    return w1sq * lineshape(pool, delta)


def _solid(pos: np.ndarray, n_max: int, r0: float):
    """(N, L, L) cosine and sine solid harmonics R0 (r/R0)^n N_nm P_n^m(cos theta) (cos m phi, sin m phi) from
    scipy's P_n^m (its Condon-Shortley phase (-1)^m removed)."""
    from scipy.special import lpmv

    r = np.linalg.norm(pos, axis=1)
    ct = np.where(r > 0, pos[:, 2] / np.where(r > 0, r, 1.0), 1.0)
    phi = np.arctan2(pos[:, 1], pos[:, 0])
    L = n_max + 1
    cs, sn = np.zeros((pos.shape[0], L, L)), np.zeros((pos.shape[0], L, L))
    for n in range(L):
        for m in range(n + 1):
            norm = 1.0 if m == 0 else math.sqrt((2 * n + 1) * math.factorial(n - m) / (2 * math.factorial(n + m)))
            base = r0 * (r / r0) ** n * norm * (-1.0) ** m * lpmv(m, n, ct)
            cs[:, n, m] = base * np.cos(m * phi)
            sn[:, n, m] = base * np.sin(m * phi)
    return cs, sn


def spin_fields(scanner, pos: torch.Tensor):
    """(encoding positions (N, 3), coefficients (N, 6 or 7) or None, mode) float64 for ``scanner``."""
    p = pos.detach().to(F64).cpu()
    if scanner is None:
        return p, None, 0
    enc = p
    nl = scanner.nonlinearity
    if nl is not None:
        alpha = torch.as_tensor(nl.alpha, dtype=F64).numpy()
        beta = torch.as_tensor(nl.beta, dtype=F64).numpy()
        L = alpha.shape[-1]
        cs, sn = _solid(p.numpy(), L - 1, float(nl.r0))
        keep = np.tril(np.ones((L, L)))
        d = np.einsum("pnm,anm->pa", cs, alpha * keep) + np.einsum("pnm,anm->pa", sn, beta * keep)
        enc = p + torch.from_numpy(d)
    if scanner.concomitant is None or scanner.field_strength is None:
        return enc, None, 0
    f0 = GAMMA_BAR * float(scanner.field_strength)
    a = float(scanner.z_asymmetry)
    x, y, z = p.unbind(-1)
    ax = torch.stack([z, torch.zeros_like(x), -a * x], -1)
    ay = torch.stack([torch.zeros_like(x), z, -(1 - a) * y], -1)
    if scanner.concomitant == "leading":
        # (Bx^2 + By^2) / (2 f0) as a quadratic form in g: coefficients of gx^2, gy^2, gz^2, gx gy, gx gz, gy gz
        c = torch.stack([ax[:, 0] ** 2 + ay[:, 0] ** 2, ax[:, 1] ** 2 + ay[:, 1] ** 2, ax[:, 2] ** 2 + ay[:, 2] ** 2,
                         2 * (ax[:, 0] * ax[:, 1] + ay[:, 0] * ay[:, 1]), 2 * (ax[:, 0] * ax[:, 2] + ay[:, 0] * ay[:, 2]),
                         2 * (ax[:, 1] * ax[:, 2] + ay[:, 1] * ay[:, 2])], -1) / (2 * f0)
        return enc, c, 1
    return enc, torch.cat([ax, ay, torch.full((p.shape[0], 1), f0, dtype=F64)], -1), 2


def concomitant(lin, g, conc, mode):
    """Concomitant field [Hz] per spin for gradient g (3,), the rest of the offset ``lin`` (N,)."""
    if mode == 1:
        gx, gy, gz = g[0], g[1], g[2]
        return conc @ torch.stack([gx * gx, gy * gy, gz * gz, gx * gy, gx * gz, gy * gz])
    tx, ty = conc[:, :3] @ g, conc[:, 3:6] @ g
    t2 = tx * tx + ty * ty
    u = conc[:, 6] + lin
    return t2 / (torch.sqrt(u * u + t2) + u)
