"""CPU float64 oracle of blochparty's plain-Bloch simulation — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and reference arms may import
this module, and only as the checker or the timed CPU baseline; the product path (``blochparty_b200``) never
does. Parity is pinned against the reference itself: ``tests/golden/make_golden.py`` ran blochparty's core
engine (``engines/core.py:487``) in float64 on the cases in ``tests/golden/*.npz`` and
``tests/test_oracle.py`` checks this restatement against those outputs and gradients.

What it restates (blochparty ``engines/core.py``), for static spins with PD, T1, T2, dB0, B1+, receive coils,
``b0_offset`` and ``m_init``:

* steps (``core.py:322-334``): every RF segment alone; consecutive RF-free segments as one closed-form free run
  that ends at a spoiled segment (``merge=False`` steps every segment alone, the same result to rounding);
* RF segment (``core.py:124-150``, ``:71-74``, ``:97-108``): relax dt/2, rotate by the Rodrigues formula about
  w = -2 pi dt (b1 rf_x, b1 rf_y, G.r + dB0 + b0_offset), relax dt/2 (Strang splitting);
* free run (``core.py:268-319``): with t, k and B the cumulative time, gradient moment and b0_offset integral,
  Mxy(t) = Mxy(0) exp(-t/T2) exp(-i 2 pi (k.r + dB0 t + B)), Mz relaxing exactly; every ADC sample of the run is
  a sum over spins of one such exponential;
* a sample (``core.py:182-187``) is sum_spins (Mx + i My) * coil, demodulated by exp(-i adc_phase), taken at the
  end of its segment and before that segment's spoil (``core.py:391-392``), which zeroes Mx and My.

With a bound pool (rate model) and the scanner field model (``oracle.physics``), as the core does them:

* RF segments (``core.py:124-150``): the concomitant field added to bz (``core.py:115-121``); the bound pool's Mz
  exchanging with the water's Mz over each half step, saturated at W = w1^2 G(f_rf - bz - dw); a bound-only
  segment rotates the water about z alone;
* free runs (``core.py:268-319``): the concomitant phase (``core.py:190-218``: the cumulative dt-weighted gradient
  monomials at leading order, the per-segment |B| excess in exact mode) added to the phase, and the exact
  exchange step over the run instead of Mz's relaxation.

Everything is plain torch arithmetic on float64 CPU tensors, so ``torch.autograd`` through it is the gradient
oracle (the reference's own gradients are its core's autograd, blochparty ``tests/helpers.py:95-119``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

TWO_PI = 2.0 * math.pi
F64 = torch.float64
_BLOCK = 1 << 21  # spins x samples per block of a free run's exponentials


@dataclass
class Case:
    """One simulation's inputs as float64 CPU tensors (coils complex128)."""

    pos: torch.Tensor  # (N, 3)
    pd: torch.Tensor
    t1: torch.Tensor
    t2: torch.Tensor
    db0: torch.Tensor
    b1: torch.Tensor | None
    coils: torch.Tensor  # (N, C) complex
    dt: torch.Tensor  # (S,)
    rf: torch.Tensor  # (S, 2)
    grad: torch.Tensor  # (S, 3)
    adc_phase: torch.Tensor  # (S,)
    b0_offset: torch.Tensor | None
    is_rf: list
    adc: list
    spoil: list
    m_init: torch.Tensor | None = None  # (N, 3), or (N, 4) with the bound pool's Mz
    bound: object | None = None  # physics.PoolCase
    f_rf: torch.Tensor | None = None  # (S,) the RF's frequency [Hz] (with a bound pool)
    bound_only: list | None = None
    conc: torch.Tensor | None = None  # (N, 6) or (N, 7) concomitant coefficients
    mode: int = 0  # 0 none, 1 leading order, 2 exact


def case_from(phantom, seq, coils=None, m_init=None, scanner=None) -> Case:
    """A ``Case`` from phantom / sequence objects of either package (read by attribute), cast to float64 CPU; with
    a bound pool (``phantom.bound``), bound-only RF and ``scanner`` (the field model) as the core derives them."""
    from . import physics

    d = lambda t: None if t is None else t.to(F64).cpu()
    n = phantom.pd.shape[0]
    c = torch.ones(n, 1, dtype=torch.complex128) if coils is None else coils.to(torch.complex128).cpu()
    pos, conc, mode = physics.spin_fields(scanner, phantom.pos)
    case = Case(pos, d(phantom.pd), d(phantom.t1), d(phantom.t2), d(phantom.db0),
                d(getattr(phantom, "b1", None)), c, d(seq.dt), d(seq.rf), d(seq.grad), d(seq.adc_phase),
                d(getattr(seq, "b0_offset", None)), [bool(x) for x in seq.is_rf], [bool(x) for x in seq.adc],
                [bool(x) for x in seq.spoil], d(m_init), conc=conc, mode=mode)
    bound = getattr(phantom, "bound", None)
    bo = getattr(seq, "bound_only", None)
    case.bound_only = None if bo is None else [bool(x) for x in bo]
    if bound is not None:
        case.bound = physics.pool_case(bound, n)
        rf_freq = getattr(seq, "rf_freq", None)
        case.f_rf = d(rf_freq) if rf_freq is not None else physics.rf_frequency(case.dt, case.rf, case.is_rf)
    return case


def _steps(is_rf, spoil, merge):
    """[start, end) steps: single RF segments; runs of RF-free segments ending at a spoil (or the next RF)."""
    out, s, n = [], 0, len(is_rf)
    while s < n:
        e = s + 1
        if merge and not is_rf[s]:
            while e < n and not is_rf[e] and not spoil[e - 1]:
                e += 1
        out.append((s, e))
        s = e
    return out


def _relax(mx, my, mz, t, c):
    e2, e1 = torch.exp(-t / c.t2), torch.exp(-t / c.t1)
    return mx * e2, my * e2, c.pd + (mz - c.pd) * e1


def _rotate(mx, my, mz, wx, wy, wz):
    """Rotation by the vector w (right-handed, angle |w|): m cos + (w x m) sin/phi + w (w.m) (1 - cos)/phi^2.
    sin(phi)/phi and (1 - cos phi)/phi^2 = sinc(phi / 2pi)^2 / 2 are written with torch.sinc so that phi = 0 and
    its gradient are finite; phi carries a 1e-30 floor under the square root for the same reason."""
    phi = torch.sqrt(wx * wx + wy * wy + wz * wz + 1e-30)
    cs = torch.cos(phi)
    s1 = torch.sinc(phi / math.pi)
    s2 = 0.5 * torch.sinc(phi / TWO_PI) ** 2
    dot = wx * mx + wy * my + wz * mz
    return (cs * mx + s1 * (wy * mz - wz * my) + s2 * wx * dot,
            cs * my + s1 * (wz * mx - wx * mz) + s2 * wy * dot,
            cs * mz + s1 * (wx * my - wy * mx) + s2 * wz * dot)


def _sample(mx, my, psi, c):
    """(C,) complex demodulated coil sums of the current magnetization."""
    raw = ((mx + 1j * my)[:, None] * c.coils).sum(0)
    return raw * torch.exp(-1j * psi)


def _relax_bound(mx, my, mz, mb, t, c, w=None):
    from .physics import z_exchange

    e2 = torch.exp(-t / c.t2)
    mz, mb = z_exchange(mz, mb, t, c.pd, 1.0 / c.t1, c.bound, w)
    return mx * e2, my * e2, mz, mb


def _rf_step(mx, my, mz, s, c, off, mb=None):
    from . import physics

    g = c.grad[s]
    bz = c.pos @ g + c.db0 + (off[s] if off is not None else 0.0)
    if c.mode:
        bz = bz + physics.concomitant(bz, g, c.conc, c.mode)
    half = 0.5 * c.dt[s]
    bound_only = c.bound_only is not None and c.bound_only[s]
    if c.bound is not None:
        sat = physics.saturation(c.bound, c.rf[s], c.b1, c.f_rf[s] - bz - c.bound.dw)
        mx, my, mz, mb = _relax_bound(mx, my, mz, mb, half, c, sat)
    else:
        mx, my, mz = _relax(mx, my, mz, half, c)
    w = -TWO_PI * c.dt[s]
    if bound_only:
        wx, wy = torch.zeros_like(bz), torch.zeros_like(bz)
    else:
        wx, wy = w * c.rf[s, 0], w * c.rf[s, 1]
        if c.b1 is not None:
            wx, wy = wx * c.b1, wy * c.b1
        else:
            wx, wy = wx * torch.ones_like(bz), wy * torch.ones_like(bz)
    mx, my, mz = _rotate(mx, my, mz, wx, wy, w * bz)
    if c.bound is not None:
        return _relax_bound(mx, my, mz, mb, half, c, sat)
    return (*_relax(mx, my, mz, half, c), mb)


def _extra_phase(a, b, c, off):
    """(N, n) or (n,) cumulative phase [cycles] of the uniform offset and the concomitant field over [a, b)."""
    from . import physics

    dt, g = c.dt[a:b], c.grad[a:b]
    extra = torch.cumsum(off[a:b] * dt, 0) if off is not None else torch.zeros_like(dt)
    if c.mode == 1:
        gx, gy, gz = g.unbind(-1)
        q = torch.cumsum(torch.stack([gx * gx, gy * gy, gz * gz, gx * gy, gx * gz, gy * gz], -1) * dt[:, None], 0)
        extra = extra + c.conc @ q.T
    elif c.mode == 2:
        lin = c.pos @ g.T + c.db0[:, None] + (off[a:b] if off is not None else 0.0)  # (N, n)
        exc = torch.stack([physics.concomitant(lin[:, i], g[i], c.conc, 2) for i in range(b - a)], 1)
        extra = extra + torch.cumsum(exc * dt, 1)
    return extra


def _free_run(mx, my, mz, a, b, c, off, mb=None):
    """Closed-form run of RF-free segments [a, b): samples at its ADC segments, state at its end."""
    dt = c.dt[a:b]
    t = torch.cumsum(dt, 0)
    k = torch.cumsum(c.grad[a:b] * dt[:, None], 0)
    extra = _extra_phase(a, b, c, off)
    if extra.dim() == 1:
        extra = extra.expand(mx.shape[0], -1)
    samples = []
    idx = [i for i in range(b - a) if c.adc[a + i]]
    if idx:
        ii = torch.tensor(idx)
        v = (mx + 1j * my)[:, None] * c.coils  # (N, C)
        n = mx.shape[0]
        block = max(1, _BLOCK // max(n, 1))
        for j in range(0, len(idx), block):
            sel = ii[j:j + block]
            cyc = c.pos @ k[sel].T + c.db0[:, None] * t[sel] + extra[:, sel]  # (N, n) cycles
            e = torch.exp(-t[sel][None, :] / c.t2[:, None] - 1j * TWO_PI * cyc)
            raw = v.T @ e  # (C, n)
            samples.append(raw * torch.exp(-1j * c.adc_phase[a + sel])[None, :])
    cyc = c.pos @ k[-1] + c.db0 * t[-1] + extra[:, -1]
    cs, sn = torch.cos(-TWO_PI * cyc), torch.sin(-TWO_PI * cyc)
    mx, my = cs * mx - sn * my, sn * mx + cs * my
    if c.bound is not None:
        mx, my, mz, mb = _relax_bound(mx, my, mz, mb, t[-1], c)
    else:
        mx, my, mz = _relax(mx, my, mz, t[-1], c)
    return mx, my, mz, mb, samples


def simulate_with_pool(c: Case, merge: bool = True):
    """(signal (C, n_adc) complex128, m (N, 3) float64, the bound pool's Mz (N,) or None) of case ``c``."""
    n = c.pd.shape[0]
    mb = None
    if c.m_init is None:
        mx, my, mz = torch.zeros(n, dtype=F64), torch.zeros(n, dtype=F64), c.pd
    elif c.m_init.shape[-1] == 4:
        mx, my, mz, mb = c.m_init.unbind(-1)
    else:
        mx, my, mz = c.m_init.unbind(-1)
    if c.bound is not None and mb is None:
        mb = c.bound.f * c.pd
    is_rf = list(c.is_rf)
    if c.bound is None and c.bound_only is not None:  # RF only a bound pool would feel: free for the water
        is_rf = [r and not bo for r, bo in zip(is_rf, c.bound_only)]
    off = c.b0_offset
    cols = []
    for a, b in _steps(is_rf, c.spoil, merge):
        if is_rf[a]:
            mx, my, mz, mb = _rf_step(mx, my, mz, a, c, off, mb)
            if c.adc[a]:
                cols.append(_sample(mx, my, c.adc_phase[a], c)[:, None])
        else:
            mx, my, mz, mb, samples = _free_run(mx, my, mz, a, b, c, off, mb)
            cols += samples
        if c.spoil[b - 1]:
            mx, my = torch.zeros_like(mx), torch.zeros_like(my)
    n_coils = c.coils.shape[1]
    sig = torch.cat(cols, 1) if cols else torch.zeros(n_coils, 0, dtype=torch.complex128)
    return sig, torch.stack([mx, my, mz], -1), mb


def simulate(c: Case, merge: bool = True):
    """(signal (C, n_adc) complex128, m (N, 3) float64) of case ``c`` (module docstring)."""
    sig, m, _ = simulate_with_pool(c, merge)
    return sig, m


GRAD_INPUTS = ("pos", "pd", "t1", "t2", "db0", "b1", "coils", "dt", "rf", "grad", "adc_phase", "b0_offset", "m_init")


def gradients(c: Case, loss_fn, names=GRAD_INPUTS, merge: bool = True):
    """(loss value, {name: d loss / d input}) by autograd through ``simulate``; ``loss_fn(signal, m)`` -> scalar.
    Inputs that are None in the case are skipped."""
    from dataclasses import replace

    leaves = {}
    kw = {}
    for name in names:
        t = getattr(c, name)
        if t is None:
            continue
        leaf = t.detach().clone().requires_grad_()
        leaves[name] = leaf
        kw[name] = leaf
    cc = replace(c, **kw)
    sig, m = simulate(cc, merge)
    loss = loss_fn(sig, m)
    grads = torch.autograd.grad(loss, list(leaves.values()), allow_unused=True)
    return float(loss.detach()), {k: (None if g is None else g.detach()) for k, g in zip(leaves, grads)}
