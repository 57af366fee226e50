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
    m_init: torch.Tensor | None = None  # (N, 3)


def case_from(phantom, seq, coils=None, m_init=None) -> Case:
    """A ``Case`` from phantom / sequence objects of either package (read by attribute), cast to float64 CPU."""
    d = lambda t: None if t is None else t.to(F64).cpu()
    n = phantom.pd.shape[0]
    c = torch.ones(n, 1, dtype=torch.complex128) if coils is None else coils.to(torch.complex128).cpu()
    return Case(d(phantom.pos), d(phantom.pd), d(phantom.t1), d(phantom.t2), d(phantom.db0),
                d(getattr(phantom, "b1", None)), c, d(seq.dt), d(seq.rf), d(seq.grad), d(seq.adc_phase),
                d(getattr(seq, "b0_offset", None)), [bool(x) for x in seq.is_rf], [bool(x) for x in seq.adc],
                [bool(x) for x in seq.spoil], d(m_init))


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


def _rf_step(mx, my, mz, s, c, off):
    g = c.grad[s]
    bz = c.pos @ g + c.db0 + (off[s] if off is not None else 0.0)
    half = 0.5 * c.dt[s]
    mx, my, mz = _relax(mx, my, mz, half, c)
    w = -TWO_PI * c.dt[s]
    wx, wy = w * c.rf[s, 0], w * c.rf[s, 1]
    if c.b1 is not None:
        wx, wy = wx * c.b1, wy * c.b1
    else:
        wx, wy = wx * torch.ones_like(bz), wy * torch.ones_like(bz)
    mx, my, mz = _rotate(mx, my, mz, wx, wy, w * bz)
    return _relax(mx, my, mz, half, c)


def _free_run(mx, my, mz, a, b, c, off):
    """Closed-form run of RF-free segments [a, b): samples at its ADC segments, state at its end."""
    dt = c.dt[a:b]
    t = torch.cumsum(dt, 0)
    k = torch.cumsum(c.grad[a:b] * dt[:, None], 0)
    extra = torch.cumsum(off[a:b] * dt, 0) if off is not None else torch.zeros_like(t)
    samples = []
    idx = [i for i in range(b - a) if c.adc[a + i]]
    if idx:
        ii = torch.tensor(idx)
        v = (mx + 1j * my)[:, None] * c.coils  # (N, C)
        n = mx.shape[0]
        block = max(1, _BLOCK // max(n, 1))
        for j in range(0, len(idx), block):
            sel = ii[j:j + block]
            cyc = c.pos @ k[sel].T + c.db0[:, None] * t[sel] + extra[sel]  # (N, n) cycles
            e = torch.exp(-t[sel][None, :] / c.t2[:, None] - 1j * TWO_PI * cyc)
            raw = v.T @ e  # (C, n)
            samples.append(raw * torch.exp(-1j * c.adc_phase[a + sel])[None, :])
    cyc = c.pos @ k[-1] + c.db0 * t[-1] + extra[-1]
    cs, sn = torch.cos(-TWO_PI * cyc), torch.sin(-TWO_PI * cyc)
    mx, my = cs * mx - sn * my, sn * mx + cs * my
    mx, my, mz = _relax(mx, my, mz, t[-1], c)
    return mx, my, mz, samples


def simulate(c: Case, merge: bool = True):
    """(signal (C, n_adc) complex128, m (N, 3) float64) of case ``c`` (module docstring)."""
    n = c.pd.shape[0]
    if c.m_init is None:
        mx, my, mz = torch.zeros(n, dtype=F64), torch.zeros(n, dtype=F64), c.pd
    else:
        mx, my, mz = c.m_init.unbind(-1)
    off = c.b0_offset
    cols = []
    for a, b in _steps(c.is_rf, c.spoil, merge):
        if c.is_rf[a]:
            mx, my, mz = _rf_step(mx, my, mz, a, c, off)
            if c.adc[a]:
                cols.append(_sample(mx, my, c.adc_phase[a], c)[:, None])
        else:
            mx, my, mz, samples = _free_run(mx, my, mz, a, b, c, off)
            cols += samples
        if c.spoil[b - 1]:
            mx, my = torch.zeros_like(mx), torch.zeros_like(my)
    n_coils = c.coils.shape[1]
    sig = torch.cat(cols, 1) if cols else torch.zeros(n_coils, 0, dtype=torch.complex128)
    return sig, torch.stack([mx, my, mz], -1)


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
