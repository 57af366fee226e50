"""CPU float64 oracles of the learned RF surrogate — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` may import this module, as the checker.
The reference (blochparty) has no learned surrogate: its closest parts are the exact per-spin maps of reused
pulses (``engines/gpu/cuda/pulse.cu.in:3-32``, ``engines/gpu/driver.py:112-164``). What this oracle restates is
the plain integrator's rotation part (blochparty ``engines/core.py:97-108``: a rotation by
w = -2 pi dt (b1 rf_x, b1 rf_y, G z + df) per RF segment), composed over a pulse as unit quaternions, and the
surrogate's network in float64 with autograd (to check the hand-written training kernels' gradients), and the
map the inference kernels apply to one pulse occurrence (``pulse_map``).

Conventions (shared with ``blochparty_b200/csrc/surrogate.cu``):

* a rotation by angle |w| about w/|w| is the unit quaternion (cos |w|/2, sin |w|/2 w/|w|); applying q1 then q2
  is the Hamilton product q2 q1; the Cayley-Klein pair of q = (q0, q1, q2, q3) is alpha = q0 - i q3,
  beta = -i (q1 + i q2);
* the pulse's whole precession without RF is the z rotation by wz = -2 pi (G z + df) T; the network learns
  the reduced rotation R~ with R = Rz(wz / 2) R~ Rz(wz / 2), smooth in z where R itself winds around z;
* the pulse acts on a spin through its off-resonance in the slice gradient f = df + G (z - z0) and its B1 scale
  alone: the network's inputs are (f^, b^) = (f / F, (b1 - 1) / dom_b1) with F the largest |f| of the training
  domain, and its first layer sees the 14 features f^, b^, sin(k pi f^), cos(k pi f^), k = 1..6;
* relaxation during the pulse, to first order in the rates: the plain integrator's pulse is the affine map
  m -> M m + v with M = R - r2 A - r1 B + O(r^2), v = r1 pd C + O(r^2); A + B = T R, so the network learns what
  the relax (T/2) / rotate / relax (T/2) splitting misses, dA = A - (T/2)(P R + R P) (P = diag(1, 1, 0)) and
  dC = C - (T/2)(R e_z + e_z), reduced like R (dA~ = Rz(-wz/2) dA Rz(-wz/2), dC~ = Rz(-wz/2) dC) and divided by
  T. The pulse is then m -> E (R - (r2 - r1) dA) (E m + c) + c + r1 pd dC, E and c the exact half-pulse relaxation.
"""

from __future__ import annotations

import math

import torch

F64 = torch.float64
TWO_PI = 2.0 * math.pi


def qmul(a, b):
    """Hamilton product of quaternion tensors (..., 4)."""
    a0, a1, a2, a3 = a.unbind(-1)
    b0, b1, b2, b3 = b.unbind(-1)
    return torch.stack([a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3,
                        a0 * b1 + a1 * b0 + a2 * b3 - a3 * b2,
                        a0 * b2 - a1 * b3 + a2 * b0 + a3 * b1,
                        a0 * b3 + a1 * b2 - a2 * b1 + a3 * b0], -1)


def quat_of_rotvec(w):
    """(..., 3) rotation vectors -> (..., 4) unit quaternions."""
    phi = torch.linalg.vector_norm(w, dim=-1, keepdim=True)
    half = 0.5 * phi
    s = torch.where(phi > 1e-300, torch.sin(half) / phi.clamp_min(1e-300), torch.full_like(phi, 0.5))
    return torch.cat([torch.cos(half), s * w], -1)


def qz(angle):
    """Quaternion of the z rotation by ``angle`` (tensor (...,))."""
    z = torch.zeros_like(angle)
    return torch.stack([torch.cos(0.5 * angle), z, z, torch.sin(0.5 * angle)], -1)


def rotmat(q):
    """(..., 3, 3) rotation matrices of unit quaternions."""
    s, x, y, z = q.unbind(-1)
    return torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - s * z), 2 * (x * z + s * y)], -1),
        torch.stack([2 * (x * y + s * z), 1 - 2 * (x * x + z * z), 2 * (y * z - s * x)], -1),
        torch.stack([2 * (x * z - s * y), 2 * (y * z + s * x), 1 - 2 * (x * x + y * y)], -1)], -2)


def pulse_quaternions(rf, dt, gz, z, df, b1):
    """Whole-pulse rotation q and reduced rotation q~ of every sample (z [m], df [Hz], b1), float64.
    ``rf`` (K, 2) [Hz] at steps of ``dt`` [s] under the slice gradient ``gz`` [Hz/m]."""
    rf = torch.as_tensor(rf, dtype=F64)
    z, df, b1 = (torch.as_tensor(t, dtype=F64) for t in (z, df, b1))
    q = torch.zeros(z.shape + (4,), dtype=F64)
    q[..., 0] = 1.0
    w = -TWO_PI * dt
    wz = w * (gz * z + df)
    for k in range(rf.shape[0]):
        wv = torch.stack([w * b1 * rf[k, 0], w * b1 * rf[k, 1], wz], -1)
        q = qmul(quat_of_rotvec(wv), q)
    total = wz * rf.shape[0]
    qr = qmul(qmul(qz(-0.5 * total), q), qz(-0.5 * total))
    return q, qr  # (the rotation alone; pulse_targets adds the first-order relaxation terms)


def pulse_targets(rf, dt, gz, z, df, b1):
    """(q (n, 4), targets (n, 16)): the whole-pulse rotation q and the network's targets of every sample, float64:
    the reduced rotation q~ (4), dA~ / T (9, row-major) and dC~ / T (3), from the discrete first-order expansion of
    the plain Strang steps (each step E(h) R_k E(h) with h = dt / 2)."""
    rf = torch.as_tensor(rf, dtype=F64)
    z, df, b1 = (torch.as_tensor(t, dtype=F64) for t in (z, df, b1))
    K, h = rf.shape[0], 0.5 * dt
    q = torch.zeros(z.shape + (4,), dtype=F64)
    q[..., 0] = 1.0
    R = torch.eye(3, dtype=F64).expand(z.shape + (3, 3)).clone()
    A = torch.zeros(z.shape + (3, 3), dtype=F64)
    C = torch.zeros(z.shape + (3,), dtype=F64)
    P = torch.diag(torch.tensor([1.0, 1.0, 0.0], dtype=F64))
    ez = torch.tensor([0.0, 0.0, 1.0], dtype=F64)
    w = -TWO_PI * dt
    wz = w * (gz * z + df)
    for k in range(K):
        qk = quat_of_rotvec(torch.stack([w * b1 * rf[k, 0], w * b1 * rf[k, 1], wz], -1))
        Rk = rotmat(qk)
        A = Rk @ A + h * (P @ Rk + Rk @ P) @ R
        C = (Rk @ C[..., None])[..., 0] + h * (Rk @ ez + ez)
        R = Rk @ R
        q = qmul(qk, q)
    T = K * dt
    dA = A - 0.5 * T * (P @ R + R @ P)
    dC = C - 0.5 * T * (R @ ez + ez)
    half = qz(-0.5 * wz * K)
    Rh = rotmat(half)
    qr = qmul(qmul(half, q), half)
    dAr = Rh @ dA @ Rh / T
    dCr = (Rh @ dC[..., None])[..., 0] / T
    return q, torch.cat([qr, dAr.reshape(z.shape + (9,)), dCr], -1)


def gelu(x):
    """GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) (Hendrycks and Gimpel)."""
    return 0.5 * x * (1.0 + torch.tanh(math.sqrt(2.0 / math.pi) * (x + 0.044715 * x ** 3)))


# parameter layout of the flat vector (as the kernels): W1 (64, 14), b1 (64), W2 (64, 64), b2, W3 (64, 64), b3,
# W4 (16, 64), b4 (16): 10,320 floats
SHAPES = ((64, 14), (64,), (64, 64), (64,), (64, 64), (64,), (16, 64), (16,))
FOURIER_ORDERS = 6
N_PARAMS = sum(math.prod(s) for s in SHAPES)


def unflatten(p):
    out, o = [], 0
    for s in SHAPES:
        k = math.prod(s)
        out.append(p[o:o + k].reshape(s))
        o += k
    return out


def features(x):
    """The first layer's features (B, 14) of inputs x (B, 2) = (f^, b^): f^, b^, then sin(k pi f^), cos(k pi f^) for
    k = 1..6 (the kernels' ``mlp_features``, which builds the higher orders by angle addition)."""
    f = x[:, :1]
    k = torch.arange(1, FOURIER_ORDERS + 1, dtype=x.dtype)
    a = math.pi * f * k
    sc = torch.stack([torch.sin(a), torch.cos(a)], -1).reshape(x.shape[0], 2 * FOURIER_ORDERS)
    return torch.cat([x, sc], -1)


def mlp(p, x):
    """Network output (B, 16) for inputs x (B, 2) = (f^, b^): the quaternion (normalised to unit length), then the
    12 correction outputs as they are."""
    w1, b1, w2, b2, w3, b3, w4, b4 = unflatten(p)
    h = gelu(features(x) @ w1.T + b1)
    h = gelu(h @ w2.T + b2)
    h = gelu(h @ w3.T + b3)
    y = h @ w4.T + b4
    return torch.cat([y[:, :4] / torch.linalg.vector_norm(y[:, :4], dim=-1, keepdim=True), y[:, 4:]], -1)


def loss_and_grad(p, x, target, vweight: float = 1.0, cweight: float = 1.0):
    """Mean over the batch of (q0 - t0)^2 + vweight |q_vec - t_vec|^2 + cweight |corrections - their targets|^2
    and its gradient w.r.t. the flat parameters (float64)."""
    p = p.detach().to(F64).clone().requires_grad_()
    w = torch.tensor([1.0, vweight, vweight, vweight] + [cweight] * 12, dtype=F64)
    loss = (w * (mlp(p, x.to(F64)) - target.to(F64)) ** 2).sum(-1).mean()
    (g,) = torch.autograd.grad(loss, [p])
    return float(loss), g


def _rz(a):
    c, s = torch.cos(a), torch.sin(a)
    z, o = torch.zeros_like(a), torch.ones_like(a)
    return torch.stack([torch.stack([c, -s, z], -1), torch.stack([s, c, z], -1), torch.stack([z, z, o], -1)], -2)


def pulse_map(t, T, half, phi0, r1, r2, pd, m, first_order=True):
    """The surrogate's map of one pulse occurrence in float64, as the inference kernels apply it
    (``apply_pulse_map`` in ``blochparty_b200/csrc/surrogate.cu``): targets (or network outputs) ``t`` (n, 16), the
    pulse's duration ``T``, ``half`` (n,) = -pi (G z + df) T (half the whole-pulse precession), the occurrence's RF
    phase ``phi0``, the spins' rates and PD, magnetisation ``m`` (n, 3) -> (n, 3). With a1 = half + phi0 and
    a2 = half - phi0: R = Rz(a1) R~ Rz(a2), dA = Rz(a1) dA~ Rz(a2), dC = Rz(a1) dC~; relax T/2, apply
    R - (r2 - r1) dA, relax T/2, add r1 pd dC (``first_order=False``: the splitting alone)."""
    q = t[:, :4] / torch.linalg.vector_norm(t[:, :4], dim=-1, keepdim=True)
    ra, rb = _rz(half + phi0), _rz(half - phi0)
    M = ra @ rotmat(q) @ rb
    if first_order:
        dA = ra @ (T * t[:, 4:13].reshape(-1, 3, 3)) @ rb
        M = M - ((r2 - r1) * 1.0)[:, None, None] * dA
    e2, e1 = torch.exp(-0.5 * T * r2), torch.exp(-0.5 * T * r1)
    E = lambda v: torch.stack([v[:, 0] * e2, v[:, 1] * e2, pd + (v[:, 2] - pd) * e1], -1)
    out = E((M @ E(m)[..., None])[..., 0])
    if first_order:
        out = out + (r1 * pd * T)[:, None] * (ra @ t[:, 13:16, None])[..., 0]
    return out
