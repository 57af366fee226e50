"""Seeded synthetic phantoms and analytic receive coils for the measured workloads.

Every phantom is built directly as a ``Phantom`` (one isochromat per voxel or several sub-voxel isochromats),
not through a map-to-phantom conversion, so a "4096-spin" phantom has exactly 4096 spins, background voxels
(PD 0) included. All randomness comes from ``torch.Generator().manual_seed(seed)``.
"""

from __future__ import annotations

import math

import torch

from .types import Phantom

F64 = torch.float64


def grid_positions(shape, fov: float) -> torch.Tensor:
    """(*shape, 3) voxel-centre positions [m] of a Cartesian grid with isotropic ``fov``; the last axis is x and
    index i along an axis of length n sits at (i - n/2) fov / n (the Cartesian k-space layout; blochparty
    ``phantom.py:54-70`` places voxels the same way). A 2D shape lies at z = 0."""
    axes = [(torch.arange(n, dtype=F64) - n // 2) * (fov / n) for n in shape]
    xyz = list(reversed(torch.meshgrid(*axes, indexing="ij")))
    if len(xyz) == 2:
        xyz.append(torch.zeros_like(xyz[0]))
    return torch.stack(xyz, dim=-1)


def _rand(g, *shape):
    return torch.rand(*shape, generator=g, dtype=F64)


def ellipse_phantom_2d(n=64, fov=0.25, n_ellipses=10, seed=0, pd_range=(0.0, 1.0), t1_range=(0.5, 2.0),
                       t2_range=(0.05, 0.15), background=(0.0, 1.0, 0.1)) -> Phantom:
    """n x n voxels, one spin each: ``n_ellipses`` random ellipses (later ones paint over earlier ones) with
    piecewise-constant PD, T1, T2 drawn uniformly from the ranges; ``background`` (pd, t1, t2) elsewhere."""
    g = torch.Generator().manual_seed(seed)
    pos = grid_positions((n, n), fov).reshape(-1, 3)
    x, y = pos[:, 0] / (0.5 * fov), pos[:, 1] / (0.5 * fov)
    pd = torch.full((n * n,), background[0], dtype=F64)
    t1 = torch.full((n * n,), background[1], dtype=F64)
    t2 = torch.full((n * n,), background[2], dtype=F64)
    for _ in range(n_ellipses):
        cx, cy = (_rand(g, 2) - 0.5) * 1.0
        a, b = 0.15 + 0.55 * _rand(g, 2)
        th = math.pi * float(_rand(g, 1))
        vals = _rand(g, 3)
        xr = (x - cx) * math.cos(th) + (y - cy) * math.sin(th)
        yr = -(x - cx) * math.sin(th) + (y - cy) * math.cos(th)
        inside = (xr / a) ** 2 + (yr / b) ** 2 <= 1.0
        pd[inside] = pd_range[0] + (pd_range[1] - pd_range[0]) * vals[0]
        t1[inside] = t1_range[0] + (t1_range[1] - t1_range[0]) * vals[1]
        t2[inside] = t2_range[0] + (t2_range[1] - t2_range[0]) * vals[2]
    return Phantom(pos, pd, t1, t2, torch.zeros(n * n, dtype=F64))


def _smooth_noise_3d(n, sigma_vox, seed, amplitude):
    """Gaussian-filtered N(0,1) noise on an n^3 grid (separable FFT-free convolution), scaled to +-amplitude."""
    g = torch.Generator().manual_seed(seed)
    v = torch.randn(n, n, n, generator=g, dtype=F64)
    r = int(math.ceil(3 * sigma_vox))
    k = torch.exp(-0.5 * (torch.arange(-r, r + 1, dtype=F64) / sigma_vox) ** 2)
    k = (k / k.sum()).reshape(1, 1, -1)
    for axis in range(3):
        v = v.movedim(axis, -1)
        shp = v.shape
        v = torch.nn.functional.conv1d(v.reshape(-1, 1, n), k, padding=r).reshape(shp)
        v = v.movedim(-1, axis)
    return v * (amplitude / v.abs().max())


def _subvoxel(pos_vox, fov, n, spins_per_voxel, seed):
    """Each voxel centre repeated ``spins_per_voxel`` times at uniform random offsets within the voxel."""
    g = torch.Generator().manual_seed(seed)
    nv = pos_vox.shape[0]
    off = (_rand(g, nv, spins_per_voxel, 3) - 0.5) * (fov / n)
    return (pos_vox[:, None, :] + off).reshape(-1, 3)


def ellipsoid_phantom_3d(n=64, fov=0.25, n_ellipsoids=10, spins_per_voxel=4, seed=0, subvoxel_seed=1,
                         b0_seed=2, b0_max=100.0, sigma_vox=4.0) -> Phantom:
    """n^3 voxels of random ellipsoids (tissue values as ``ellipse_phantom_2d``), ``spins_per_voxel`` spins per
    voxel at uniform offsets, and a smooth B0 map (Gaussian-filtered noise, sigma ``sigma_vox`` voxels, scaled to
    +-``b0_max`` Hz) shared by the spins of a voxel."""
    g = torch.Generator().manual_seed(seed)
    vox = grid_positions((n, n, n), fov).reshape(-1, 3)
    u = vox / (0.5 * fov)
    nv = vox.shape[0]
    pd, t1, t2 = torch.zeros(nv, dtype=F64), torch.ones(nv, dtype=F64), torch.full((nv,), 0.1, dtype=F64)
    for _ in range(n_ellipsoids):
        c = (_rand(g, 3) - 0.5) * 0.8
        ax = 0.15 + 0.5 * _rand(g, 3)
        vals = _rand(g, 3)
        inside = (((u - c) / ax) ** 2).sum(-1) <= 1.0
        pd[inside] = vals[0]
        t1[inside] = 0.5 + 1.5 * vals[1]
        t2[inside] = 0.05 + 0.1 * vals[2]
    db0 = _smooth_noise_3d(n, sigma_vox, b0_seed, b0_max).reshape(-1)
    s = spins_per_voxel
    rep = lambda t: t.repeat_interleave(s)
    return Phantom(_subvoxel(vox, fov, n, s, subvoxel_seed), rep(pd), rep(t1), rep(t2), rep(db0))


# tissue label -> (T1, T2) [s] for the head-like phantom: fat, white matter, grey matter, CSF
HEAD_TISSUES = {"fat": (0.3, 0.08), "wm": (0.8, 0.07), "gm": (1.3, 0.09), "csf": (4.0, 2.0)}


def head_phantom_3d(n=128, fov=0.25, spins_per_voxel=4, subvoxel_seed=1, b0_seed=2, b0_max=150.0,
                    sigma_vox=8.0) -> Phantom:
    """A head-like n^3 phantom of nested ellipsoids in four labels: a fat shell (scalp), grey matter, white matter,
    and CSF ventricles, with PD 0.9 / 0.8 / 0.7 / 1.0; ``spins_per_voxel`` spins per voxel; smooth B0 to
    +-``b0_max`` Hz."""
    vox = grid_positions((n, n, n), fov).reshape(-1, 3)
    u = vox / (0.5 * fov)
    nv = vox.shape[0]
    inside = lambda ax, c=(0.0, 0.0, 0.0): (((u - torch.tensor(c, dtype=F64)) / torch.tensor(ax, dtype=F64)) ** 2
                                            ).sum(-1) <= 1.0
    pd, t1, t2 = torch.zeros(nv, dtype=F64), torch.ones(nv, dtype=F64), torch.full((nv,), 0.1, dtype=F64)

    def paint(mask, label, p):
        pd[mask] = p
        t1[mask], t2[mask] = HEAD_TISSUES[label]

    paint(inside((0.72, 0.9, 0.8)), "fat", 0.9)
    paint(inside((0.66, 0.84, 0.74)), "gm", 0.8)
    paint(inside((0.55, 0.72, 0.6)), "wm", 0.7)
    paint(inside((0.12, 0.3, 0.2), (0.15, 0.0, 0.05)) | inside((0.12, 0.3, 0.2), (-0.15, 0.0, 0.05)), "csf", 1.0)
    paint(inside((0.1, 0.1, 0.12), (0.3, 0.35, -0.2)) | inside((0.1, 0.1, 0.12), (-0.3, 0.35, -0.2)), "gm", 0.8)
    db0 = _smooth_noise_3d(n, sigma_vox, b0_seed, b0_max).reshape(-1)
    s = spins_per_voxel
    rep = lambda t: t.repeat_interleave(s)
    return Phantom(_subvoxel(vox, fov, n, s, subvoxel_seed), rep(pd), rep(t1), rep(t2), rep(db0))


def birdcage_sensitivities(pos: torch.Tensor, n_coils: int = 8, radius: float = 0.18) -> torch.Tensor:
    """(N, C) complex receive sensitivities of ``n_coils`` elements evenly spaced on a circle of ``radius`` around
    the z axis: magnitude radius / distance to the element (clamped at 5 % of the radius), phase the in-plane
    angle of the spin as seen from the element, relative to the element's own angle; the same analytic model as
    blochparty ``coils.py:12-43`` (its default options), so cases carry over unchanged."""
    theta = 2 * math.pi * torch.arange(n_coils, dtype=pos.dtype) / n_coils
    dx = pos[:, :1] - radius * torch.cos(theta)
    dy = pos[:, 1:2] - radius * torch.sin(theta)
    dist = torch.sqrt(dx * dx + dy * dy).clamp_min(0.05 * radius)
    return torch.polar(radius / dist, torch.atan2(dy, dx) - theta)


def radial_b1(pos: torch.Tensor, lo=0.8, hi=1.2) -> torch.Tensor:
    """A smooth radial transmit scale: ``hi`` on the z axis falling linearly in the in-plane radius to ``lo`` at the
    largest radius of ``pos``."""
    rho = torch.sqrt(pos[:, 0] ** 2 + pos[:, 1] ** 2)
    return hi - (hi - lo) * rho / rho.max().clamp_min(1e-30)
