"""The five measured workloads, built from seeded synthetic inputs (no dataset is needed or read).

Each function returns ``(phantom, seq, coils)`` (plus extras where stated) as float64 CPU objects:

* ``gre2d_64``: 64 x 64 ellipse phantom (10 ellipses, PD in [0, 1], T1 in [0.5, 2] s, T2 in [0.05, 0.15] s,
  4096 spins, FOV 0.25 m), 8 birdcage coils; spoiled 2D GRE 64 x 64, hard 15-degree pulse, TR 10 ms, TE 5 ms,
  200 dummy TRs, RF spoiling with the 117-degree quadratic phase.
* ``gre3d_64``: 64^3 ellipsoids with 4 sub-voxel spins at uniform random offsets (1,048,576 spins), B0 from
  Gaussian-smoothed noise (sigma 4 voxels) scaled to +-100 Hz, 8 coils; spoiled 3D GRE 64 x 64 phase encodes x
  64 samples, slab-selective windowed sinc (time-bandwidth 4, 2 ms, 200 steps of 10 us), flip 10 degrees, TR 8 ms.
* ``adjoint_2d_128``: 128 x 128 ellipse phantom, 8 coils, 128 per-TR flips drawn uniformly in [5, 30] degrees
  (seed 3), a radial B1+ in [0.8, 1.2]; hard 20 us pulses, TR 10 ms, TE 5 ms; extras: the flips and the target
  T1 map (T1 (1 + 0.05 N(0, 1)), seed 4).
* ``tse_3slice_128``: 3 contiguous 5 mm slices of 128 x 128 with 8 spins per voxel spread through the slice thickness (393,216
  spins); multi-slice TSE, 90 / 180 windowed sincs (time-bandwidth 4, 3 ms, 300 steps), ETL 16, ESP 12 ms,
  TR 3 s.
* ``gre3d_128_4echo``: 128^3 head-like phantom (fat, WM, GM, CSF), 4 spins per voxel (8,388,608 spins), B0 smooth
  +-150 Hz, 8 coils; 4-echo 3D GRE, TR 20 ms, 128 x 128 phase encodes x 128 samples, 200-step sinc slab pulses.
"""

from __future__ import annotations

import numpy as np
import torch

from . import phantoms, sequences
from .types import Phantom, Sequence

F64 = torch.float64


def gre2d_64():
    ph = phantoms.ellipse_phantom_2d(64, 0.25, n_ellipses=10, seed=0)
    seq = sequences.gre((64, 64), 0.25, flip_deg=15.0, tr=10e-3, te=5e-3, n_dummy=200, dwell=10e-6,
                        rf_duration=100e-6, rf_steps=1, spoiling="rf")
    return ph, seq, phantoms.birdcage_sensitivities(ph.pos, 8)


def gre3d_64(n=64):
    ph = phantoms.ellipsoid_phantom_3d(n, 0.25, n_ellipsoids=10, spins_per_voxel=4, seed=0, subvoxel_seed=1,
                                       b0_seed=2, b0_max=100.0, sigma_vox=4.0)
    seq = sequences.gre((n, n, n), 0.25, flip_deg=10.0, tr=8e-3, te=3e-3, dwell=10e-6, rf="sinc",
                        rf_duration=2e-3, rf_steps=200, slab_thickness=0.2, time_bw_product=4.0, spoiling="rf")
    return ph, seq, phantoms.birdcage_sensitivities(ph.pos, 8)


def adjoint_2d_128_sequence(flips, n=128):
    """The 2D GRE of ``adjoint_2d_128`` with the per-TR flip train ``flips`` [deg] (n values)."""
    return sequences.gre((n, n), 0.25, flip_deg=np.asarray(flips, dtype=np.float64), tr=10e-3, te=5e-3, dwell=10e-6,
                         rf_duration=20e-6, rf_steps=1, spoiling="rf")


def adjoint_2d_128(n=128):
    ph = phantoms.ellipse_phantom_2d(n, 0.25, n_ellipses=10, seed=0)
    ph.b1 = phantoms.radial_b1(ph.pos, 0.8, 1.2)
    g = torch.Generator().manual_seed(3)
    flips = 5.0 + 25.0 * torch.rand(n, generator=g, dtype=F64)
    seq = adjoint_2d_128_sequence(flips.numpy(), n)
    g4 = torch.Generator().manual_seed(4)
    t1_target = ph.t1 * (1.0 + 0.05 * torch.randn(ph.t1.shape, generator=g4, dtype=F64))
    return ph, seq, phantoms.birdcage_sensitivities(ph.pos, 8), flips, t1_target


def tse_3slice_128(n=128, slice_thickness=5e-3, slice_gap=5e-3, spins_per_voxel=8):
    slices = (-slice_gap, 0.0, slice_gap)
    base = phantoms.ellipse_phantom_2d(n, 0.25, n_ellipses=10, seed=0)
    z_off = (torch.arange(spins_per_voxel, dtype=F64) + 0.5) / spins_per_voxel - 0.5
    pos, rep = [], lambda t: t.repeat_interleave(spins_per_voxel).repeat(len(slices))
    for z0 in slices:
        p = base.pos.repeat_interleave(spins_per_voxel, 0).clone()
        p[:, 2] = z0 + z_off.repeat(base.pos.shape[0]) * slice_thickness
        pos.append(p)
    ph = Phantom(torch.cat(pos), rep(base.pd), rep(base.t1), rep(base.t2), rep(base.db0))
    seq = sequences.tse_2d(n, 0.25, slices=slices, slice_thickness=slice_thickness, etl=16, esp=12e-3, tr=3.0,
                           rf_duration=3e-3, rf_steps=300)
    return ph, seq, phantoms.birdcage_sensitivities(ph.pos, 8)


def gre3d_128_4echo(n=128):
    ph = phantoms.head_phantom_3d(n, 0.25, spins_per_voxel=4, b0_max=150.0)
    seq = sequences.gre((n, n, n), 0.25, flip_deg=15.0, tr=20e-3, te=3.5e-3, dwell=10e-6, rf="sinc",
                        rf_duration=2e-3, rf_steps=200, slab_thickness=0.2, n_echoes=4, echo_spacing=2.6e-3,
                        spoiling="rf")
    return ph, seq, phantoms.birdcage_sensitivities(ph.pos, 8)


def first_trs(seq, max_segments: int):
    """The sequence's first segments, up to the last RF pulse that starts at or before ``max_segments`` (whole TRs
    of a TR-periodic sequence): a bounded sample of a long workload with its per-TR structure."""
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    starts = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    cut = int(starts[starts <= max_segments].max()) if (starts <= max_segments).any() else len(seq)
    if cut == 0:
        cut = len(seq)
    sl = slice(0, cut)
    return Sequence(seq.dt[sl], seq.rf[sl], seq.grad[sl], seq.adc_phase[sl], list(seq.is_rf[:cut]),
                    list(seq.adc[:cut]), list(seq.spoil[:cut]), dict(seq.meta, first_segments=cut),
                    None if seq.b0_offset is None else seq.b0_offset[sl])


def first_n_trs(seq, n_tr: int):
    """The sequence's first ``n_tr`` TRs (cut at the start of the pulse that begins TR ``n_tr``; the whole sequence
    if it has no more TRs): a bounded sample of a TR-periodic workload with the same work per segment."""
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    starts = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    if n_tr >= len(starts) or n_tr < 1:
        return seq
    cut = int(starts[n_tr])
    sl = slice(0, cut)
    return Sequence(seq.dt[sl], seq.rf[sl], seq.grad[sl], seq.adc_phase[sl], list(seq.is_rf[:cut]),
                    list(seq.adc[:cut]), list(seq.spoil[:cut]), dict(seq.meta, n_tr=n_tr, first_segments=cut),
                    None if seq.b0_offset is None else seq.b0_offset[sl])
