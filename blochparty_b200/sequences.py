"""Sequence construction: a small segment builder and the Cartesian GRE / multi-slice TSE families.

The builder follows blochparty's segment conventions (``sequences/builder.py:366-570``): a hard pulse is
``n_steps`` equal RF segments, ``readout(n, dwell)`` is a half-dwell segment, ``n - 1`` dwell segments and a
closing half-dwell segment, with the ``n`` samples at the ends of the first ``n`` of them (samples at
(i + 0.5) dwell, blochparty ``builder.py:458-468``), and ``spoil`` marks the last segment. Gradients switch
instantly (no ramps): every segment is piecewise constant either way, and ramps only add free segments.

The library functions build the workloads this package is measured on (``configs``): spoiled Cartesian GRE
in 2D and 3D with hard or windowed-sinc (slab) pulses, RF spoiling by the quadratic phase increment
(blochparty ``library.py:285-287``), per-TR flip trains, several echoes per TR, and a multi-slice TSE with
sinc excitation and refocusing pulses.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from .types import Sequence

F64 = torch.float64


class SequenceBuilder:
    """Appends segments; ``build()`` returns a float64 ``Sequence`` (all arithmetic in float64 numpy)."""

    def __init__(self):
        self._dt, self._rf, self._g, self._ph = [], [], [], []
        self._is_rf, self._adc, self._spoil = [], [], []
        self.time = 0.0

    def _append(self, dt, rf, g, ph, is_rf, adc):
        dt = np.atleast_1d(np.asarray(dt, dtype=np.float64))
        n = dt.shape[0]
        self._dt.append(dt)
        self._rf.append(np.broadcast_to(np.asarray(rf, dtype=np.float64), (n, 2)))
        self._g.append(np.broadcast_to(np.asarray(g, dtype=np.float64), (n, 3)))
        self._ph.append(np.broadcast_to(np.asarray(ph, dtype=np.float64), (n,)))
        self._is_rf += [is_rf] * n
        self._adc += adc if isinstance(adc, list) else [adc] * n
        self._spoil += [False] * n
        self.time += float(dt.sum())
        return self

    def rf(self, duration, *, flip_deg=None, amplitude=None, phase=0.0, grad=(0.0, 0.0, 0.0), n_steps=1):
        """Hard pulse of ``flip_deg`` (amplitude flip / 360 / duration [Hz]) or ``amplitude``, ``n_steps`` segments."""
        amp = flip_deg / 360.0 / duration if flip_deg is not None else amplitude
        rf = (amp * math.cos(phase), amp * math.sin(phase))
        return self._append(np.full(n_steps, duration / n_steps), rf, grad, 0.0, True, False)

    def rf_waveform(self, samples, dt, grad=(0.0, 0.0, 0.0)):
        """Shaped RF: ``samples`` (k, 2) [Hz], one segment of ``dt`` each."""
        samples = np.asarray(samples, dtype=np.float64)
        return self._append(np.full(samples.shape[0], dt), samples, grad, 0.0, True, False)

    def delay(self, duration, grad=(0.0, 0.0, 0.0)):
        if duration <= 0:
            return self
        return self._append([duration], (0.0, 0.0), grad, 0.0, False, False)

    def readout(self, n, dwell, grad=(0.0, 0.0, 0.0), phase=0.0):
        dt = np.concatenate([[0.5 * dwell], np.full(n - 1, dwell), [0.5 * dwell]])
        return self._append(dt, (0.0, 0.0), grad, phase, False, [True] * n + [False])

    def spoil(self):
        self._spoil[-1] = True
        return self

    def build(self, **meta) -> Sequence:
        cat = lambda xs: torch.from_numpy(np.ascontiguousarray(np.concatenate(xs))).to(F64)
        return Sequence(
            dt=cat(self._dt),
            rf=cat(self._rf),
            grad=cat(self._g),
            adc_phase=cat(self._ph),
            is_rf=list(self._is_rf),
            adc=list(self._adc),
            spoil=list(self._spoil),
            meta=meta,
        )


def sinc_pulse(flip_deg, duration, n_steps, *, slice_thickness, time_bw_product=4.0, apodization=0.5,
               slice_offset=0.0, phase=0.0):
    """Windowed-sinc slice-selective pulse sampled at the centres of ``n_steps`` equal steps.

    Envelope ((1 - a) + a cos(2 pi t / T)) sinc(BW t) on |t| < T/2, BW = time_bw_product / T, scaled to unit
    area so that the on-resonance flip is ``flip_deg``; slice-select gradient G = BW / slice_thickness on z.
    A slice at ``slice_offset`` z0 is reached by the frequency shift f = G z0 (phase -2 pi f t).
    Returns (samples (n_steps, 2) [Hz], dt, gz [Hz/m], rephase moment [cycles/m] on z).
    """
    dt = duration / n_steps
    t = (np.arange(n_steps) + 0.5) * dt - 0.5 * duration
    bw = time_bw_product / duration
    env = ((1.0 - apodization) + apodization * np.cos(2 * np.pi * t / duration)) * np.sinc(bw * t)
    env = env / (env.sum() * dt)
    amp = flip_deg / 360.0 * env
    gz = bw / slice_thickness
    ph = phase - 2 * np.pi * gz * slice_offset * t
    samples = np.stack([amp * np.cos(ph), amp * np.sin(ph)], -1)
    return samples, dt, gz, -gz * 0.5 * duration


def rf_spoil_phase(j: int, increment_deg: float = 117.0) -> float:
    """Quadratic RF-spoiling phase of the j-th excitation [rad]: increment * j (j + 1) / 2, wrapped in degrees."""
    return math.radians((increment_deg * j * (j + 1) / 2) % 360.0)


def gre(shape, fov, *, flip_deg=15.0, tr=10e-3, te=5e-3, n_dummy=0, dwell=10e-6, rf="hard",
        rf_duration=100e-6, rf_steps=1, slab_thickness=None, time_bw_product=4.0, spoiling="rf",
        spoiler_cycles=2.0, n_echoes=1, echo_spacing=None, t_pre=None) -> Sequence:
    """Cartesian spoiled gradient echo, 2D (``shape = (ny, nx)``) or 3D (``(nz, ny, nx)``).

    Per TR: excitation (hard pulse of ``rf_steps`` segments, or a windowed-sinc slab pulse of ``rf_steps`` steps
    with slab-select gradient and its rephaser folded into the prephaser), a prephaser to the line's
    (kx_min, ky, kz) in ``t_pre``, ``n_echoes`` readouts of ``nx`` samples (monopolar: a flyback lobe between
    echoes), a spoiler of ``spoiler_cycles`` cycles per voxel on x with the phase-encode rewinders, and a fill
    delay to ``tr``. ``flip_deg`` is a scalar or one flip per TR (dummies first). RF spoiling
    (``spoiling="rf"``) sets pulse and receiver phase to ``rf_spoil_phase(j)``; ``"none"`` keeps them at zero.
    The first echo's k-space centre is at ``te`` after the pulse centre.
    """
    *pe_shape, nx = shape
    dk = 1.0 / fov
    lines = []
    if len(pe_shape) == 1:
        for iy in range(pe_shape[0]):
            lines.append(((iy - pe_shape[0] // 2) * dk, 0.0))
    else:
        nz, ny = pe_shape
        for iz in range(nz):
            for iy in range(ny):
                lines.append(((iy - ny // 2) * dk, (iz - nz // 2) * dk))
    n_tr = n_dummy + len(lines)
    flips = np.broadcast_to(np.asarray(flip_deg, dtype=np.float64), (n_tr,))
    g_ro = dk / dwell  # [Hz/m]: one k-space step per dwell
    ro_len = nx * dwell
    k_start = -(nx // 2) * dk - 0.5 * dk  # moment at the readout start (first sample half a dwell in)
    if rf == "sinc" and slab_thickness is None:
        raise ValueError("rf='sinc' needs slab_thickness")
    rf_post = 0.5 * rf_duration
    t_k0 = (nx // 2 + 0.5) * dwell  # readout start to the sample at k = 0
    if t_pre is None:
        t_pre = te - rf_post - t_k0
    if t_pre <= 0:
        raise ValueError(f"TE too short: prephaser would last {t_pre * 1e3:.3f} ms")
    esp = echo_spacing if echo_spacing is not None else 2 * ro_len
    t_fly = esp - ro_len
    spoil_x = spoiler_cycles * nx / fov
    t_spoil = 0.5e-3
    used = rf_duration + t_pre + ro_len + (n_echoes - 1) * esp + t_spoil
    t_fill = tr - used
    if t_fill < -1e-12:
        raise ValueError(f"TR too short by {-t_fill * 1e3:.3f} ms")
    b = SequenceBuilder()
    for j in range(n_tr):
        acquire = j >= n_dummy
        ky, kz = lines[j - n_dummy] if acquire else (0.0, 0.0)
        psi = rf_spoil_phase(j) if spoiling == "rf" else 0.0
        reph_z = 0.0
        if rf == "sinc":
            samples, sdt, gz, reph_z = sinc_pulse(flips[j], rf_duration, rf_steps, slice_thickness=slab_thickness,
                                                  time_bw_product=time_bw_product, phase=psi)
            b.rf_waveform(samples, sdt, grad=(0.0, 0.0, gz))
        else:
            b.rf(rf_duration, flip_deg=float(flips[j]), phase=psi, n_steps=rf_steps)
        b.delay(t_pre, grad=(k_start / t_pre, ky / t_pre, (kz + reph_z) / t_pre))
        for e in range(n_echoes):
            if e > 0:  # flyback to the readout start
                b.delay(t_fly, grad=(-(ro_len * g_ro) / t_fly, 0.0, 0.0))
            b.readout(nx, dwell, grad=(g_ro, 0.0, 0.0), phase=psi if acquire else 0.0)
            if not acquire:  # dummies: the same gradients, no samples
                b._adc[-(nx + 1):] = [False] * (nx + 1)
        k_end_x = k_start + ro_len * g_ro
        b.delay(t_spoil, grad=((spoil_x - k_end_x) / t_spoil, -ky / t_spoil, -kz / t_spoil))
        b.delay(t_fill)
    return b.build(kspace_shape=tuple(shape), fov=fov, tr=tr, te=te, n_echoes=n_echoes, dwell=dwell,
                   n_tr=n_tr, n_dummy=n_dummy, rf=rf, slab_thickness=slab_thickness)


def tse_2d(n, fov, *, slices=(0.0,), slice_thickness=5e-3, etl=16, esp=12e-3, tr=3.0, dwell=10e-6,
           rf_duration=3e-3, rf_steps=300, time_bw_product=4.0, excite_flip_deg=90.0, refocus_flip_deg=180.0,
           n_shots=None) -> Sequence:
    """Multi-slice 2D turbo spin echo with windowed-sinc pulses.

    Per shot and slice: a 90-degree excitation (phase 0, x) with its slice rephaser and the readout prephaser,
    then ``etl`` refocusing pulses (phase pi/2, y: CPMG) each between crushers, a phase encode, a readout of ``n``
    samples centred between two refocusing pulses, and a rewinder. Slices are reached by frequency offset and
    interleaved within a TR; ``n_shots`` (default n / etl) shots cover the ``n`` phase encodes in sequential order.
    """
    dk = 1.0 / fov
    shots = n_shots if n_shots is not None else n // etl
    g_ro = dk / dwell
    ro_len = n * dwell
    crush = 4.0 / slice_thickness  # crusher moment [cycles/m] on z
    b = SequenceBuilder()
    t_start = 0.0
    for shot in range(shots):
        for sl, z0 in enumerate(slices):
            t0 = b.time
            exc, sdt, gz, reph = sinc_pulse(excite_flip_deg, rf_duration, rf_steps, slice_thickness=slice_thickness,
                                            time_bw_product=time_bw_product, slice_offset=z0)
            ref, _, _, _ = sinc_pulse(refocus_flip_deg, rf_duration, rf_steps, slice_thickness=slice_thickness,
                                      time_bw_product=time_bw_product, slice_offset=z0, phase=0.5 * math.pi)
            b.rf_waveform(exc, sdt, grad=(0.0, 0.0, gz))
            # excitation centre to first refocusing centre: esp / 2
            gap = 0.5 * esp - rf_duration
            pre_x = -(n // 2) * dk  # readout start moment; every refocusing pulse negates the readout's n dk to it
            b.delay(gap, grad=(-pre_x / gap, 0.0, reph / gap))
            for e in range(etl):
                line = shot * etl + e
                ky = (line - n // 2) * dk
                b.rf_waveform(ref, sdt, grad=(0.0, 0.0, gz))
                # crusher + phase encode, readout, rewinder + crusher: esp - rf_duration in total
                t_side = 0.5 * (esp - rf_duration - ro_len)
                b.delay(t_side, grad=(0.0, ky / t_side, crush / t_side))
                b.readout(n, dwell, grad=(g_ro, 0.0, 0.0))
                b.delay(t_side, grad=(0.0, -ky / t_side, crush / t_side))
            b.spoil()
            t_used = b.time - t0
            b.delay(tr / len(slices) - t_used)
    return b.build(kspace_shape=(n, n), fov=fov, tr=tr, esp=esp, etl=etl, slices=tuple(slices))
