"""Pulseq input: a ``.seq`` file (format 1.4) -> ``Sequence``, the on-disk sequence format that feeds the path.

Restates the conversion of blochparty ``sequences/pulseq/read.py:64-221`` (conventions in
``sequences/pulseq/__init__.py:1-36``) with a parser of its own: the reference reads files through pypulseq, a
dependency that this package does not have. The conversion, block by block:

* Every block is cut at all of its event boundaries: the RF raster steps (or the points of a time-shaped pulse),
  the RF centre, gradient corner points, every ADC sample time and the block end. Each ADC sample therefore ends
  a segment. Gradients are piecewise linear in Pulseq and every corner is a cut, so a segment's midpoint value is
  its exact average: the moments are exact at every segment end. Sloped gradient pieces are cut further at
  ``ramp_raster``; sloped or frequency-shifted RF pieces off the RF raster at ``rf_raster``; RF pieces in general
  at ``max_rf_step``.
* Units already match: RF in Hz, gradients in Hz/m, time in s.
* ``convention="physical"``: a pulse with frequency offset f excites the spins whose Larmor frequency is higher by
  f, so the field is the complex conjugate of the Pulseq waveform, rf_x + i rf_y = conj(signal exp(i phase(t)))
  with phase(t) = phase_offset + 2 pi f t from the shape's start; an ADC sample's receiver phase is
  -(phase_offset + 2 pi f t_i), t_i = (i + 1/2) dwell from the ADC's start. ``convention="mrzero"`` takes the
  phases as written (no conjugate, receiver phase +).

Format 1.4 details this reader follows (the published Pulseq specification):
* block durations in units of ``BlockDurationRaster``; RF and gradient delays and trapezoid times in us; ADC
  dwell in ns and delay in us;
* shapes compressed as run-length coded derivatives (two equal values followed by the count of further
  repetitions), decoded by a cumulative sum; stored plainly when the listed values number ``num_samples``;
* RF phase shapes in units of 2 pi; time shapes in units of the raster; time shape 0 = samples at the centres of
  the raster cells;
* an arbitrary gradient on the raster has its edge values implicit: the first is the last value of the previous
  block's gradient on the same axis (0 if none), and the next edges follow from each sample being the mean of
  its two edges (the reading pypulseq gives such files);
* the RF centre (a cut only): the middle of the samples at the peak magnitude.
Label and trigger extensions are ignored; other extensions raise ``NotImplementedError``.

Not pinned against the reference's reader (pypulseq is absent here): ``tests/test_pulseq_host.py`` checks the
conventions against closed forms through the float64 oracle, as blochparty's ``tests/sequences/test_pulseq.py``
does against its own engine.
"""

from __future__ import annotations

import math
import re
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from .types import Sequence

T_TOL = 1e-11      # [s] event times closer than this are one cut
MAX_RF_STEP = 20e-6  # [s] the longest RF piece
IGNORED_EXTENSIONS = {"LABELSET", "LABELINC", "TRIGGERS"}


def decompress_shape(values: np.ndarray, n: int) -> np.ndarray:
    """A Pulseq shape's samples from its listed values (see the module docstring)."""
    v = np.asarray(values, dtype=np.float64)
    if v.shape[0] == n:
        return v.copy()
    out, i = [], 0
    while i < v.shape[0]:
        if i + 2 < v.shape[0] and v[i] == v[i + 1]:
            reps = int(round(v[i + 2]))
            if reps < 0:
                raise ValueError(f"a negative repetition count ({reps}) in a compressed shape")
            out.extend([v[i]] * (reps + 2))
            i += 3
        else:
            out.append(v[i])
            i += 1
    if len(out) != n:
        raise ValueError(f"a compressed shape decodes to {len(out)} samples, not {n}")
    return np.cumsum(out)


@dataclass
class _File:
    version: tuple
    definitions: dict
    blocks: list       # rows of ints: id dur rf gx gy gz adc ext
    rf: dict           # id -> (amp, mag_id, phase_id, time_id, delay_us, freq, phase)
    grads: dict        # id -> (amp, shape_id, time_id, delay_us)
    traps: dict        # id -> (amp, rise_us, flat_us, fall_us, delay_us)
    adc: dict          # id -> (num, dwell_ns, delay_us, freq, phase)
    shapes: dict       # id -> samples
    extensions: dict   # id -> (type_id, ref, next_id); types: id -> name


def _read_sections(text: str) -> dict:
    sections, name = {}, None
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        m = re.fullmatch(r"\[(\w+)\]", line)
        if m:
            name = m.group(1).upper()
            sections.setdefault(name, [])
        elif name is not None:
            sections[name].append(line)
    return sections


def parse(text: str) -> _File:
    """The sections of a format-1.4 ``.seq`` file."""
    sec = _read_sections(text)
    ver = {k: int(v) for k, v in (line.split()[:2] for line in sec.get("VERSION", []))}
    version = (ver.get("major", 0), ver.get("minor", 0), ver.get("revision", 0))
    if version[:2] != (1, 4):
        raise NotImplementedError(f"Pulseq format {version[0]}.{version[1]}: this reader takes format 1.4 files")
    definitions = {}
    for line in sec.get("DEFINITIONS", []):
        key, *vals = line.split()
        nums = []
        for v in vals:
            try:
                nums.append(float(v))
            except ValueError:
                nums = None
                break
        definitions[key] = (nums[0] if len(nums) == 1 else nums) if nums else " ".join(vals)
    rows = lambda name, n: [line.split() for line in sec.get(name, []) if len(line.split()) >= n]
    blocks = [[int(x) for x in r[:8]] for r in rows("BLOCKS", 8)]
    rf = {int(r[0]): (float(r[1]), int(r[2]), int(r[3]), int(r[4]), float(r[5]), float(r[6]), float(r[7]))
          for r in rows("RF", 8)}
    grads = {int(r[0]): (float(r[1]), int(r[2]), int(r[3]), float(r[4])) for r in rows("GRADIENTS", 5)}
    traps = {int(r[0]): tuple(float(x) for x in r[1:6]) for r in rows("TRAP", 6)}
    adc = {int(r[0]): (int(r[1]), float(r[2]), float(r[3]), float(r[4]), float(r[5])) for r in rows("ADC", 6)}
    shapes, sid, n, vals = {}, None, 0, []

    def close():
        if sid is not None:
            shapes[sid] = decompress_shape(np.array(vals), n)

    for line in sec.get("SHAPES", []):
        parts = line.split()
        if parts[0] == "shape_id":
            close()
            sid, n, vals = int(parts[1]), 0, []
        elif parts[0] == "num_samples":
            n = int(parts[1])
        else:
            vals.extend(float(x) for x in parts)
    close()
    # the extension list (id type ref next) comes first; each "extension NAME type_id" line then opens that
    # extension's own table, which this reader does not need
    ext_types, ext_rows, in_list = {}, {}, True
    for line in sec.get("EXTENSIONS", []):
        parts = line.split()
        if parts[0] == "extension":
            ext_types[int(parts[2])] = parts[1].upper()
            in_list = False
        elif in_list and len(parts) == 4:
            ext_rows[int(parts[0])] = (int(parts[1]), int(parts[2]), int(parts[3]))
    return _File(version, definitions, blocks, rf, grads, traps, adc, shapes, {"rows": ext_rows, "types": ext_types})


def _subdivide(t: np.ndarray, sloped: np.ndarray, step: float) -> np.ndarray:
    """Extra cuts splitting each flagged interval of ``t`` into equal pieces of at most ``step``."""
    out = [np.zeros(0)]
    for a, b in zip(t[:-1][sloped], t[1:][sloped]):
        k = math.ceil((b - a) / step - 1e-9)
        if k > 1:
            out.append(a + (b - a) * np.arange(1, k) / k)
    return np.concatenate(out)


def _rf_center(t: np.ndarray, sig: np.ndarray) -> float:
    mag = np.abs(sig)
    peak = np.flatnonzero(mag >= mag.max() * (1 - 1e-5))
    return 0.5 * (t[peak[0]] + t[peak[-1]])


class _Reader:
    def __init__(self, f: _File, ramp_raster, rf_raster, max_rf_step, sign):
        d = f.definitions
        self.f, self.sign = f, sign
        self.grad_raster = float(d.get("GradientRasterTime", 1e-5))
        self.rf_raster_def = float(d.get("RadiofrequencyRasterTime", 1e-6))
        self.block_raster = float(d.get("BlockDurationRaster", 1e-5))
        self.ramp_raster = ramp_raster or self.grad_raster
        self.rf_raster = rf_raster or self.rf_raster_def
        self.max_rf_step = max_rf_step or MAX_RF_STEP
        self.last = [0.0, 0.0, 0.0]  # the last value of each axis's gradient in the block before

    def shape(self, sid: int) -> np.ndarray:
        if sid not in self.f.shapes:
            raise ValueError(f"shape {sid} is referenced but not defined")
        return self.f.shapes[sid]

    def gradient(self, axis: int, gid: int, trap: bool):
        """(times, values) of one block's gradient on ``axis`` as a piecewise-linear waveform from the block start."""
        if trap:
            amp, rise, flat, fall, delay = self.f.traps[gid]
            t = np.cumsum([0.0, rise, flat, fall]) * 1e-6
            v = amp * np.array([0.0, 1.0, 1.0, 0.0])
        else:
            amp, sid, tid, delay = self.f.grads[gid]
            w = amp * self.shape(sid)
            if tid == 0:  # samples at the raster cells' centres; edges from continuity and the cells' means
                edges = np.empty(w.shape[0] + 1)
                # a delayed waveform starts from the zero gradient of its delay, else from the previous block's end
                edges[0] = 0.0 if delay > 0 else self.last[axis]
                for i in range(w.shape[0]):
                    edges[i + 1] = 2.0 * w[i] - edges[i]
                t = np.concatenate([[0.0], (np.arange(w.shape[0]) + 0.5) * self.grad_raster,
                                    [w.shape[0] * self.grad_raster]])
                v = np.concatenate([[edges[0]], w, [edges[-1]]])
            else:  # an explicit time shape (an extended trapezoid)
                t, v = self.shape(tid) * self.grad_raster, w
        keep = np.concatenate([[True], np.diff(t) > T_TOL])
        return delay * 1e-6 + t[keep], v[keep]

    def block(self, row):
        """(dt, grad (n, 3), b1 (n,) complex, is_rf, is_adc, psi, n_adc) of one block."""
        _, dur_ticks, rf_id, gx, gy, gz, adc_id, ext_id = row
        self.check_extensions(ext_id)
        dur = dur_ticks * self.block_raster
        if dur <= 0:
            return None
        cuts = [np.array([0.0, dur])]
        shapes = [None, None, None]
        last = [0.0, 0.0, 0.0]
        for axis, gid in enumerate((gx, gy, gz)):
            if gid == 0:
                continue
            if gid not in self.f.traps and gid not in self.f.grads:
                raise ValueError(f"block {row[0]}: gradient {gid} is referenced but not defined")
            t, v = self.gradient(axis, gid, gid in self.f.traps)
            shapes[axis] = (t, v)
            last[axis] = float(v[-1])
            cuts.append(np.concatenate([t, _subdivide(t, np.diff(v) != 0, self.ramp_raster)]))
        self.last = last
        rf = None
        if rf_id:
            amp, mag_id, ph_id, tid, delay_us, freq, phase = self.f.rf[rf_id]
            sig = amp * self.shape(mag_id) * np.exp(2j * math.pi * self.shape(ph_id))
            on_raster = tid == 0
            t_rf = (np.arange(sig.shape[0]) + 0.5) * self.rf_raster_def if on_raster else self.shape(tid) * \
                self.rf_raster_def
            if on_raster:
                edges = np.arange(sig.shape[0] + 1) * self.rf_raster_def
            else:
                sloped = (np.diff(sig) != 0) | (freq != 0)
                edges = np.sort(np.concatenate([t_rf, _subdivide(t_rf, sloped, self.rf_raster)]))
                edges = np.concatenate([edges, _subdivide(edges, np.ones(edges.shape[0] - 1, dtype=bool),
                                                          self.max_rf_step)])
            delay = delay_us * 1e-6
            cuts += [delay + edges, np.array([delay + _rf_center(t_rf, sig)])]
            rf = (sig, t_rf, on_raster, delay, freq, phase, delay + edges.min(), delay + edges.max())
        t_adc = None
        if adc_id:
            num, dwell_ns, adc_delay_us, adc_freq, adc_phase = self.f.adc[adc_id]
            dwell, adc_delay = dwell_ns * 1e-9, adc_delay_us * 1e-6
            t_adc = adc_delay + (np.arange(num) + 0.5) * dwell
            cuts.append(t_adc)
        t = np.sort(np.concatenate(cuts))
        t = t[np.concatenate([[True], np.diff(t) > T_TOL])]
        if t[-1] > dur + T_TOL:
            raise ValueError(f"block {row[0]}: its events last {t[-1]:.9g} s, longer than the block ({dur:.9g} s)")
        t = np.append(t[t < dur - T_TOL], dur)
        if t[0] > T_TOL:
            t = np.concatenate([[0.0], t])
        mid, n = 0.5 * (t[1:] + t[:-1]), t.shape[0] - 1
        g = np.zeros((n, 3))
        for axis, sh in enumerate(shapes):
            if sh is not None:
                g[:, axis] = np.interp(mid, sh[0], sh[1], left=0.0, right=0.0)
        b1 = np.zeros(n, dtype=complex)
        is_rf = np.zeros(n, dtype=bool)
        if rf is not None:
            sig, t_rf, on_raster, delay, freq, phase, lo, hi = rf
            is_rf = (mid > lo) & (mid < hi)
            tr = mid[is_rf] - delay
            if on_raster:
                k = np.clip(np.floor(tr / self.rf_raster_def).astype(int), 0, sig.shape[0] - 1)
                ts, vals = t_rf[k], sig[k]
            else:
                ts = tr
                vals = np.interp(tr, t_rf, sig.real) + 1j * np.interp(tr, t_rf, sig.imag)
            b1[is_rf] = vals * np.exp(1j * (phase + 2 * math.pi * freq * ts))
        if self.sign < 0:
            b1 = b1.conj()
        is_adc = np.zeros(n, dtype=bool)
        psi = np.zeros(n)
        n_adc = 0
        if t_adc is not None:
            ends = np.searchsorted(t, t_adc - T_TOL)
            if not np.all(np.abs(t[ends] - t_adc) <= T_TOL):
                raise ValueError(f"block {row[0]}: an ADC sample does not fall on a cut")
            is_adc[ends - 1] = True
            psi[ends - 1] = self.sign * (adc_phase + 2 * math.pi * adc_freq * (t_adc - adc_delay))
            n_adc = t_adc.shape[0]
        return np.diff(t), g, b1, is_rf, is_adc, psi, n_adc

    def check_extensions(self, ext_id: int) -> None:
        seen = 0
        while ext_id:
            if ext_id not in self.f.extensions["rows"] or seen > 10000:
                raise ValueError(f"extension {ext_id} is referenced but not defined")
            type_id, _, ext_id = self.f.extensions["rows"][ext_id]
            name = self.f.extensions["types"].get(type_id, f"type {type_id}")
            if name not in IGNORED_EXTENSIONS:
                raise NotImplementedError(f"unsupported Pulseq extension: {name}")
            seen += 1


def read_pulseq(seq_file, *, dtype=torch.float64, device=None, ramp_raster: float | None = None,
                rf_raster: float | None = None, max_rf_step: float | None = None, convention: str = "physical",
                **meta) -> Sequence:
    """A ``Sequence`` from a Pulseq format-1.4 file (a path, or the file's text), as blochparty's
    ``read_pulseq`` (``sequences/pulseq/read.py:64-221``) converts one: see the module docstring.

    ramp_raster: the longest piece a sloped gradient section is cut into (default: the gradient raster).
    rf_raster: the same for time-shaped RF pulses that vary or carry a frequency offset (default: the RF raster;
        pulses on the RF raster are always stepped sample by sample).
    max_rf_step: the longest piece of an RF pulse off the raster (default 20 us).
    convention: "physical" (default) or "mrzero".
    meta: extra entries for ``Sequence.meta``."""
    if convention not in ("physical", "mrzero"):
        raise ValueError(f"convention must be 'physical' or 'mrzero', not {convention!r}")
    text = seq_file
    if isinstance(seq_file, Path) or (isinstance(seq_file, str) and "\n" not in seq_file):
        text = Path(seq_file).read_text()
    f = parse(text)
    reader = _Reader(f, ramp_raster, rf_raster, max_rf_step, -1.0 if convention == "physical" else 1.0)
    parts, block_segments, adc_counts, n_seg = [], [], [], 0
    for row in f.blocks:
        out = reader.block(row)
        if out is None:
            block_segments.append((n_seg, n_seg))
            continue
        parts.append(out)
        n = out[0].shape[0]
        block_segments.append((n_seg, n_seg + n))
        n_seg += n
        if out[6]:
            adc_counts.append(out[6])
    if not parts:
        raise ValueError("the file holds no block with a duration")
    cat = lambda k: np.concatenate([p[k] for p in parts])
    b1 = cat(2)
    tensor = lambda x: torch.as_tensor(x, dtype=dtype, device=device)
    return Sequence(
        dt=tensor(cat(0)), rf=tensor(np.stack([b1.real, b1.imag], -1)), grad=tensor(cat(1)),
        adc_phase=tensor(cat(5)), is_rf=cat(3).tolist(), adc=cat(4).tolist(), spoil=[False] * n_seg,
        meta={"adc_per_readout": adc_counts, "block_segments": block_segments, "definitions": f.definitions,
              "convention": convention, **meta})
