"""Pulseq input (``blochparty_b200.pulseq``) on the CPU: format-1.4 files written here, read into a ``Sequence`` and
simulated by the float64 oracle, against closed forms (as blochparty ``tests/sequences/test_pulseq.py`` checks its
reader against its own engine): the flip and phase conventions, the slice a frequency-shifted pulse excites, ADC
timing and receiver phases, gradient moments, the shape compression, and the refusals."""

import math

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import pulseq
from oracle import bloch

F64 = torch.float64


def seq_text(blocks, rf=(), traps=(), grads=(), adc=(), shapes=(), defs=None, version=(1, 4, 1), extensions=""):
    """A format-1.4 file from rows: blocks (id dur rf gx gy gz adc ext), rf (id amp mag phase time delay freq
    phase), traps (id amp rise flat fall delay), grads (id amp shape time delay), adc (id num dwell delay freq
    phase), shapes [(id, num_samples, listed values)]."""
    d = {"GradientRasterTime": 1e-5, "RadiofrequencyRasterTime": 1e-6, "AdcRasterTime": 1e-7,
         "BlockDurationRaster": 1e-5}
    d.update(defs or {})
    out = ["# Pulseq sequence file", "[VERSION]", f"major {version[0]}", f"minor {version[1]}",
           f"revision {version[2]}", "", "[DEFINITIONS]"] + [f"{k} {v}" for k, v in d.items()] + ["", "[BLOCKS]"]
    out += [" ".join(str(x) for x in b) for b in blocks]
    for name, rows in (("RF", rf), ("TRAP", traps), ("GRADIENTS", grads), ("ADC", adc)):
        if rows:
            out += ["", f"[{name}]"] + [" ".join(str(x) for x in r) for r in rows]
    if extensions:
        out += ["", extensions]
    if shapes:
        out += ["", "[SHAPES]"]
        for sid, n, vals in shapes:
            out += ["", f"shape_id {sid}", f"num_samples {n}"] + [repr(float(v)) for v in vals]
    return "\n".join(out) + "\n"


def spins(z=(0.0,), t1=1e9, t2=1e9):
    n = len(z)
    pos = torch.zeros(n, 3, dtype=F64)
    pos[:, 2] = torch.tensor(z, dtype=F64)
    f = lambda v: torch.full((n,), float(v), dtype=F64)
    return bpb.Phantom(pos, f(1.0), f(t1), f(t2), f(0.0))


def final_m(seq, ph):
    return bloch.simulate(bloch.case_from(ph, seq, torch.ones(len(ph.pd), 1, dtype=torch.complex128)))[1]


def hard_pulse(phase, flip=90.0, n=100):
    """A block pulse of n 1-us samples (constant magnitude shape, compressed) with the given phase offset."""
    amp = flip / 360.0 / (n * 1e-6)
    return seq_text([[1, n // 10, 1, 0, 0, 0, 0, 0]], rf=[[1, amp, 1, 2, 0, 0, 0, phase]],
                    shapes=[(1, n, [1.0, 0.0, 0.0, n - 3]), (2, n, [0.0, 0.0, n - 2])])


@pytest.mark.parametrize("phase", [0.0, 0.5 * math.pi, 1.0])
def test_hard_pulse_flip_and_phase_follow_the_physical_convention(phase):
    """A 90-degree pulse with Pulseq phase phi leaves Mxy = i exp(-i phi) (a real pulse tips +z to +y)."""
    seq = pulseq.read_pulseq(hard_pulse(phase))
    assert len(seq) == 100 + 1 or len(seq) == 100  # the RF centre may add one cut inside a raster cell
    m = final_m(seq, spins())
    expect = 1j * np.exp(-1j * phase)
    assert abs(complex(m[0, 0], m[0, 1]) - expect) < 1e-9 and abs(float(m[0, 2])) < 1e-9


def test_mrzero_convention_turns_the_other_way():
    seq = pulseq.read_pulseq(hard_pulse(0.5 * math.pi), convention="mrzero")
    m = final_m(seq, spins())
    assert abs(complex(m[0, 0], m[0, 1]) - 1j * np.exp(0.5j * math.pi)) < 1e-9


def test_sinc_pulse_with_a_frequency_offset_excites_the_slice_at_f_over_g():
    """A slice-selective sinc (200 samples of 10 us, time-bandwidth 8: a 4 kHz band, frequency offset f) under a
    trapezoid G along z turns the spin at z = f / G by its flip angle, and leaves the spins at -f / G and 0 (6 and
    12 kHz off the band's centre) untouched: a positive offset f excites spins precessing faster by f."""
    n, raster, G, f = 200, 1e-5, 4e5, 6000.0  # Hz/m, Hz: the slice at z = 15 mm
    x = (np.arange(n) + 0.5) / n * 2 - 1
    s = np.sinc(4 * x)
    mag, ph = np.abs(s) / np.abs(s).max(), np.where(s < 0, 0.5, 0.0)
    amp = 30.0 / 360.0 / (np.sum(s / np.abs(s).max()) * raster)  # 30 degrees on resonance
    text = seq_text([[1, 202, 1, 0, 0, 1, 0, 0]], rf=[[1, amp, 1, 2, 0, 10, f, 0]],
                    traps=[[1, G, 10, 2000, 10, 0]], shapes=[(1, n, mag), (2, n, ph)],
                    defs={"RadiofrequencyRasterTime": raster})
    seq = pulseq.read_pulseq(text)
    z0 = f / G
    m = final_m(seq, spins((z0, -z0, 0.0)))
    mxy = torch.sqrt(m[:, 0] ** 2 + m[:, 1] ** 2)
    # on the RF raster the field holds each sample's phase for a cell while the spin turns 2 pi f raster in it:
    # the cell's mean field shrinks by sinc(f raster), and the flip with it
    expect = math.sin(math.radians(30.0) * np.sinc(f * raster))
    assert abs(float(mxy[0]) - expect) < 1e-4 and float(mxy[1]) < 0.01 and float(mxy[2]) < 0.01


def test_adc_samples_end_segments_with_their_receiver_phases():
    num, dwell_ns, delay_us, freq, phase = 4, 10000, 20, 250.0, 0.3
    text = seq_text([[1, 8, 0, 0, 0, 0, 1, 0]], adc=[[1, num, dwell_ns, delay_us, freq, phase]])
    for convention, sign in (("physical", -1.0), ("mrzero", 1.0)):
        seq = pulseq.read_pulseq(text, convention=convention)
        ends = torch.cumsum(seq.dt, 0)
        idx = [i for i, a in enumerate(seq.adc) if a]
        t_i = 20e-6 + (np.arange(num) + 0.5) * 1e-5
        assert len(idx) == num and np.allclose(ends[idx].numpy(), t_i, atol=1e-12)
        assert np.allclose(seq.adc_phase[idx].numpy(), sign * (phase + 2 * math.pi * freq * (t_i - 20e-6)))
        assert abs(float(seq.duration) - 80e-6) < 1e-12 and seq.meta["adc_per_readout"] == [num]


def test_gradient_moments_are_exact_and_ramps_are_cut():
    """A trapezoid's moment is amp (flat + (rise + fall) / 2) to rounding, whatever the cuts; its ramps are cut into
    pieces no longer than ramp_raster; an extended trapezoid (explicit time shape) likewise."""
    amp = 1000.0
    text = seq_text([[1, 20, 0, 1, 0, 0, 0, 0], [2, 10, 0, 0, 2, 0, 0, 0]], traps=[[1, amp, 20, 100, 40, 10]],
                    grads=[[2, 500.0, 1, 2, 0]], shapes=[(1, 3, [0.0, 1.0, 0.0]), (2, 3, [0.0, 3.0, 10.0])])
    for ramp in (None, 5e-6):
        seq = pulseq.read_pulseq(text, ramp_raster=ramp)
        bs = seq.meta["block_segments"]
        g, dt = seq.grad.numpy(), seq.dt.numpy()
        a, b = bs[0]
        assert abs(float(np.sum(g[a:b, 0] * dt[a:b])) - amp * (100 + 30) * 1e-6) < 1e-12
        sloped = (g[a:b, 0] != 0) & (g[a:b, 0] != amp)
        assert dt[a:b][sloped].max() <= (ramp or 1e-5) + 1e-12
        a, b = bs[1]  # 0 -> 500 over 30 us, back to 0 over 70 us: moment 500 x 100 us / 2
        assert abs(float(np.sum(g[a:b, 1] * dt[a:b])) - 500.0 * 100e-6 / 2) < 1e-12


def test_arbitrary_gradient_on_the_raster_is_continuous_with_the_block_before():
    """Samples at the raster cells' centres, linear in between; the first edge takes the previous block's last
    value (0 at the start), and the last edge follows from each sample being the mean of its two edges. A ramp
    (100, 200) from 0 ends at 200; the next block's constant 200 then starts at 200, with no dip."""
    text = seq_text([[1, 2, 0, 1, 0, 0, 0, 0], [2, 2, 0, 2, 0, 0, 0, 0]],
                    grads=[[1, 200.0, 1, 0, 0], [2, 200.0, 2, 0, 0]], shapes=[(1, 2, [0.5, 1.0]), (2, 2, [1.0, 1.0])])
    seq = pulseq.read_pulseq(text)
    g, dt = seq.grad[:, 0].numpy(), seq.dt.numpy()
    (a, b), (c, d) = seq.meta["block_segments"]
    # (0, 0), (5 us, 100), (15 us, 200), (20 us, 200): 250 + 1500 + 1000 Hz/m us
    assert abs(float(np.sum(g[a:b] * dt[a:b])) - 2750e-6) < 1e-12
    assert np.allclose(g[c:d], 200.0, rtol=0, atol=1e-9)


def test_delayed_arbitrary_gradient_starts_from_zero():
    """A raster-sampled gradient with a delay, after a block whose gradient ends at 200: the axis is at zero during
    the delay, so the waveform's first edge is 0 (not the previous block's 200). Samples (100, 200) then give the
    edges 0, 200, 200 and the points (0, 0), (5 us, 100), (15 us, 200), (20 us, 200) after the 10 us delay: 250 +
    1500 + 1000 Hz/m us (from the previous block's 200, the edges 200, 0, 400 would give 3750)."""
    text = seq_text([[1, 2, 0, 1, 0, 0, 0, 0], [2, 3, 0, 2, 0, 0, 0, 0]],
                    grads=[[1, 200.0, 1, 0, 0], [2, 200.0, 2, 0, 10]], shapes=[(1, 2, [0.5, 1.0]), (2, 2, [0.5, 1.0])])
    seq = pulseq.read_pulseq(text)
    g, dt = seq.grad[:, 0].numpy(), seq.dt.numpy()
    (a, b), (c, d) = seq.meta["block_segments"]
    assert abs(float(np.sum(g[c:d] * dt[c:d])) - 2750e-6) < 1e-12
    assert np.allclose(g[c:d][np.cumsum(dt[c:d]) <= 10e-6 + 1e-12], 0.0, atol=1e-9)


def test_shape_compression():
    assert np.array_equal(pulseq.decompress_shape([1.0, 0.0, 0.0, 97.0], 100), np.ones(100))
    assert np.array_equal(pulseq.decompress_shape([0.5, 0.25, 0.25], 3), np.array([0.5, 0.25, 0.25]))
    assert np.allclose(pulseq.decompress_shape([0.1, 0.1, 3.0], 5), np.arange(1, 6) * 0.1)
    with pytest.raises(ValueError, match="decodes to"):
        pulseq.decompress_shape([1.0, 0.0, 0.0, 5.0], 100)


def test_reads_a_file_by_path(tmp_path):
    path = tmp_path / "hard.seq"
    path.write_text(hard_pulse(0.0))
    seq = bpb.read_pulseq(path)
    assert seq.n_adc == 0 and abs(float(seq.duration) - 100e-6) < 1e-12 and seq.meta["convention"] == "physical"


def test_refusals():
    with pytest.raises(NotImplementedError, match="format 1.5"):
        pulseq.read_pulseq(seq_text([[1, 1, 0, 0, 0, 0, 0, 0]], version=(1, 5, 0)))
    with pytest.raises(ValueError, match="longer than the block"):
        pulseq.read_pulseq(seq_text([[1, 2, 0, 0, 0, 0, 1, 0]], adc=[[1, 4, 10000, 0, 0, 0]]))
    ext = "[EXTENSIONS]\n1 1 0 0\nextension ROTATIONS 1\n1 0 0 0 1 0 0 0 1"
    with pytest.raises(NotImplementedError, match="ROTATIONS"):
        pulseq.read_pulseq(seq_text([[1, 1, 0, 0, 0, 0, 0, 1]], extensions=ext))
    ext = "[EXTENSIONS]\n1 1 1 0\nextension LABELSET 1\n1 3 LIN"
    assert len(pulseq.read_pulseq(seq_text([[1, 1, 0, 0, 0, 0, 0, 1]], extensions=ext))) == 1
    with pytest.raises(ValueError, match="convention"):
        pulseq.read_pulseq(seq_text([[1, 1, 0, 0, 0, 0, 0, 0]]), convention="other")
