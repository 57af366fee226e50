"""Parity at every measured configuration's own size, against the float64 CPU oracle.

Spins are independent, so a seeded subsample of a configuration's spins runs the kernels through exactly the
configuration's own sequence (every segment and every window of the plan) at a size the float64 oracle finishes
in seconds. The oracle here is its C restatement (``oracle/bloch_c.c``, pinned to the reference's core by the
golden fixtures); configuration 3 runs at its full size against the reference's own float64 autograd
(``tests/golden/adjoint128.npz``). Every test prints its errors; the bars:

* plain float32 signal: 1e-5 relative L2 against the oracle fed the engine's float32 inputs (positions, rates,
  coils rounded once, as the engine packs them); against the oracle fed the float64 inputs the difference is that
  rounding's own effect, printed (about 1e-5 with random sub-voxel positions);
* split-bfloat16 readout: 3e-5 (16 mantissa bits per factor);
* learned RF surrogate: 1e-3 against float64;
* gradients: 2e-4 (largest error over the largest value) against the reference's autograd; central differences
  (relative steps of 1e-3 for the spin maps; for the flips a 4-point stencil with steps of 0.25 degree) within 2e-3
  of the difference quotient plus the loss's float32 rounding amplified by the stencil.

Mirrors blochparty ``tests/engines/test_gpu.py:15-83`` and ``tests/engines/test_gpu_grad.py:22-131``.
"""

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import surrogate, workloads
from golden_cases import load_adjoint128
from oracle import bloch, fast

pytestmark = pytest.mark.gpu
F64, C128 = torch.float64, torch.complex128


def l2(a, b):
    return float(torch.linalg.vector_norm(a.to(b.dtype) - b) / torch.linalg.vector_norm(b))


def rel(a, b):
    return float((a.to(b.dtype) - b).abs().max() / b.abs().max())


def subsample(ph, coils, n, seed):
    """n spins of a phantom, drawn without replacement by a seeded generator."""
    idx = torch.randperm(len(ph.pd), generator=torch.Generator().manual_seed(seed))[:n]
    b1 = None if ph.b1 is None else ph.b1[idx]
    return bpb.Phantom(ph.pos[idx], ph.pd[idx], ph.t1[idx], ph.t2[idx], ph.db0[idx], b1=b1), coils[idx]


def f32_inputs(ph, coils):
    """The spin inputs as the engine packs them: positions, PD, 1/T1, 1/T2, dB0, B1 and coils rounded once to
    float32 from float64."""
    r = lambda t: t.to(torch.float32).to(F64)
    b1 = None if ph.b1 is None else r(ph.b1)
    return (bpb.Phantom(r(ph.pos), r(ph.pd), 1.0 / r(1.0 / ph.t1), 1.0 / r(1.0 / ph.t2), r(ph.db0), b1=b1),
            coils.to(torch.complex64).to(C128))


def oracles(ph, seq, coils):
    """The float64 oracle's signal and m on the float64 inputs and on the engine's float32-rounded inputs."""
    sig64, m64 = fast.simulate(bloch.case_from(ph, seq, coils))
    ph32, c32 = f32_inputs(ph, coils)
    sig32, m32 = fast.simulate(bloch.case_from(ph32, seq, c32))
    return sig64, m64, sig32, m32


def test_config2_gre3d_64_both_readouts_over_the_whole_sequence():
    """Configuration 2 (3D GRE 64^3, 1,048,576 spins, 1,097,728 segments): 1,024 seeded spins through every
    segment, the float32 and the split-bfloat16 readouts."""
    ph, seq, coils = workloads.gre3d_64()
    ph, coils = subsample(ph, coils, 1024, seed=0)
    sig64, m64, sig32, m32 = oracles(ph, seq, coils)
    r = bpb.simulate(ph, seq, coils)
    rb = bpb.simulate(ph, seq, coils, readout="bf16x3")
    e = {"fp32": l2(r.signal, sig32), "fp32_vs_f64_inputs": l2(r.signal, sig64), "bf16x3": l2(rb.signal, sig32),
         "bf16x3_vs_f64_inputs": l2(rb.signal, sig64), "m": rel(r.m, m32)}
    print("\nconfig 2, 1,024 spins x 1,097,728 segments: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert e["fp32"] < 1e-5 and e["m"] < 1e-5
    assert e["bf16x3"] < 3e-5


def _loss(signal, s_t):
    d = signal.to(C128) - s_t
    return (d.real ** 2 + d.imag ** 2).sum()


def _flip_grad(g_rf, seq, flips):
    """dL/dflip_i from dL/drf: every TR's hard pulse is flip_i / 360 / duration times its spoiling phase, so
    d rf / d flip_i = rf / flip_i on TR i's pulse segments."""
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    starts = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    rf, g = seq.rf.detach().double(), g_rf.double()
    out = torch.zeros(len(flips), dtype=F64)
    for i, a in enumerate(starts):
        e = a + int(np.argmin(is_rf[a:])) if not is_rf[a:].all() else len(is_rf)
        out[i] = (g[a:e] * rf[a:e]).sum() / float(flips[i])
    return out


def test_config3_adjoint_2d_128_at_full_size():
    """Configuration 3 (2D 128^2, 16,384 spins, 8 coils, 128 per-TR flips, radial B1+) at its full size: the loss
    |s - s_t|^2 against the perturbed-T1 target, its gradients with respect to T1, T2, PD, dB0, B1, the coil
    sensitivities and the flip train with checkpoints every 33 adjoint windows (1,056 segments, the 32-segment
    multiple next to 8 TRs of 133 segments), against the reference's float64 autograd and central differences."""
    z, (ph, seq, coils, flips, t1_target), same = load_adjoint128()
    assert all(same.values()), same
    s_t = torch.complex(torch.from_numpy(z["s_t_re"]).to(F64), torch.from_numpy(z["s_t_im"]).to(F64))
    sig64, _ = fast.simulate(bloch.case_from(ph, seq, coils))
    leaves = {k: v.detach().clone().requires_grad_() for k, v in
              (("t1", ph.t1), ("t2", ph.t2), ("pd", ph.pd), ("db0", ph.db0), ("b1", ph.b1), ("coils", coils),
               ("rf", seq.rf))}
    phg = bpb.Phantom(ph.pos, leaves["pd"], leaves["t1"], leaves["t2"], leaves["db0"], b1=leaves["b1"])
    seqg = bpb.Sequence(seq.dt, leaves["rf"], seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                        list(seq.spoil))
    r = bpb.simulate(phg, seqg, leaves["coils"], checkpoint_every=1056)
    loss = _loss(r.signal, s_t)
    loss.backward()
    e = {"signal": l2(r.signal.detach(), sig64),
         "loss": abs(float(loss.detach()) - float(z["loss"])) / float(z["loss"])}
    for k in ("t1", "t2", "pd", "db0", "b1"):
        e[k] = rel(leaves[k].grad, torch.from_numpy(z[f"grad_{k}"]).to(F64))
    gc_ref = torch.complex(torch.from_numpy(z["grad_coils8_re"]).to(F64), torch.from_numpy(z["grad_coils8_im"]).to(F64))
    e["coils"] = rel(leaves["coils"].grad[::8], gc_ref)
    g_flip = _flip_grad(leaves["rf"].grad, seq, flips)
    e["flips"] = rel(g_flip, torch.from_numpy(z["grad_flips"]))
    print("\nconfig 3 at 128^2 against the reference's float64 autograd: " + ", ".join(f"{k} {v:.2e}"
                                                                                       for k, v in e.items()))
    assert e["signal"] < 1e-5 and e["loss"] < 1e-4
    assert max(e[k] for k in ("t1", "t2", "pd", "db0", "b1", "coils", "flips")) < 2e-4, e

    # central differences: flips through the 4-point stencil (-f(2h) + 8 f(h) - 8 f(-h) + f(-2h)) / 12h with h = 0.25
    # degree, whose truncation error is below 1e-4 of every derivative here in float64 (the 2-point stencil's is 2 %
    # at h = 0.1 degree, flip 3); the float32 forward rounds each loss by about 4e-7 of its value, which the stencil
    # turns into at most 1.5 * 4e-7 * loss / h; and seeded directions of the spin maps (relative steps of 1e-3)
    def loss_at(phx=ph, seqx=seq):
        with torch.no_grad():
            return float(_loss(bpb.simulate(phx, seqx, coils).signal, s_t))

    h, lv = 0.25, float(loss.detach())
    for i in (3, 40, 77, 127):
        f = {}
        for k in (-2, -1, 1, 2):
            fl = flips.clone()
            fl[i] += k * h
            f[k] = loss_at(seqx=workloads.adjoint_2d_128_sequence(fl.numpy()))
        fd = (-f[2] + 8 * f[1] - 8 * f[-1] + f[-2]) / (12 * h)
        assert abs(float(g_flip[i]) - fd) <= 2e-3 * abs(fd) + 1.5 * 4e-7 * lv / h, ("flip", i, float(g_flip[i]), fd)
    gen = torch.Generator().manual_seed(9)
    h = 1e-3
    for k in ("t1", "t2", "pd", "b1"):
        v = torch.randn(len(ph.pd), generator=gen, dtype=F64) * getattr(ph, k)
        moved = {}
        for sgn in (1.0, -1.0):
            kw = {f: getattr(ph, f) for f in ("pos", "pd", "t1", "t2", "db0", "b1")}
            kw[k] = kw[k] + sgn * h * v
            moved[sgn] = loss_at(phx=bpb.Phantom(**kw))
        fd = (moved[1.0] - moved[-1.0]) / (2 * h)
        an = float((leaves[k].grad * v).sum())
        assert abs(an - fd) <= 2e-3 * abs(fd) + 1e-6 * lv, (k, an, fd)


def test_config4_tse_full_size_plain_and_surrogate(tse_surrogates):
    """Configuration 4 (3-slice TSE 128^2 x 8 spins per voxel, 393,216 spins, every pulse, echo and slice): 1,536
    seeded spins through the whole sequence, plain sub-stepped pulses and the learned surrogate."""
    ph, seq, coils = workloads.tse_3slice_128()
    ph, coils = subsample(ph, coils, 1536, seed=4)
    sig64, m64, sig32, _ = oracles(ph, seq, coils)
    plain = bpb.simulate(ph, seq, coils)
    sur = bpb.simulate(ph, seq, coils, pulses="surrogate", surrogate=tse_surrogates)
    e = {"plain": l2(plain.signal, sig32), "plain_vs_f64_inputs": l2(plain.signal, sig64),
         "surrogate_vs_f64": l2(sur.signal, sig64), "surrogate_m_vs_f64": rel(sur.m, m64)}
    print(f"\nconfig 4, 1,536 spins x {len(seq):,} segments: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert e["plain"] < 1e-5
    assert e["surrogate_vs_f64"] < 1e-3


@pytest.fixture(scope="module")
def head_case():
    """Configuration 5's spins (8,388,608: the 128^3 head phantom x 4) subsampled to 512 seeded spins, and its
    sequence's first 2,048 TRs (1,478,656 segments; the full sequence has 16,384 TRs of 722 segments)."""
    ph, seq, coils = workloads.gre3d_128_4echo()
    ph, coils = subsample(ph, coils, 512, seed=5)
    return ph, workloads.first_trs(seq, 2048 * 722), coils


def test_config5_head_128_4echo_readouts_and_surrogate(head_case):
    """Configuration 5 (4-echo 3D GRE 128^3, 8 coils): 512 seeded spins through its first 2,048 TRs, the float32
    and split-bfloat16 readouts with stepped pulses, and the slab pulse through a trained network."""
    ph, seq, coils = head_case
    sig64, m64, sig32, m32 = oracles(ph, seq, coils)
    r = bpb.simulate(ph, seq, coils)
    rb = bpb.simulate(ph, seq, coils, readout="bf16x3")
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    a = int(np.flatnonzero(is_rf)[0])
    k = int(np.flatnonzero(~is_rf[a:])[0])
    sgs = surrogate.pulse_pieces(seq.rf[a:a + k].numpy(), float(seq.dt[a]), float(seq.grad[a, 2]),
                                 float(seq.meta["slab_thickness"]))
    for sg in sgs:
        sg.train()
    rs = bpb.simulate(ph, seq, coils, pulses="surrogate", surrogate=sgs)
    e = {"fp32": l2(r.signal, sig32), "fp32_vs_f64_inputs": l2(r.signal, sig64), "m": rel(r.m, m32),
         "bf16x3": l2(rb.signal, sig32), "surrogate_vs_f64": l2(rs.signal, sig64)}
    print(f"\nconfig 5, 512 spins x {len(seq):,} segments: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert e["fp32"] < 1e-5 and e["m"] < 1e-5
    assert e["bf16x3"] < 3e-5
    assert e["surrogate_vs_f64"] < 1e-3


def test_config5_whole_scan():
    """Configuration 5's whole sequence (16,384 TRs, 11,829,248 segments, 8,388,608 samples per coil): 256 seeded
    spins through every segment, against the float64 oracle fed the engine's float32 inputs."""
    ph, seq, coils = workloads.gre3d_128_4echo()
    ph, coils = subsample(ph, coils, 256, seed=8)
    ph32, c32 = f32_inputs(ph, coils)
    sig32, m32 = fast.simulate(bloch.case_from(ph32, seq, c32))
    r = bpb.simulate(ph, seq, coils)
    e = {"fp32": l2(r.signal, sig32), "m": rel(r.m, m32)}
    print(f"\nconfig 5 whole scan, 256 spins x {len(seq):,} segments: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert r.signal.shape == (8, 8_388_608)
    assert e["fp32"] < 1e-5 and e["m"] < 1e-5


def test_config5_flip_gradient_against_central_differences(head_case):
    """Configuration 5's adjoint: a seeded linear loss of the signal, its gradient with respect to the RF waveform
    (default checkpoint interval) reduced to the flips of three TRs (every pulse segment of TR i scaled by 1 + a),
    against central differences in a (h = 1e-2: the loss sums 8 M float32 samples, whose rounding a smaller step
    would amplify; the quotient's own truncation error is O(h^2)). Bar: 2e-3 of the difference quotient plus 1e-7
    of sum |w| |s|, the loss's scale."""
    ph, seq, coils = head_case
    n_adc = int(sum(seq.adc))
    g = torch.Generator().manual_seed(11)
    wr, wi = torch.randn(coils.shape[1], n_adc, generator=g), torch.randn(coils.shape[1], n_adc, generator=g)
    rf = seq.rf.clone().requires_grad_()

    def seq_with(rfx):
        return bpb.Sequence(seq.dt, rfx, seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc), list(seq.spoil))

    lin = lambda s: float((s.real.double() * wr).sum() + (s.imag.double() * wi).sum())
    r = bpb.simulate(ph, seq_with(rf), coils)
    ((r.signal.real * wr).sum() + (r.signal.imag * wi).sum()).backward()
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    starts = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    h = 1e-2
    sig = r.signal.detach()
    scale = 1e-7 * float((wr * sig.real.double()).abs().sum() + (wi * sig.imag.double()).abs().sum())
    for tr in (100, 1000, 2000):
        a = int(starts[tr])
        e = a + int(np.argmin(is_rf[a:]))
        an = float((rf.grad[a:e].double() * seq.rf[a:e].double()).sum())
        vals = []
        for sgn in (1.0, -1.0):
            rx = seq.rf.clone()
            rx[a:e] *= 1.0 + sgn * h
            with torch.no_grad():
                vals.append(lin(bpb.simulate(ph, seq_with(rx), coils).signal))
        fd = (vals[0] - vals[1]) / (2 * h)
        print(f"\nconfig 5 flip of TR {tr}: adjoint {an:.6e}, central difference {fd:.6e}")
        assert abs(an - fd) <= 2e-3 * abs(fd) + scale, (tr, an, fd)
