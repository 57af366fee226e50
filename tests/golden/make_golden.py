"""Writes the golden fixtures ``tests/golden/*.npz`` by running blochparty's own core engine in float64.

Run once, with the reference source tree (its ``src`` directory) on PYTHONPATH:

    PYTHONPATH=<reference>/src python tests/golden/make_golden.py            # the plain cases and adjoint128
    PYTHONPATH=<reference>/src python tests/golden/make_golden.py physics    # bound pool and field model

Each case's inputs are built here with this package's builders and phantoms (seeded), converted to the
reference's ``Phantom`` / ``Sequence`` classes, and simulated by ``blochparty.simulate(..., engine="core")``
(``engines/core.py:487``) in float64. The fixture stores the inputs, the reference's signal and final
magnetization, and, for the gradient cases, the reference's autograd gradients of a fixed linear loss
(the loss of blochparty ``tests/helpers.py:77-92``: seeded float64 weights on signal and m) with respect to
every input tensor. The tests never import the reference: they read these files.
"""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import blochparty as bp  # noqa: E402  (the reference, from PYTHONPATH)
from blochparty.exchange import BoundPool  # noqa: E402

from blochparty_b200 import phantoms, sequences  # noqa: E402

F64 = torch.float64


def ref_objects(ph, seq):
    """The reference's Phantom and Sequence with the same tensors."""
    rph = bp.Phantom(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, b1=ph.b1)
    rseq = bp.Sequence(seq.dt, seq.rf, seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc), list(seq.spoil),
                       {}, seq.b0_offset)
    return rph, rseq


def weights_like(sig, m, seed=1):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(sig.shape, generator=g, dtype=F64), torch.randn(sig.shape, generator=g, dtype=F64),
            torch.randn(m.shape, generator=g, dtype=F64))


def pack(name, ph, seq, coils, m_init, sig, m, grads=None, weights=None):
    out = dict(
        pos=ph.pos.numpy(), pd=ph.pd.numpy(), t1=ph.t1.numpy(), t2=ph.t2.numpy(), db0=ph.db0.numpy(),
        b1=(ph.b1.numpy() if ph.b1 is not None else np.zeros(0)),
        coils_re=coils.real.numpy(), coils_im=coils.imag.numpy(),
        dt=seq.dt.numpy(), rf=seq.rf.numpy(), grad=seq.grad.numpy(), adc_phase=seq.adc_phase.numpy(),
        b0_offset=(seq.b0_offset.numpy() if seq.b0_offset is not None else np.zeros(0)),
        is_rf=np.array(seq.is_rf, bool), adc=np.array(seq.adc, bool), spoil=np.array(seq.spoil, bool),
        m_init=(m_init.numpy() if m_init is not None else np.zeros(0)),
        sig_re=sig.real.numpy(), sig_im=sig.imag.numpy(), m=m.numpy(),
    )
    if grads is not None:
        for k, v in grads.items():
            if v is None:
                continue
            if v.is_complex():
                out[f"grad_{k}_re"], out[f"grad_{k}_im"] = v.real.numpy(), v.imag.numpy()
            else:
                out[f"grad_{k}"] = v.numpy()
        out["w_re"], out["w_im"], out["w_m"] = (w.numpy() for w in weights)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, {k: v.shape for k, v in out.items() if k.startswith(("sig", "m"))})


def run(name, ph, seq, coils, m_init=None, with_grads=False):
    rph, rseq = ref_objects(ph, seq)
    r = bp.simulate(rph, rseq, coils, m_init=m_init, engine="core")
    sig, m = r.signal.detach(), r.m.detach()
    grads = weights = None
    if with_grads:
        weights = weights_like(sig, m)
        leaves = {}

        def leaf(k, t):
            t = t.detach().clone().requires_grad_()
            leaves[k] = t
            return t

        gph = bp.Phantom(leaf("pos", ph.pos), leaf("pd", ph.pd), leaf("t1", ph.t1), leaf("t2", ph.t2),
                         leaf("db0", ph.db0), b1=None if ph.b1 is None else leaf("b1", ph.b1))
        gseq = bp.Sequence(leaf("dt", seq.dt), leaf("rf", seq.rf), leaf("grad", seq.grad),
                           leaf("adc_phase", seq.adc_phase), list(seq.is_rf), list(seq.adc), list(seq.spoil), {},
                           None if seq.b0_offset is None else leaf("b0_offset", seq.b0_offset))
        gc = leaf("coils", coils)
        gm = None if m_init is None else leaf("m_init", m_init)
        rr = bp.simulate(gph, gseq, gc, m_init=gm, engine="core")
        wr, wi, wm = weights
        loss = (rr.signal.real * wr).sum() + (rr.signal.imag * wi).sum() + (rr.m * wm).sum()
        gs = torch.autograd.grad(loss, list(leaves.values()), allow_unused=True)
        grads = dict(zip(leaves, gs))
    pack(name, ph, seq, coils, m_init, sig, m, grads, weights)


def rand_case(seed, n=6, n_coils=3):
    g = torch.Generator().manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    ph = bp.Phantom(pos=(rnd(n, 3) - 0.5) * 0.2, pd=0.5 + rnd(n), t1=0.2 + rnd(n), t2=0.02 + 0.1 * rnd(n),
                    db0=(rnd(n) - 0.5) * 200, b1=0.8 + 0.4 * rnd(n))
    b = sequences.SequenceBuilder()
    for _ in range(4):
        b.rf_waveform(((rnd(40, 2) - 0.5) * 2000).numpy(), 10e-6, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.delay(float(rnd(())) * 3e-3, grad=((rnd(3) - 0.5) * 4000).numpy())
        b.rf(100e-6, flip_deg=180 * float(rnd(())), phase=2 * math.pi * float(rnd(())))
        b.readout(8, 20e-6, grad=((rnd(3) - 0.5) * 3000).numpy(), phase=float(rnd(())) * 6.0)
        b.delay(float(rnd(())) * 3e-3, grad=((rnd(3) - 0.5) * 4000).numpy())
    b.spoil()
    b.rf(200e-6, flip_deg=90.0, n_steps=10)
    b.readout(16, 10e-6, grad=(800.0, -300.0, 150.0), phase=0.7)
    seq = b.build()
    seq.b0_offset = (rnd(len(seq)) - 0.5) * 40
    coils = torch.complex(rnd(n, n_coils) - 0.5, rnd(n, n_coils) - 0.5)
    return ph, seq, coils


def busy_case(seed=3, n=40, n_coils=4):
    """RF of varying phase, readouts split across runs, a spoiled run without ADC, an ADC right after RF, m_init."""
    g = torch.Generator().manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    ph = bp.Phantom(pos=(rnd(n, 3) - 0.5) * 0.2, pd=0.5 + rnd(n), t1=0.2 + rnd(n), t2=0.02 + 0.1 * rnd(n),
                    db0=(rnd(n) - 0.5) * 200)
    b = sequences.SequenceBuilder()
    for i in range(4):
        b.rf(100e-6, amplitude=1500.0, phase=1.3 * i)
        b.delay(0.4e-3, grad=(2000.0, float(rnd(()) - 0.5) * 3000, 0.0))
        b.readout(8, 20e-6, grad=(-2000.0, 0.0, 400.0), phase=0.2 * i)
        b.delay(0.2e-3, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.readout(5, 30e-6, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.delay(1e-3).spoil()
    b.rf(50e-6, amplitude=1500.0)
    b._adc[-1] = True  # a sample at the end of the RF segment itself
    b.readout(3, 10e-6).delay(2e-3, grad=(1e3, 0.0, 0.0)).spoil()
    seq = b.build()
    m_init = torch.stack([(rnd(n) - 0.5) * 0.4, (rnd(n) - 0.5) * 0.4, 0.3 + 0.5 * rnd(n)], -1)
    coils = torch.complex(rnd(n, n_coils) - 0.5, rnd(n, n_coils) - 0.5)
    return ph, seq, coils, m_init


def adjoint128():
    """The 128^2 flip-train case at its own size (16,384 spins, 128 TRs, 8 coils): the reference's float64 core
    and its autograd. Loss = sum |s(T1) - s_t|^2, s_t the signal of the perturbed T1 map. Stored: the target
    signal (complex64), the loss, the gradients with respect to T1, T2, PD, dB0, B1 (float32), the coil
    sensitivities of every 8th spin (complex64) and the flip train (through the RF waveform: every TR's hard
    pulse is flip / 360 / duration times its spoiling phase), and float64 sums of the inputs, so a test can check
    that this package's builders still make the same case."""
    from blochparty_b200 import workloads

    ph, seq, coils, flips, t1_target = workloads.adjoint_2d_128()
    rph, rseq = ref_objects(ph, seq)
    rph_t = bp.Phantom(ph.pos, ph.pd, t1_target, ph.t2, ph.db0, b1=ph.b1)
    s_t = bp.simulate(rph_t, rseq, coils, engine="core").signal.detach()
    leaves = {k: v.detach().clone().requires_grad_() for k, v in
              (("t1", ph.t1), ("t2", ph.t2), ("pd", ph.pd), ("db0", ph.db0), ("b1", ph.b1), ("coils", coils),
               ("rf", seq.rf))}
    gph = bp.Phantom(ph.pos, leaves["pd"], leaves["t1"], leaves["t2"], leaves["db0"], b1=leaves["b1"])
    gseq = bp.Sequence(seq.dt, leaves["rf"], seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc),
                       list(seq.spoil), {}, seq.b0_offset)
    r = bp.simulate(gph, gseq, leaves["coils"], engine="core")
    loss = ((r.signal - s_t).abs() ** 2).sum()
    g = dict(zip(leaves, torch.autograd.grad(loss, list(leaves.values()))))
    # d rf / d flip_i on TR i's pulse segments: rf = flip / 360 / duration (cos phi, sin phi)
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    starts = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    gflip = np.zeros(len(flips))
    rf = seq.rf.numpy()
    for i, a in enumerate(starts[-len(flips):] if len(starts) >= len(flips) else starts):
        e = a
        while e < len(is_rf) and is_rf[e]:
            e += 1
        amp = np.hypot(rf[a:e, 0], rf[a:e, 1])
        unit = rf[a:e] / amp[:, None]
        gflip[i] = float((g["rf"].numpy()[a:e] * unit).sum(1) @ (amp / flips[i].item()))
    sums = {k: float(v.double().sum()) for k, v in (("pos", ph.pos), ("pd", ph.pd), ("t1", ph.t1), ("t2", ph.t2),
                                                     ("db0", ph.db0), ("b1", ph.b1), ("dt", seq.dt),
                                                     ("rf", seq.rf), ("grad", seq.grad), ("t1_target", t1_target),
                                                     ("coils_abs", coils.abs()))}
    out = dict(s_t_re=s_t.real.float().numpy(), s_t_im=s_t.imag.float().numpy(), loss=np.array(float(loss.detach())),
               flips=flips.numpy(), grad_flips=gflip,
               **{f"grad_{k}": g[k].float().numpy() for k in ("t1", "t2", "pd", "db0", "b1")},
               grad_coils8_re=g["coils"][::8].real.float().numpy(), grad_coils8_im=g["coils"][::8].imag.float().numpy(),
               **{f"sum_{k}": np.array(v) for k, v in sums.items()})
    np.savez_compressed(HERE / "adjoint128.npz", **out)
    print("adjoint128", float(loss), {k: v.shape for k, v in out.items() if k.startswith("grad")})


def nonlinearity():
    """x and y coils with third- and fifth-order terms and a z-coil term (r0 = 0.25 m): a few pixels of distortion
    at the edge of a 0.25 m field of view."""
    alpha, beta = torch.zeros(3, 6, 6, dtype=F64), torch.zeros(3, 6, 6, dtype=F64)
    alpha[0, 3, 1], alpha[0, 5, 1], alpha[0, 3, 3] = -0.9, 0.35, 0.2
    beta[1, 3, 1], beta[1, 5, 1], beta[1, 3, 3] = -0.8, 0.3, -0.15
    alpha[2, 3, 0], alpha[2, 2, 1] = -0.4, 0.1
    return alpha, beta, 0.25


def mt_case(seed, shape, n=48, n_coils=4):
    """Spins with a bound pool, three off-resonant shaped saturation pulses (phase ramps) with gradients between
    delays, a hard pulse and a readout, a spoil, an 8-step pulse and a second readout."""
    g = torch.Generator().manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, dtype=F64)
    pool = dict(f=0.08 + 0.12 * rnd(n), k=15 + 45 * rnd(n), t1=0.8 + 0.4 * rnd(n), t2=(8 + 6 * rnd(n)) * 1e-6,
                dw=(rnd(n) - 0.5) * 600)
    ph = bp.Phantom(pos=(rnd(n, 3) - 0.5) * 0.2, pd=0.5 + rnd(n), t1=0.4 + rnd(n), t2=0.02 + 0.08 * rnd(n),
                    db0=(rnd(n) - 0.5) * 200, b1=0.8 + 0.4 * rnd(n),
                    bound=BoundPool(**pool, lineshape=shape))
    b = sequences.SequenceBuilder()
    for _ in range(3):
        k, dt = 48, 10e-6
        t = (torch.arange(k, dtype=F64) + 0.5) * dt
        f_off = float(rnd(()) - 0.5) * 8000
        amp = 200 + 1600 * rnd(k)
        wave = torch.stack([amp * torch.cos(-2 * math.pi * f_off * t), amp * torch.sin(-2 * math.pi * f_off * t)], -1)
        b.rf_waveform(wave.numpy(), dt, grad=((rnd(3) - 0.5) * 2000).numpy())
        b.delay(0.2e-3 + float(rnd(())) * 2e-3, grad=((rnd(3) - 0.5) * 4000).numpy())
    b.rf(100e-6, flip_deg=30.0)
    b.readout(16, 10e-6, grad=(800.0, -300.0, 150.0), phase=0.7)
    b.delay(1e-3).spoil()
    b.rf(200e-6, flip_deg=60.0, n_steps=8)
    b.readout(12, 20e-6, grad=(-500.0, 200.0, 0.0), phase=0.3)
    seq = b.build()
    seq.b0_offset = (rnd(len(seq)) - 0.5) * 20
    coils = torch.complex(rnd(n, n_coils) - 0.5, rnd(n, n_coils) - 0.5)
    return ph, seq, coils, pool


def run_physics(name, ph, seq, coils, pool=None, shape=None, bound_only=None, m_init=None, scanner=None,
                scanner_args=None):
    """The reference's core in float64 on a case with a bound pool and / or a field model; stores the inputs (the
    pool's parameters, bound-only flags, the scanner's), the signal, m and the bound pool's Mz, and what the
    reference derives on the way (its RF frequency per segment, encoding positions and concomitant
    coefficients)."""
    from blochparty.exchange import rf_frequency
    from blochparty.fields import spin_fields

    rseq = bp.Sequence(seq.dt, seq.rf, seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc), list(seq.spoil),
                       {}, seq.b0_offset, None, bound_only)
    rph = bp.Phantom(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, b1=ph.b1, bound=ph.bound)
    r = bp.simulate(rph, rseq, coils, m_init=m_init, scanner=scanner, engine="core")
    plain = bp.simulate(bp.Phantom(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, b1=ph.b1), rseq, coils,
                        m_init=None if m_init is None else m_init[:, :3], engine="core")
    effect = float((r.signal - plain.signal).abs().max() / r.signal.abs().max())
    if scanner is not None and scanner.concomitant is not None:  # the concomitant field's own share
        from blochparty.fields import Scanner

        nl_only = bp.simulate(rph, rseq, coils, m_init=m_init, scanner=Scanner(nonlinearity=scanner.nonlinearity),
                              engine="core")
        conc_effect = float((r.signal - nl_only.signal).abs().max() / r.signal.abs().max())
        print(name, "effect of the concomitant field", f"{conc_effect:.2e}")
        assert conc_effect > 1e-3, conc_effect
    fields = spin_fields(scanner, ph.pos)
    out = dict(
        pos=ph.pos.numpy(), pd=ph.pd.numpy(), t1=ph.t1.numpy(), t2=ph.t2.numpy(), db0=ph.db0.numpy(),
        b1=(ph.b1.numpy() if ph.b1 is not None else np.zeros(0)),
        coils_re=coils.real.numpy(), coils_im=coils.imag.numpy(),
        dt=seq.dt.numpy(), rf=seq.rf.numpy(), grad=seq.grad.numpy(), adc_phase=seq.adc_phase.numpy(),
        b0_offset=(seq.b0_offset.numpy() if seq.b0_offset is not None else np.zeros(0)),
        is_rf=np.array(seq.is_rf, bool), adc=np.array(seq.adc, bool), spoil=np.array(seq.spoil, bool),
        m_init=(m_init.numpy() if m_init is not None else np.zeros(0)),
        bound_only=np.array(bound_only if bound_only is not None else [], bool),
        sig_re=r.signal.real.numpy(), sig_im=r.signal.imag.numpy(), m=r.m.numpy(),
        m_bound=(r.m_bound.numpy() if r.m_bound is not None else np.zeros(0)),
        ref_enc=fields.pos.numpy(), ref_conc=(fields.conc.numpy() if fields.conc is not None else np.zeros(0)),
        ref_mode=np.array(fields.mode), effect=np.array(effect),
    )
    if pool is not None:
        out.update({f"pool_{k}": v.numpy() for k, v in pool.items()})
        out["pool_shape"] = np.array(shape)
        out["ref_rf_freq"] = rf_frequency(rseq).numpy()
    if scanner_args is not None:
        b0, conc, alpha, beta, r0 = scanner_args
        out.update(sc_b0=np.array(np.nan if b0 is None else b0), sc_conc=np.array(conc or ""),
                   sc_alpha=alpha.numpy() if alpha is not None else np.zeros(0),
                   sc_beta=beta.numpy() if beta is not None else np.zeros(0), sc_r0=np.array(r0))
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "effect of the physics on the signal", f"{effect:.2e}")


def field_grad(name, concomitant):
    """Gradients through the scanner field model: a seeded random case (RF waveforms, gradients x 30, a readout)
    at 0.55 T with a nonlinearity, the reference's float64 autograd of a fixed linear loss of signal and m with
    respect to the nonlinearity's alpha, the field strength, T1, the positions, dB0, the RF waveform and the
    gradients."""
    from blochparty.fields import GradientNonlinearity, Scanner

    ph, seq, coils = rand_case(21, n=24, n_coils=2)
    seq.grad = seq.grad * 30
    alpha, beta, r0 = nonlinearity()
    leaves = {"alpha": alpha.clone().requires_grad_(), "b0": torch.tensor(0.55, dtype=F64, requires_grad=True),
              "t1": ph.t1.clone().requires_grad_(), "pos": ph.pos.clone().requires_grad_(),
              "db0": ph.db0.clone().requires_grad_(), "rf": seq.rf.clone().requires_grad_(),
              "grad": seq.grad.clone().requires_grad_()}
    sc = Scanner(field_strength=leaves["b0"], concomitant=concomitant,
                 nonlinearity=GradientNonlinearity(leaves["alpha"], beta, r0))
    rph = bp.Phantom(leaves["pos"], ph.pd, leaves["t1"], ph.t2, leaves["db0"], b1=ph.b1)
    rseq = bp.Sequence(seq.dt, leaves["rf"], leaves["grad"], seq.adc_phase, list(seq.is_rf), list(seq.adc),
                       list(seq.spoil), {}, seq.b0_offset)
    r = bp.simulate(rph, rseq, coils, scanner=sc, engine="core")
    wr, wi, wm = weights_like(r.signal.detach(), r.m.detach())
    loss = (r.signal.real * wr).sum() + (r.signal.imag * wi).sum() + (r.m * wm).sum()
    g = dict(zip(leaves, torch.autograd.grad(loss, list(leaves.values()))))
    out = dict(
        pos=ph.pos.numpy(), pd=ph.pd.numpy(), t1=ph.t1.numpy(), t2=ph.t2.numpy(), db0=ph.db0.numpy(),
        b1=ph.b1.numpy(), coils_re=coils.real.numpy(), coils_im=coils.imag.numpy(),
        dt=seq.dt.numpy(), rf=seq.rf.numpy(), grad=seq.grad.numpy(), adc_phase=seq.adc_phase.numpy(),
        b0_offset=seq.b0_offset.numpy(), is_rf=np.array(seq.is_rf, bool), adc=np.array(seq.adc, bool),
        spoil=np.array(seq.spoil, bool), sc_alpha=alpha.numpy(), sc_beta=beta.numpy(), sc_r0=np.array(r0),
        sc_b0=np.array(0.55), sc_conc=np.array(concomitant), w_re=wr.numpy(), w_im=wi.numpy(), w_m=wm.numpy(),
        sig_re=r.signal.detach().real.numpy(), sig_im=r.signal.detach().imag.numpy(), m=r.m.detach().numpy(),
        **{f"grad_{k}": v.numpy() for k, v in g.items()})
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, {k: float(v.abs().max()) for k, v in g.items()})


def physics():
    """The bound-pool and field-model fixtures, and the reference's super-Lorentzian table."""
    from blochparty.exchange import _sl_table
    from blochparty.fields import GradientNonlinearity, Scanner

    lx, lf = _sl_table(F64, torch.device("cpu"))
    np.savez_compressed(HERE / "sl_table.npz", lx=lx.numpy(), log_f=lf.numpy())
    ph, seq, coils, pool = mt_case(11, "superlorentzian")
    run_physics("mt_sl", ph, seq, coils, pool, "superlorentzian")
    ph, seq, coils, pool = mt_case(12, "lorentzian")
    g = torch.Generator().manual_seed(13)
    m0 = torch.cat([(torch.rand(len(ph.pd), 2, generator=g, dtype=F64) - 0.5) * 0.4,
                    0.3 + 0.5 * torch.rand(len(ph.pd), 1, generator=g, dtype=F64),
                    0.05 * torch.rand(len(ph.pd), 1, generator=g, dtype=F64)], 1)
    bo = [False] * len(seq)
    for s in range(48, 96):  # the second saturation pulse: felt by the bound pool alone
        bo[s] = bool(seq.is_rf[s])
    run_physics("mt_lor", ph, seq, coils, pool, "lorentzian", bound_only=bo, m_init=m0)
    alpha, beta, r0 = nonlinearity()
    # a 3D slab GRE (8^3 ellipsoids, a 20-step sinc slab, two echoes): spins off the z = 0 plane and gradients on
    # every axis, where the concomitant field matters
    p = phantoms.ellipsoid_phantom_3d(8, 0.25, spins_per_voxel=1, b0_max=30.0, sigma_vox=1.0)
    gseq = sequences.gre((8, 8, 8), 0.25, flip_deg=20.0, tr=8e-3, te=3e-3, dwell=20e-6, rf="sinc", rf_duration=1e-3,
                         rf_steps=20, slab_thickness=0.2, n_echoes=2, echo_spacing=0.5e-3, n_dummy=2)
    gcoils = phantoms.birdcage_sensitivities(p.pos, 4)
    gph = bp.Phantom(p.pos, p.pd, p.t1, p.t2, p.db0, b1=p.b1)
    for name, conc in (("field_nl", None), ("field_leading", "leading"), ("field_exact", "exact")):
        nl = GradientNonlinearity(alpha, beta, r0)
        sc = Scanner(field_strength=None if conc is None else 0.55, concomitant=conc, nonlinearity=nl)
        run_physics(name, gph, gseq, gcoils, scanner=sc,
                    scanner_args=(None if conc is None else 0.55, conc, alpha, beta, r0))
    # the same 3D slab GRE with a bound pool on every spin
    g = torch.Generator().manual_seed(14)
    n = len(p.pd)
    rnd = lambda *sh: torch.rand(*sh, generator=g, dtype=F64)
    pool = dict(f=0.08 + 0.12 * rnd(n), k=15 + 45 * rnd(n), t1=0.8 + 0.4 * rnd(n), t2=(8 + 6 * rnd(n)) * 1e-6,
                dw=(rnd(n) - 0.5) * 600)
    mph = bp.Phantom(p.pos, p.pd, p.t1, p.t2, p.db0, b1=p.b1, bound=BoundPool(**pool))
    sc = Scanner(field_strength=0.55, concomitant="leading", nonlinearity=GradientNonlinearity(alpha, beta, r0))
    run_physics("mt_field", mph, gseq, gcoils, pool, "superlorentzian", scanner=sc,
                scanner_args=(0.55, "leading", alpha, beta, r0))
    field_grad("grad_field_leading", "leading")
    field_grad("grad_field_exact", "exact")


def main():
    torch.set_default_dtype(F64)
    if "adjoint128" in sys.argv[1:]:
        adjoint128()
        return
    if "physics" in sys.argv[1:]:
        physics()
        return
    for seed in (0, 1):
        ph, seq, coils = rand_case(seed)
        run(f"rand{seed}", ph, seq, coils)
    ph, seq, coils, m_init = busy_case()
    run("busy", ph, seq, coils, m_init)
    # 2D GRE, 16 x 16 ellipses, 4 coils, RF spoiling, 5 dummies, radial B1, a b0_offset ramp
    p = phantoms.ellipse_phantom_2d(16, 0.25, seed=0)
    p.b1 = phantoms.radial_b1(p.pos)
    seq = sequences.gre((16, 16), 0.25, flip_deg=30.0, tr=6e-3, te=3e-3, n_dummy=5, dwell=20e-6)
    seq.b0_offset = torch.linspace(-5.0, 5.0, len(seq), dtype=F64)
    run("gre16", p, seq, phantoms.birdcage_sensitivities(p.pos, 4))
    # 3D GRE, 4^3 ellipsoids x 2 sub-voxel spins, a 20-step sinc slab pulse, 2 echoes
    p = phantoms.ellipsoid_phantom_3d(4, 0.25, spins_per_voxel=2, b0_max=50.0, sigma_vox=1.0)
    seq = sequences.gre((4, 4, 8), 0.25, flip_deg=20.0, tr=6e-3, te=2.5e-3, dwell=20e-6, rf="sinc",
                        rf_duration=1e-3, rf_steps=20, slab_thickness=0.2, n_echoes=2, echo_spacing=0.4e-3)
    run("sinc3d", p, seq, phantoms.birdcage_sensitivities(p.pos, 3))
    # gradients: small cases with every input differentiated
    ph, seq, coils = rand_case(7, n=5, n_coils=2)
    run("grad_rand", ph, seq, coils, with_grads=True)
    ph, seq, coils, m_init = busy_case(seed=8, n=6, n_coils=2)
    run("grad_busy", ph, seq, coils, m_init, with_grads=True)


if __name__ == "__main__":
    main()
    if not sys.argv[1:]:
        adjoint128()
