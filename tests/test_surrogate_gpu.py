"""The learned RF surrogate on the GPU: training kernels against the float64 oracle, training, tensor-core
inference against float32 inference, and the TSE workload through the surrogate against the float64 plain
integrator.

Bars: targets (float64 composition rounded to float32) within 1e-6 of the oracle; the training kernel's gradient
within 1e-4 (largest relative error) of float64 autograd; tensor-core inference within 1e-4 of float32 inference
(magnetization, unit PD scale), the fallback spins bit-identical; the TSE and the 3D GRE through the surrogate
within 1e-3 relative L2 of the float64 oracle (whole-pulse relax / rotate / relax splitting alone is 2.3e-2 off on
the TSE's refocusing train; the networks' first-order relaxation terms bring the splitting to 1.0e-4 with exact
terms, `test_surrogate_host.py::test_first_order_pulse_map_reaches_the_stepped_signal`, so the rest is the
networks' own error: the refocusing pulses' rotations dominate it); and a measured speed-up over plain
sub-stepping on the same GPU.
"""

import math
import time

import numpy as np
import pytest
import torch

import blochparty_b200 as bpb
from blochparty_b200 import _lib, sequences, surrogate, workloads
from blochparty_b200._lib import ptr
from oracle import bloch
from oracle import surrogate as S

pytestmark = pytest.mark.gpu
F64 = torch.float64


def _pulse(flip=90.0, z0=0.0, phase=0.0):
    return sequences.sinc_pulse(flip, 3e-3, 300, slice_thickness=5e-3, slice_offset=z0, phase=phase)


def test_targets_match_the_float64_oracle():
    w, dt, gz, _ = _pulse(180.0, 5e-3, 0.5 * math.pi)
    sg = surrogate.RFSurrogate(w, dt, gz, 5e-3)
    s = sg.samples(2000, seed=3)
    tg, qf = sg.targets(s, full=True)
    sc = s.double().cpu()
    q_ref, tg_ref = S.pulse_targets(w, dt, gz, sg.z0 + sc[:, 2] * 5e-3, sc[:, 0], sc[:, 1])
    assert float((tg.double().cpu()[:, :4] - tg_ref[:, :4]).abs().max()) < 1e-6
    assert float((qf.double().cpu() - q_ref).abs().max()) < 1e-6
    # the first-order terms (float64 sums of float64 steps on both sides, rounded once to float32)
    assert float((tg.double().cpu()[:, 4:] - tg_ref[:, 4:]).abs().max()) < 1e-6


@pytest.mark.parametrize("vweight,cweight", [(1.0, 1.0), (130.0, 0.01)])
def test_training_gradient_matches_float64_autograd(vweight, cweight):
    w, dt, gz, _ = _pulse()
    sg = surrogate.RFSurrogate(w, dt, gz, 5e-3, seed=11)
    s = sg.samples(300, seed=4)  # 300: the last CTA is partly empty
    x, t = sg.normalise(s), sg.targets(s)
    loss, grad = sg.gradient(x, t, vweight, cweight)
    ref_loss, ref_grad = S.loss_and_grad(sg.params.double().cpu(), x.double().cpu(), t.double().cpu(), vweight,
                                         cweight)
    assert abs(float(loss) - ref_loss) < 1e-5 * max(1.0, ref_loss)
    err = float((grad.double().cpu() - ref_grad).abs().max() / ref_grad.abs().max())
    assert err < 1e-4, err


def test_adam_step():
    lib = _lib.lib()
    g = torch.Generator().manual_seed(0)
    p = torch.randn(_lib.BP_MLP_PARAMS, generator=g).cuda()
    grad = torch.randn(_lib.BP_MLP_PARAMS, generator=g).cuda()
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    ref = p.clone()
    rm, rv = torch.zeros_like(p), torch.zeros_like(p)
    for step in (1, 2, 3):
        _lib.check(lib.bp_adam(ptr(p), ptr(grad), ptr(m), ptr(v), 1e-3, 0.9, 0.999, 1e-8, step, _lib.stream_ptr()),
                   "bp_adam")
        rm = 0.9 * rm + 0.1 * grad
        rv = 0.999 * rv + 0.001 * grad * grad
        ref -= 1e-3 * (rm / (1 - 0.9 ** step)) / ((rv / (1 - 0.999 ** step)).sqrt() + 1e-8)
    torch.cuda.synchronize()
    assert float((p - ref).abs().max()) < 1e-6


def test_training_lowers_the_loss_and_the_error():
    w, dt, gz, _ = _pulse()
    sg = surrogate.RFSurrogate(w, dt, gz, 5e-3)
    before = sg.validate(1 << 14)
    log = sg.train(n_samples=1 << 17, epochs=20, batch=8192)
    after = sg.validate(1 << 14)
    print("\nshort training: loss %.2e -> %.2e, max error %.2e -> %.2e" % (log.loss[0], log.loss[-1], before[0],
                                                                           after[0]))
    assert log.loss[-1] < 0.05 * log.loss[0]
    assert after[1] < 0.1 * before[1]


def test_tse_through_the_surrogate_against_the_float64_oracle(tse_surrogates):
    ph, seq, coils = workloads.tse_3slice_128(16)
    sig64, m64 = bloch.simulate(bloch.case_from(ph, seq, coils))
    plain = bpb.simulate(ph, seq, coils)
    sur = bpb.simulate(ph, seq, coils, pulses="surrogate", surrogate=tse_surrogates)
    l2 = lambda a: float(torch.linalg.vector_norm(a.to(sig64.dtype) - sig64) / torch.linalg.vector_norm(sig64))
    e_sur, e_plain = l2(sur.signal), l2(plain.signal)
    print(f"\nTSE 16^2 x 3 slices: surrogate rel L2 {e_sur:.2e}, plain sub-stepping {e_plain:.2e} (vs float64)")
    # splitting alone is 2.3e-2 off here; with exact first-order terms 1.0e-4 (the host test of pulse_map)
    assert e_plain < 2e-5
    assert e_sur < 1e-3


def test_surrogate_gain_on_the_tse_workload(tse_surrogates):
    """What the trained networks gain over the method without them: the full 3-slice TSE (393,216 spins), the
    same GPU, plain sub-stepped pulses against the surrogate (timed after a warm-up run of each)."""
    from blochparty_b200.api import Inputs

    ph, seq, coils = workloads.tse_3slice_128()
    inp = Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase, None,
                 list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    dev = torch.device("cuda", 0)
    from blochparty_b200 import engine

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t, out

    t_plain, (s_plain, _) = timed(lambda: engine.forward(inp, dev))
    t_fp32, _ = timed(lambda: surrogate.run_with_surrogates(inp, dev, tse_surrogates, "fp32"))
    t_sur, (s_sur, _, counts) = timed(lambda: surrogate.run_with_surrogates(inp, dev, tse_surrogates))
    rel = float(torch.linalg.vector_norm(s_sur - s_plain) / torch.linalg.vector_norm(s_plain))
    frac = counts[0] / max(1, sum(counts))
    print(f"\nTSE 393,216 spins: plain {t_plain:.3f} s, surrogate {t_sur:.3f} s (tensor cores; float32 inference "
          f"{t_fp32:.3f} s), speed-up {t_plain / t_sur:.2f}x; {100 * frac:.1f}% of spin-pulse pairs through the "
          f"networks; signal difference {rel:.1e}")
    assert t_sur < t_plain
    assert rel < 1e-3

    # one pulse occurrence at kernel level (CUDA events, 20 repetitions): the plain forward over the pulse's
    # windows against both inference kernels, on the same state
    pk = engine.pack(inp, dev)
    s, k, i, phi0, b0 = surrogate.find_occurrences(tse_surrogates, inp)[1]
    breaks = np.zeros(pk.flags.shape[0], dtype=np.uint8)
    breaks[s] = breaks[s + k] = 1
    windows = engine.plan_windows(pk.flags, _lib.lib().bp_forward_samp_max(pk.n_coils), breaks=breaks)
    wdev = torch.from_numpy(windows).to(dev)
    wa, wb = int(np.searchsorted(windows[:, 0], s)), int(np.searchsorted(windows[:, 0], s + k))
    state = engine.initial_state(inp.pd, None, dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    lib, st, sg = _lib.lib(), _lib.stream_ptr(), tse_surrogates[i]
    wt = sg.wtiles()

    def events(fn, reps=20):
        fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    host = sg.params_host().ctypes.data
    plain = lambda: engine.run_forward(pk, state, wdev, wa, wb, None, status)
    mma = lambda: lib.bp_surrogate_pulse_mma(ptr(pk.spins), ptr(state), pk.n, host, ptr(wt), ptr(pk.segs), s, k,
                                             sg.T, sg.gz, sg.thickness, sg.z0, phi0, b0, *sg.domain, None,
                                             ptr(status), 0, st)
    # three rounds, each timing both forms back to back; the best round's ratio (the forms share the GPU's state)
    rounds = [(events(plain), events(mma)) for _ in range(3)]
    p_plain, p_mma = max(rounds, key=lambda r: r[0] / r[1])
    p_fp32 = events(lambda: lib.bp_surrogate_pulse(ptr(pk.spins), ptr(state), pk.n, ptr(sg.params), ptr(pk.segs), s,
                                                   k, sg.T, sg.gz, sg.thickness, sg.z0, phi0, b0, *sg.domain, None,
                                                   st))
    assert int(status) == 0
    print(f"one {k}-step pulse over {pk.n:,} spins: plain {p_plain:.3f} ms, float32 network {p_fp32:.3f} ms, "
          f"tensor-core network {p_mma:.3f} ms ({p_plain / p_mma:.2f}x; rounds "
          + ", ".join(f"{a / b:.2f}x" for a, b in rounds) + ")")
    # the target: the surrogate form of a pulse at least 3x faster than its plain sub-stepping, at the accuracy the
    # TSE test above checks (1e-3 against float64)
    assert p_plain / p_mma >= 3.0


def test_weight_tiles_layout():
    """bp_mlp_wtiles: every weight is hi + lo at its operand-layout position, hi = bf16(w) (nearest); W1's two
    padding columns are zero."""
    sg = surrogate.RFSurrogate(*_pulse()[:3], 5e-3, seed=21)
    all_ = sg.wtiles().cpu().view(torch.int16).view(torch.bfloat16).float()
    assert all_.numel() == 16384 + 2048 + 2048
    # element (n / 8) 512 + (k / 8) 64 + (n % 8) 8 + k % 8 -> [n // 8, k // 8, n % 8, k % 8]
    t = all_[:16384].reshape(4, 8, 8, 8, 8).permute(0, 1, 3, 2, 4).reshape(4, 64, 64)
    # W1 (64 x 16): (n / 8) 128 + (k / 8) 64 + (n % 8) 8 + k % 8; W4 (16 x 64) as W2
    t1 = all_[16384:18432].reshape(2, 8, 2, 8, 8).permute(0, 1, 3, 2, 4).reshape(2, 64, 16)
    t4 = all_[18432:].reshape(2, 2, 8, 8, 8).permute(0, 1, 3, 2, 4).reshape(2, 16, 64)
    w1, _, w2, _, w3, _, w4, _ = S.unflatten(sg.params.cpu())
    w1 = torch.cat([w1, torch.zeros(64, 2)], 1)
    for hi, lo, w in ((t[0], t[1], w2), (t[2], t[3], w3), (t1[0], t1[1], w1), (t4[0], t4[1], w4)):
        assert torch.equal(hi, w.to(torch.bfloat16).float())
        assert float(((hi + lo) - w).abs().max() / w.abs().max()) < 2 ** -16


@pytest.mark.parametrize("n,max_ctas", [(300, 0), (300, 1), (5000, 7)])
def test_tensor_core_inference_matches_fp32_inference(n, max_ctas):
    """bp_surrogate_pulse_mma against bp_surrogate_pulse on one occurrence: the same counts, spins outside the
    domain bit-identical (both take the plain fallback), spins inside within the split-bfloat16 rounding."""
    w, dt, gz, _ = _pulse(90.0)
    sg = surrogate.RFSurrogate(w, dt, gz, 5e-3, seed=7)
    sg.train(n_samples=1 << 15, epochs=4, batch=4096)
    seq = sequences.SequenceBuilder().rf_waveform(w, dt, grad=(0.0, 0.0, gz)).build()
    g = torch.Generator().manual_seed(n)
    pos = torch.zeros(n, 3, dtype=F64)
    pos[:, 2] = (torch.rand(n, generator=g, dtype=F64) - 0.5) * 6 * 5e-3  # |z_rel| up to 3: some outside
    ph = bpb.Phantom(pos, torch.rand(n, generator=g, dtype=F64), 0.3 + torch.rand(n, generator=g, dtype=F64),
                     0.02 + 0.1 * torch.rand(n, generator=g, dtype=F64),
                     (torch.rand(n, generator=g, dtype=F64) - 0.5) * 500.0)
    from blochparty_b200 import engine
    from blochparty_b200.api import Inputs

    ones = torch.ones(n, 1, dtype=torch.complex128)
    inp = Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, ones, seq.dt, seq.rf, seq.grad, seq.adc_phase, None,
                 list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    dev = torch.device("cuda", 0)
    pk = engine.pack(inp, dev)
    m0 = torch.rand(n, 3, generator=g, dtype=F64) - 0.5
    lib, st = _lib.lib(), _lib.stream_ptr()
    out = []
    for mma in (False, True):
        state = engine.initial_state(inp.pd, m0, dev)
        counts = torch.zeros(2, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        phi0 = 0.3  # (the fallback steps the sequence's own segments; both kernels see the same arguments)
        if mma:
            code = lib.bp_surrogate_pulse_mma(ptr(pk.spins), ptr(state), n, sg.params_host().ctypes.data,
                                              ptr(sg.wtiles()), ptr(pk.segs), 0, sg.K, sg.T, sg.gz, sg.thickness,
                                              sg.z0, phi0, 10.0,
                                              *sg.domain, ptr(counts), ptr(status), max_ctas, st)
        else:
            code = lib.bp_surrogate_pulse(ptr(pk.spins), ptr(state), n, ptr(sg.params), ptr(pk.segs), 0, sg.K, sg.T,
                                          sg.gz, sg.thickness, sg.z0, phi0, 10.0, *sg.domain, ptr(counts), st)
        _lib.check(code, "surrogate pulse")
        torch.cuda.synchronize()
        assert int(status) == 0
        out.append((state.cpu(), counts.cpu().tolist()))
    (s32, c32), (smma, cmma) = out
    assert c32 == cmma and c32[0] > 0 and c32[1] > 0 and sum(c32) == n
    # the kernels' domain test, in their float32 / float64 arithmetic
    df = ph.db0.numpy().astype(np.float32) + np.float32(10.0)
    zr = ((pos[:, 2].numpy().astype(np.float32).astype(np.float64) - sg.z0) / 5e-3).astype(np.float32)
    inside = torch.from_numpy((np.abs(df) <= np.float32(200.0)) & (np.abs(zr) <= np.float32(2.0)))
    assert int(inside.sum()) == c32[0]
    assert torch.equal(s32[:, ~inside], smma[:, ~inside])
    err = float((s32[:3, inside] - smma[:3, inside]).abs().max())
    print(f"\ntensor-core vs fp32 inference, n={n}: largest magnetization difference {err:.1e}")
    assert err < 1e-4


@pytest.mark.parametrize("pieces", [1, 2])
def test_gre_slab_pulse_against_the_float64_oracle(pieces):
    """The RF-spoiled 3D GRE (16^3 voxels x 4 spins, 256 TRs) with its 200-step slab pulse through ``pieces``
    networks of 200 / pieces steps, against the float64 oracle fed the engine's float32 spin inputs: within 1e-3
    either way."""
    ph, seq, coils = workloads.gre3d_64(16)
    is_rf = np.asarray(seq.is_rf, dtype=bool)
    a = int(np.flatnonzero(is_rf)[0])
    k = int(np.flatnonzero(~is_rf[a:])[0])
    sgs = surrogate.pulse_pieces(seq.rf[a:a + k].numpy(), float(seq.dt[a]), float(seq.grad[a, 2]),
                                 float(seq.meta["slab_thickness"]), pieces=pieces)
    for sg in sgs:
        sg.train()
    r32 = lambda t: t.to(torch.float32).to(torch.float64)
    phq = bpb.Phantom(r32(ph.pos), r32(ph.pd), 1.0 / r32(1.0 / ph.t1), 1.0 / r32(1.0 / ph.t2), r32(ph.db0))
    sig64, _ = bloch.simulate(bloch.case_from(phq, seq, coils))
    sur = bpb.simulate(ph, seq, coils, pulses="surrogate", surrogate=sgs)
    err = float(torch.linalg.vector_norm(sur.signal.to(sig64.dtype) - sig64) / torch.linalg.vector_norm(sig64))
    print(f"\nGRE 16^3 slab pulse in {pieces} piece(s): surrogate rel L2 {err:.2e} against float64")
    assert err < 1e-3
