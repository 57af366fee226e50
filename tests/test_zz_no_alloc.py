"""The allocation-free adjoint entry point against the regular one, through the C ABI.

``bp_adjoint_noalloc`` serves callers that cannot allocate device memory (a host runtime that hands the library
fixed buffers and forbids allocation while it runs, or a foreign-language binding that passes device pointers but
cannot call cudaMalloc): it keeps the sweep's scratch in a device array inside the library. This test runs one
checkpoint interval of the 2D adjoint workload through ``bp_adjoint`` + ``bp_seg_reduce`` (with scratch allocated
here) and through ``bp_adjoint_noalloc``, twice in a row, and compares lambda, the per-spin and coil gradients and
the segment gradients within the adjoint tests' tolerance (2e-4, largest relative error). It sets up everything
it needs itself, so it passes alone in a fresh process as well as after the other tests.
"""

import numpy as np
import pytest
import torch

from blochparty_b200 import _lib, adjoint, api, engine, workloads
from blochparty_b200._lib import ptr

pytestmark = pytest.mark.gpu
TOL = 2e-4


def rel(a, b):
    s = b.abs().max()
    return float((a - b).abs().max() / s) if s > 0 else float((a - b).abs().max())


def _interval_inputs():
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ph, seq, coils, _, _ = workloads.adjoint_2d_128(16)
    inp = api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, ph.b1, coils, seq.dt, seq.rf, seq.grad, seq.adc_phase,
                     None, list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    pk = engine.pack(inp, dev)
    plan = adjoint.Plan(pk, 8 * _lib.BP_ADJ_WIN, dev)
    k = len(plan.starts) // 2  # an interval in the middle of the sequence
    state = engine.initial_state(inp.pd, None, dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    engine.run_forward(pk, state, plan.fwin_dev, 0, plan.franges[k][0], None, status)
    aa, ab = plan.aranges[k]
    wstates = torch.empty(ab - aa + 1, 6, pk.n, dtype=torch.float32, device=dev)
    engine.run_forward(pk, state, plan.awin_dev, aa, ab, None, status, wstates=wstates, wstate_stride=1)
    wstates[ab - aa].copy_(state)  # the state after the interval's last window
    g = torch.Generator(device="cpu").manual_seed(7)
    h = torch.randn(pk.n_adc, 2 * pk.n_coils, generator=g).to(dev).contiguous()
    lam0 = torch.randn(3, pk.n, generator=g).to(dev).contiguous()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return pk, plan, k, wstates, h, lam0


def _outputs(pk, S):
    dev = pk.device
    return (torch.zeros(8, pk.n, device=dev), torch.zeros(2 * pk.n_coils, pk.n, device=dev),
            torch.zeros(S, 8, dtype=torch.float64, device=dev))


def test_noalloc_adjoint_matches_the_allocating_entry_point():
    lib = _lib.lib()
    pk, plan, k, wstates, h, lam0 = _interval_inputs()
    aa, ab = plan.aranges[k]
    s0, s1 = plan.seg_ranges[k]
    S = pk.flags.shape[0]
    stream = _lib.stream_ptr()

    # the allocating entry point: scratch for the per-CTA segment gradients allocated here
    grid = lib.bp_adjoint_grid(pk.n, pk.n_coils)
    gseg = torch.empty(grid, s1 - s0, 8, device=pk.device)
    lam_ref = lam0.clone()
    gs_ref, gc_ref, seg_ref = _outputs(pk, S)
    status = torch.zeros(1, dtype=torch.int32, device=pk.device)
    _lib.check(lib.bp_adjoint(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                              ptr(plan.awin_dev), aa, ab, s0, s1 - s0, ptr(wstates), ptr(h), pk.n_adc, ptr(lam_ref),
                              ptr(gs_ref), ptr(gc_ref), ptr(gseg), _lib.BP_SEG_ALL, grid, ptr(status), stream),
               "bp_adjoint")
    _lib.check(lib.bp_seg_reduce(ptr(gseg), grid, s1 - s0, s0, ptr(seg_ref), stream), "bp_seg_reduce")
    torch.cuda.synchronize()
    assert seg_ref.abs().max() > 0 and gs_ref.abs().max() > 0

    for call in range(2):  # twice in a row: the shared scratch keeps the first call's contents
        lam = lam0.clone()
        gs, gc, seg = _outputs(pk, S)
        code = lib.bp_adjoint_noalloc(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                      ptr(plan.awin_dev), aa, ab, s0, s1 - s0, ptr(wstates), ptr(h), pk.n_adc,
                                      ptr(lam), ptr(gs), ptr(gc), ptr(seg), ptr(status), stream)
        _lib.check(code, "bp_adjoint_noalloc")
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        errors = {"lam": rel(lam, lam_ref), "gs": rel(gs, gs_ref), "gc": rel(gc, gc_ref),
                  "seg": rel(seg[s0:s1], seg_ref[s0:s1])}
        assert max(errors.values()) < TOL, (call, errors)
        outside = torch.cat([seg[:s0], seg[s1:]])  # rows of other intervals stay untouched
        assert outside.numel() == 0 or float(outside.abs().max()) == 0.0


def test_noalloc_adjoint_rejects_an_interval_beyond_its_scratch():
    lib = _lib.lib()
    pk, plan, k, wstates, h, lam0 = _interval_inputs()
    aa, ab = plan.aranges[k]
    gs, gc, seg = _outputs(pk, pk.flags.shape[0])
    too_long = _lib.BP_NOALLOC_SCRATCH_BYTES // 4 // 8 + 1  # segments: one CTA's share exceeds the array
    status = torch.zeros(1, dtype=torch.int32, device=pk.device)
    code = lib.bp_adjoint_noalloc(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                  ptr(plan.awin_dev), aa, ab, 0, too_long, ptr(wstates), ptr(h), pk.n_adc, ptr(lam0),
                                  ptr(gs), ptr(gc), ptr(seg), ptr(status), _lib.stream_ptr())
    assert code == _lib.BP_E_SIZE


def test_noalloc_adjoint_skips_windows_outside_the_interval():
    """An interval start that does not match the windows (seg0 one adjoint window late, the interval's end
    unchanged): the sweep skips the windows that begin before seg0 instead of writing before its rows of the
    shared scratch, and reports them in the status word; the segment gradients stay inside [seg0, s1)."""
    lib = _lib.lib()
    pk, plan, k, wstates, h, lam0 = _interval_inputs()
    aa, ab = plan.aranges[k]
    s0, s1 = plan.seg_ranges[k]
    S = pk.flags.shape[0]
    seg0 = s0 + _lib.BP_ADJ_WIN
    assert seg0 < s1
    gs, gc, seg = _outputs(pk, S)
    status = torch.zeros(1, dtype=torch.int32, device=pk.device)
    code = lib.bp_adjoint_noalloc(ptr(pk.spins), ptr(pk.sens), pk.n, pk.n_coils, ptr(pk.segs), ptr(pk.seg64),
                                  ptr(plan.awin_dev), aa, ab, seg0, s1 - seg0, ptr(wstates), ptr(h), pk.n_adc,
                                  ptr(lam0.clone()), ptr(gs), ptr(gc), ptr(seg), ptr(status), _lib.stream_ptr())
    _lib.check(code, "bp_adjoint_noalloc")
    torch.cuda.synchronize()
    assert int(status.item()) & 2
    assert float(seg[:seg0].abs().max()) == 0.0
    assert s1 == S or float(seg[s1:].abs().max()) == 0.0
    assert float(seg[seg0:s1].abs().max()) > 0.0
