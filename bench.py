"""Benchmark: isochromat-steps/s (spins x segments / s, blochparty's spin-segments/s, benchmarks/bench.py:64) of
the forward simulation and of the forward + adjoint, on N GPUs of one node, one process per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference|reference_gpu]
                    [--workload gre3d_128_4echo|gre3d_64] [--trs T] [--readout fp32|bf16x3]
                    [--pulses step|reuse|surrogate] [--no-grad]

Default workload: the 4-echo 3D GRE on the 128^3 head phantom (8,388,608 spins, 8 coils, 200-step sinc slab
pulses, TR 20 ms; ``blochparty_b200/workloads.py``), its first ``--trs`` TRs (64 of 16,384: the sequence is
TR-periodic, so a whole-TR prefix has the full sequence's work per segment). ``--workload gre3d_64``: the 3D GRE
64^3 (1,048,576 spins), all of its 1,097,728 segments by default.

Prints ONE JSON line on rank 0. ``value``: the whole job's forward isochromat-steps/s with the inputs resident in
HBM, timed with CUDA events (max over ranks). ``fwd_adjoint`` (one GPU): the same for the checkpointed forward +
the hand-written adjoint (gradient of a seeded linear loss of the signal with respect to the RF waveform, the flip
train), with its own roofline. ``e2e``: the forward through the public ``simulate`` call with host inputs, packing
and host<->device copies inside the timed region (wall clock around a synchronising call). Multi-GPU: weak
scaling; every rank simulates its own phantom (the workload with its own sub-voxel offsets), and the float64 raw
signal is summed onto rank 0 with one NCCL reduce per step (the spin sum is the path's only exchange).
``--impl reference``: the reference algorithm on the host CPU (the float64 oracle restating blochparty's core
engine), on a bounded sample of the same workload; rank 0 only. ``--impl reference_gpu``: the reference's own CUDA
engine (installed in ``baseline/_ref``) against this engine on the reference's benchmark cases.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "isochromat-steps/s (fwd)"
UNIT = "isochromat-steps/s"
DEFAULT_TRS = {"gre3d_128_4echo": 64, "gre3d_64": 0}

# algorithmic FP32 flops per spin and segment of the forward kernel (counted from its formulas in
# blochparty_b200/csrc/bloch_common.cuh; kept fixed across versions): RF segment, free segment with cached
# factors, free segment recomputing them, and an ADC sample per coil (complex multiply-add, 8 flops) + 2.
FLOP_RF, FLOP_FREE, FLOP_FREE_MISS, FLOP_ADC_PER_COIL, FLOP_ADC = 125, 16, 34, 8, 2
# (the free segment is counted at its plain float32 cost, 16 flops, although the kernel evaluates it in
# float-float arithmetic; the extra work is precision, not algorithm)


def flops_per_spin(flags: np.ndarray, n_coils: int) -> int:
    rf = (flags & 1) != 0
    same = (flags & 8) != 0
    n_rf = int(rf.sum())
    n_free_cached = int((~rf & same).sum())
    n_free_miss = int((~rf & ~same).sum())
    n_adc = int(((flags & 2) != 0).sum())
    return (FLOP_RF * n_rf + FLOP_FREE * n_free_cached + FLOP_FREE_MISS * n_free_miss
            + (FLOP_ADC_PER_COIL * n_coils + FLOP_ADC) * n_adc)


# the backward's work per spin and segment (counted from blochparty_b200/csrc/adjoint.cu): the interval replay
# repeats the forward's propagation (no coil contraction); the in-window recompute steps in plain float32: RF
# segment 61 flops (rf_step_plain), free segment 13 (free_step_plain) + 18 when it recomputes its factors; the
# reverse sweep without the offsets' gradients (the RF waveform's gradient needs none): RF segment 130 (rf_reverse
# with its rotation factors; 163 with the offsets'), free segment 30 (free_reverse; 58), ADC sample 8 per coil (the
# signal's cotangent; 16 with the coil gradients) + 2.
FLOP_RF_RECOMP, FLOP_FREE_RECOMP, FLOP_FACTORS = 61, 13, 18
# the NUFFT readout's work per spin and run (readout="nufft", counted from bp_forward_kernel's NUFFT path): the
# factors and first sample (34 + 8), the centring shift (6), per grid cell the kernel weight (8) and per (cell,
# term) the weight product (6) and the coil contraction (8 per coil)
FLOP_NUF_RUN, FLOP_NUF_CELL, FLOP_NUF_TERM, FLOP_NUF_TERM_PER_COIL = 48, 8, 6, 8
FLOP_RF_REV, FLOP_FREE_REV, FLOP_ADC_REV_PER_COIL, FLOP_ADC_REV = 130, 30, 8, 2
# the sweep without per-spin gradients (the RF waveform's gradient alone): an RF segment's reverse is 103 flops
# (rf_reverse without the relaxation, PD and B1 terms: rotation factors 25, rotated state 5, R^T a 30, n x a 9, the
# rotation's two gradient components 22, lambda 6, the segment's two partials 4, p2 2); in a window of RF segments
# integrated backward (rf_back) 138, with the input state from R^T n (30) and the relaxation undone (5), and no
# recompute; a free segment's reverse is lambda's alone, 9 flops, and a window of free segments with one factor set
# recomputes nothing
FLOP_RF_REV_NO_SPIN, FLOP_RF_BACK, FLOP_FREE_LAMBDA = 103, 138, 9
# DRAM bytes per spin-segment of the forward kernel, measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of
# one launch over its spins x segments): the float32 readout on the 4-echo head sequence at 96^3 x 4 TRs (14.16 GB for
# 3,538,944 x 2,376) and the NUFFT readout at 64^3 x 4 TRs (3.015 GB for 1,048,576 x 1,864). The traffic is the
# per-window state, spin parameters and coil sensitivities, so it scales with spins x windows.
TRAFFIC_FP32_PER_SPIN_SEGMENT = 14.162e9 / (3538944 * 2376)
TRAFFIC_NUFFT_PER_SPIN_SEGMENT = 3.0147e9 / (1048576 * 1864)


def nufft_flops_per_spin(flags: np.ndarray, n_coils: int, plan) -> int:
    """The forward's algorithmic flops per spin with the NUFFT readout runs: the plain model for every segment
    outside the runs, the NUFFT path's for every run (W + 1 cells per warp on average: a tile's spread), and the
    grid's float64 DFT counted in the finish kernel, not here."""
    keep = np.ones(flags.shape[0], dtype=bool)
    for a, k in plan.runs:
        keep[a:a + k] = False
    cells = plan.W + 1
    per_run = FLOP_NUF_RUN + cells * (FLOP_NUF_CELL + plan.M * (FLOP_NUF_TERM + FLOP_NUF_TERM_PER_COIL * n_coils))
    return flops_per_spin(flags[keep], n_coils) + len(plan.runs) * per_run


def no_recompute_segments(flags: np.ndarray, windows: np.ndarray):
    """((S,) bool, (S,) bool): the segments of the adjoint windows the sweep without per-spin gradients does not
    recompute: uniform runs of free segments (every segment free, the later ones with the first one's factors, a
    spoil at most on the last), which carry lambda alone, and uniform runs of RF segments (every segment RF with the
    first one's dt and offset, no sample, no spoil), which it integrates backward (bp_adjoint_kernel's uniform
    kinds)."""
    free = np.zeros(flags.shape[0], dtype=bool)
    rf = np.zeros(flags.shape[0], dtype=bool)
    for s0, s1, _, _ in windows.tolist():
        f = flags[s0:s1]
        if ((f & 1) == 0).all() and ((f[1:] & 8) != 0).all() and not (f[:-1] & 4).any():
            free[s0:s1] = True
        elif ((f & 1) != 0).all() and ((f[1:] & 32) != 0).all() and not (f & 6).any():
            rf[s0:s1] = True
    return free, rf


def grad_flops_per_spin(flags: np.ndarray, n_coils: int, no_spin=None, replay: bool = True) -> tuple[int, int]:
    """(forward, backward) algorithmic flops per spin of a simulation with gradients (no coil gradients);
    ``no_spin``: for the sweep without per-spin gradients, ``no_recompute_segments`` of its windows; ``replay``:
    whether the backward replays the intervals (not from saved states)."""
    rf = (flags & 1) != 0
    n_adc = int(((flags & 2) != 0).sum())
    fwd = flops_per_spin(flags, n_coils)
    prop = flops_per_spin(flags, 0) - FLOP_ADC * n_adc
    adc = (FLOP_ADC_REV_PER_COIL * n_coils + FLOP_ADC_REV) * n_adc
    if no_spin is None:
        n_rf, n_free = int(rf.sum()), int((~rf).sum())
        n_free_miss = int((~rf & ((flags & 8) == 0)).sum())
        recomp = FLOP_RF_RECOMP * n_rf + FLOP_FREE_RECOMP * n_free + FLOP_FACTORS * n_free_miss
        rev = FLOP_RF_REV * n_rf + FLOP_FREE_REV * n_free + adc
        return fwd, prop + recomp + rev
    lam, back = no_spin
    n_rf_back, n_rf = int(back.sum()), int((rf & ~back).sum())
    n_free = int((~rf & ~lam).sum())
    n_free_miss = int((~rf & ~lam & ((flags & 8) == 0)).sum())
    recomp = FLOP_RF_RECOMP * n_rf + FLOP_FREE_RECOMP * n_free + FLOP_FACTORS * n_free_miss
    rev = (FLOP_RF_BACK * n_rf_back + FLOP_RF_REV_NO_SPIN * n_rf + FLOP_FREE_LAMBDA * int((~rf).sum()) + adc)
    return fwd, (prop if replay else 0) + recomp + rev


class Clocks:
    """nvidia-smi samples (every 200 ms) of the GPU's SM clock and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.rows, self.proc = [], None
        try:
            p = torch.cuda.get_device_properties(device)
            self.sel = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        except Exception:
            self.sel = str(device)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.sel], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        num = lambda v: float(v) if v.replace(".", "", 1).isdigit() else float("nan")
        sm = [num(r[0]) for r in self.rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[4:8]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": num(self.rows[0][1]), "reasons": reasons,
                "samples": len(self.rows), "power_w_max": max(num(r[2]) for r in self.rows)}


def ffma_peak_tflops(dev) -> float:
    from blochparty_b200 import _lib

    out = torch.empty(4 * torch.cuda.get_device_properties(dev).multi_processor_count * 256, device=dev)
    flops = np.zeros(1, dtype=np.int64)
    lib = _lib.lib()
    best = 0.0
    for it in (2000, 2000, 2000):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        _lib.check(lib.bp_ffma_peak(out.data_ptr(), it, flops.ctypes.data, _lib.stream_ptr()), "bp_ffma_peak")
        e.record()
        torch.cuda.synchronize()
        best = max(best, float(flops[0]) / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def build_workload(args, rank: int = 0):
    """(phantom, sequence, coils, description) of the measured workload: rank r > 0 gets the same workload with
    its own sub-voxel offsets (seed 1 + r), for weak scaling."""
    from blochparty_b200 import phantoms, workloads

    if args.workload == "gre3d_128_4echo":
        ph, seq, coils = workloads.gre3d_128_4echo(args.head_n)
        if rank:
            ph = phantoms.head_phantom_3d(args.head_n, 0.25, spins_per_voxel=4, subvoxel_seed=1 + rank, b0_max=150.0)
            coils = phantoms.birdcage_sensitivities(ph.pos, 8)
        desc = (f"gre3d_128_4echo: 4-echo 3D GRE {args.head_n}^3 head phantom, {len(ph.pd):,} spins, 8 coils, "
                f"200-step sinc slab, TR 20 ms, {args.head_n} samples per echo")
    else:
        ph, seq, coils = workloads.gre3d_64(args.n)
        if rank:
            ph = phantoms.ellipsoid_phantom_3d(args.n, 0.25, n_ellipsoids=10, spins_per_voxel=4, seed=0,
                                               subvoxel_seed=1 + rank, b0_seed=2, b0_max=100.0, sigma_vox=4.0)
            coils = phantoms.birdcage_sensitivities(ph.pos, 8)
        desc = (f"gre3d_64: 3D spoiled GRE {args.n}^3, {len(ph.pd):,} spins, 8 coils, 200-step sinc slab, "
                f"TR 8 ms")
    n_tr_all = seq.meta["n_tr"]
    trs = DEFAULT_TRS[args.workload] if args.trs is None else args.trs
    if trs and trs < n_tr_all:
        seq = workloads.first_n_trs(seq, trs)
        desc += f"; its first {trs} TRs ({len(seq):,} segments) of {n_tr_all:,}"
    else:
        desc += f"; all {n_tr_all:,} TRs ({len(seq):,} segments)"
    return ph, seq, coils, desc


def cpu_sample(ph, seq, coils, n_spins=4096, n_tr=32, seed=0):
    """A bounded sample of the workload for the CPU oracle: ``n_spins`` spins drawn with a seeded generator and
    the segments of the first ``n_tr`` TRs."""
    from dataclasses import replace

    from blochparty_b200 import workloads
    from oracle import bloch

    g = torch.Generator().manual_seed(seed)
    idx = torch.randperm(len(ph.pd), generator=g)[:n_spins]
    sub = workloads.first_n_trs(seq, min(n_tr, seq.meta.get("n_tr", n_tr)))
    c = bloch.case_from(ph, sub, coils)
    c = replace(c, pos=c.pos[idx], pd=c.pd[idx], t1=c.t1[idx], t2=c.t2[idx], db0=c.db0[idx], coils=c.coils[idx])
    return c, f"{len(idx)} seeded spins x the first {len(sub)} segments ({n_tr} TRs) of the workload"


def time_cpu(case, reps=1):
    from oracle import bloch

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    best = float("inf")
    for _ in range(reps):
        t = time.perf_counter()
        bloch.simulate(case)
        best = min(best, time.perf_counter() - t)
    n, s = case.pd.shape[0], case.dt.shape[0]
    return n * s / best, threads


def run_reference(args, rank):
    if rank != 0:
        return
    ph, seq, coils, desc = build_workload(args)
    case, sample = cpu_sample(ph, seq, coils)
    rates = []
    for i in range(args.warmup + args.steps):
        v, cores = time_cpu(case)
        if i >= args.warmup:
            rates.append(v)
    value = statistics.median(rates)
    n, s = case.pd.shape[0], case.dt.shape[0]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": n * s / value * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "sample": sample, "readout": "float64 CPU"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


REF_CASES = {"3d-32": 32, "3d-48": 48, "3d-64": 64, "3d-96": 96, "gre3d-128": 128}


def run_reference_gpu(args):
    """The reference's own CUDA engine (``engine="cuda"``: NVRTC-compiled SIMT kernels, blochparty
    ``engines/gpu/cuda/__init__.py:93-132``) on this GPU, installed unmodified in ``baseline/_ref``, against this
    engine on the same inputs: the reference's benchmark cases (``benchmarks/bench.py:36-95``: Shepp-Logan,
    Cartesian spoiled GRE, 8 birdcage coils, 200 dummy TRs, float32) and its 128^3 example
    (``examples/gre3d_128.py:15-27``), built with the reference's own builders. Both through their public
    ``simulate`` from CPU tensors (packing, copies and read-back inside the timing), one untimed warm-up each
    (NVRTC compile), then the fastest of ``--repeat`` runs, wall clock around a synchronising call. ``--grad``: forward
    + backward of sum |signal|^2 with respect to the flip angle, the T1 map and the coil maps (the reference's
    ``run_grad_case``). A case name may add ``+mt`` (every spin with the reference's default bound pool: f 0.1,
    k 30 /s, T1b 1 s, T2b 12 us, super-Lorentzian with its 1 kHz cutoff) and ``+field`` (``scanner``: 0.55 T,
    leading-order concomitant fields), the reference's own objects given to both engines. One JSON line per case."""
    ref = ROOT / "baseline" / "_ref"
    if not (ref / "blochparty").is_dir():
        print(json.dumps({"impl": "reference_gpu", "unavailable": "the reference is not installed in baseline/_ref"}))
        return
    sys.path.insert(0, str(ref))
    import blochparty as bp

    import blochparty_b200 as bpb

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    f32, F64 = torch.float32, torch.float64

    def case(name, grad):
        import dataclasses

        from blochparty.exchange import BoundPool
        from blochparty.fields import Scanner

        base, *extra = name.split("+")
        ph, seq, coils, grad_of = plain_case(base, grad)
        kw = {}
        if "mt" in extra:
            ph = dataclasses.replace(ph, bound=BoundPool(f=0.1, k=30.0, t1=1.0, t2=12e-6))
        if "field" in extra:
            kw["scanner"] = Scanner(field_strength=0.55, concomitant="leading")
        return ph, seq, coils, grad_of, kw

    def plain_case(name, grad):
        n = REF_CASES[name]
        if grad:
            maps = bp.shepp_logan_maps(n, ndim=3, dtype=f32)
            t1 = maps["t1"].clone().requires_grad_()
            ph = bp.phantom_from_maps(maps["pd"], t1, maps["t2"], 0.22)
            coils = bp.birdcage_sensitivities(ph.pos, n_coils=8).detach().requires_grad_()
            flip = torch.tensor(15.0, dtype=f32, requires_grad=True)
            seq = bp.gre_cartesian((n,) * 3, flip_deg=flip, n_dummy=200, dtype=f32)
            return ph, seq, coils, (flip, t1, coils)
        ph = bp.shepp_logan(n, ndim=3, dtype=torch.float64).to(dtype=f32)
        coils = bp.birdcage_sensitivities(ph.pos, n_coils=8)
        if name == "gre3d-128":
            seq = bp.gre_3d(n, flip_deg=15.0, tr=10e-3, n_dummy=200, dtype=f32)
        else:
            seq = bp.gre_cartesian((n,) * 3, n_dummy=200, dtype=f32)
        return ph, seq, coils, ()

    def timed(simulate, name):
        best, out = float("inf"), None
        for i in range(1 + args.repeat):
            ph, seq, coils, grad_of, kw = case(name, args.grad)  # (built outside the timing, as the reference's bench)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sig = simulate(ph, seq, coils, **kw).signal
            if grad_of:
                (sig.abs() ** 2).sum().backward()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            if i > 0:
                best = min(best, dt)
            out = (sig.detach().clone(), [t.grad.clone() for t in grad_of], len(ph.pd), len(seq), int(sum(seq.adc)))
        return best, out

    for name in args.cases.split(","):
        ctx = torch.enable_grad() if args.grad else torch.no_grad()
        with ctx:
            t_ref, (s_ref, g_ref, n, S, n_adc) = timed(lambda p, s, c, **kw: bp.simulate(p, s, c, engine="cuda", **kw),
                                                       name)
            t_b2, (s_b2, g_b2, _, _, _) = timed(bpb.simulate, name)
        rel = lambda a, b: float(torch.linalg.vector_norm((a - b).to(torch.complex128 if b.is_complex() else F64))
                                 / torch.linalg.vector_norm(b.to(torch.complex128 if b.is_complex() else F64)))
        line = {"impl": "reference_gpu", "case": name, "grad": args.grad, "spins": n, "segments": S,
                "adc": n_adc, "gpu": torch.cuda.get_device_name(dev),
                "reference_cuda_s": t_ref, "b200_s": t_b2, "speedup": t_ref / t_b2,
                "reference_cuda_isochromat_steps_per_s": n * S / t_ref, "b200_isochromat_steps_per_s": n * S / t_b2,
                "signal_rel_l2_b200_vs_reference_cuda": rel(s_b2, s_ref),
                "timing": f"fastest of {args.repeat} after one warm-up, public simulate() from CPU tensors"}
        if args.grad:
            line["grad_rel_l2_b200_vs_reference_cuda"] = {k: rel(a, b) for k, a, b in
                                                          zip(("flip", "t1", "coils"), g_b2, g_ref)}
        print(json.dumps(line), flush=True)


def saved_states_text(run) -> str:
    """How the backward of ``run`` (an ``adjoint.Checkpointed``) gets its states."""
    if run.saved is None:
        return "interval starts, each interval replayed"
    blocks = run.blocks()
    if len(blocks) == 1:
        return f"saved by the forward after each of the {run.saved.n_slots} RF runs (no replay)"
    return (f"saved after each of the {run.saved.n_slots} RF runs, {run.layout[1]} at a time: the forward stores the "
            f"starts of {len(blocks)} blocks of {run.layout[0]} intervals, the backward rebuilds each block's states "
            "by one forward of the block (no readout) before its sweep")


def measure_fwd_adjoint(args, dev, pk, state0, flush, n, S):
    """Forward + adjoint on the resident inputs: the checkpointed forward and the backward (reverse sweep and
    segment-gradient reduction per interval, from the states the forward saved after every RF run when they fit,
    else with a replay of each interval first) of a seeded linear loss of the signal, gradient with respect to the
    RF waveform (the flip train), K timed steps with CUDA events around each half. Returns the ``fwd_adjoint``
    object."""
    from blochparty_b200 import _lib, adjoint

    every, outer = adjoint.choose_checkpoints(S, pk.n)
    run = adjoint.Checkpointed(pk, every, dev, outer, saved=not args.replay)
    g = torch.Generator().manual_seed(7)
    w = torch.complex(torch.randn(pk.n_coils, pk.n_adc, generator=g, dtype=torch.float64),
                      torch.randn(pk.n_coils, pk.n_adc, generator=g, dtype=torch.float64))
    h = run.cotangent(w)  # loss = sum(Re s Re w + Im s Im w): dL/ds = w
    lam = torch.zeros(3, pk.n, dtype=torch.float32, device=dev)
    mask = _lib.BP_SEG_WX | _lib.BP_SEG_WY | _lib.BP_SPIN_NO_OFFSETS | _lib.BP_SPIN_NONE
    state = torch.empty_like(state0)

    def step(times=None):
        state.copy_(state0)
        lam.zero_()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        run.forward(state)
        e[1].record()
        run.backward(h, lam, mask, False, True)
        e[2].record()
        if times is not None:
            times.append(e)

    for _ in range(args.warmup):
        step()
    run.check()
    times = []
    clocks = Clocks(dev.index or 0)
    with clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            step(times)
            torch.cuda.synchronize()
    run.check()
    f_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in times)
    b_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in times)
    ms = f_ms + b_ms
    blocked = run.saved is not None and len(run.blocks()) > 1
    fwd, bwd = grad_flops_per_spin(pk.flags, pk.n_coils, no_recompute_segments(pk.flags, run.plan.awin),
                                   replay=run.saved is None or blocked)
    peak = ffma_peak_tflops(dev)
    achieved = n * (fwd + bwd) / (ms * 1e-3) / 1e12
    lf, lb = run.launches(True)
    return {
        "metric": "isochromat-steps/s (fwd+adjoint)", "value": n * S / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
        "forward_ms": f_ms, "backward_ms": b_ms, "steps": args.steps, "warmup": args.warmup,
        "grad_wrt": "the RF waveform (flip train), seeded linear loss of the signal",
        "checkpoint_every": run.plan.every, "intervals": len(run.plan.starts),
        "outer_every": run.outer,  # intervals per outer block (0: two levels); its rebuild forward is not counted
        "states": saved_states_text(run),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": "live FFMA probe (bp_ffma_peak) on this GPU",
                     "kernel": ("bp_forward_kernel (forward" + (")" if run.saved is not None else ", replay)")
                                + " + bp_adjoint_kernel + bp_seg_reduce_kernel"),
                     "flops_per_spin": {"forward": fwd, "backward": bwd}},
        "gpu_launches": args.steps * (lf + lb), "clocks": clocks.summary(),
    }


def e2e_fwd_adjoint(ph, seq, coils):
    """The forward + adjoint through the public API from host tensors (one run after the timed steps): simulate
    with the RF waveform requiring grad, the seeded linear loss, backward; wall clock (ms), bytes in and out."""
    import blochparty_b200 as bpb

    g = torch.Generator().manual_seed(7)
    n_adc = int(sum(seq.adc))
    wr = torch.randn(coils.shape[1], n_adc, generator=g, dtype=torch.float64)
    wi = torch.randn(coils.shape[1], n_adc, generator=g, dtype=torch.float64)
    rf = seq.rf.clone().requires_grad_()
    seqg = bpb.Sequence(seq.dt, rf, seq.grad, seq.adc_phase, list(seq.is_rf), list(seq.adc), list(seq.spoil))
    torch.cuda.synchronize()
    t = time.perf_counter()
    r = bpb.simulate(ph, seqg, coils)
    ((r.signal.real.double() * wr).sum() + (r.signal.imag.double() * wi).sum()).backward()
    torch.cuda.synchronize()
    return (time.perf_counter() - t) * 1e3, rf.grad.numel() * rf.grad.element_size()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference", "reference_gpu"),
                    help="reference: the reference algorithm on the host CPU; reference_gpu: the reference's own CUDA "
                         "engine (baseline/_ref) against this engine on the reference's benchmark cases")
    ap.add_argument("--cases", default="3d-32,3d-48,3d-64,3d-96,gre3d-128", help="--impl reference_gpu: cases")
    ap.add_argument("--repeat", type=int, default=2, help="--impl reference_gpu: timed runs per case (fastest kept)")
    ap.add_argument("--grad", action="store_true", help="--impl reference_gpu: forward + backward")
    ap.add_argument("--replay", action="store_true",
                    help="forward + adjoint: replay every interval instead of the backward from saved states")
    ap.add_argument("--workload", default="gre3d_128_4echo", choices=("gre3d_128_4echo", "gre3d_64"))
    ap.add_argument("--trs", type=int, default=None,
                    help="time the workload's first TRs only (default: 64 for gre3d_128_4echo, all for gre3d_64)")
    ap.add_argument("--head-n", type=int, default=128, help="grid size of the 4-echo head workload (128: as named)")
    ap.add_argument("--n", type=int, default=64, help="grid size of the gre3d_64 workload")
    ap.add_argument("--readout", default="fp32", choices=("fp32", "bf16x3", "nufft"))
    ap.add_argument("--pulses", default="step", choices=("step", "reuse", "surrogate"),
                    help="reuse: recurring pulses through their exact per-spin maps (composed inside every step); "
                         "surrogate: the slab pulse through a network trained before the timed region")
    ap.add_argument("--surrogate-pieces", type=int, default=1, help="networks per slab pulse (--pulses surrogate)")
    ap.add_argument("--surrogate-epochs", type=int, default=400,
                    help="training epochs per network (--pulses surrogate; speed does not depend on them)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-grad", action="store_true", help="skip the forward + adjoint measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.impl == "reference_gpu":
        if rank == 0:
            run_reference_gpu(args)
        return

    import torch.distributed as dist
    from datetime import timedelta

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    import blochparty_b200 as bpb
    from blochparty_b200 import _lib, engine

    ph, seq, coils, workload = build_workload(args, rank)
    inp = bpb.api.Inputs(ph.pos, ph.pd, ph.t1, ph.t2, ph.db0, None, coils, seq.dt, seq.rf, seq.grad,
                         seq.adc_phase, None, list(seq.is_rf), list(seq.adc), list(seq.spoil), None)
    mma = reuse = sur = nr = None
    sur_info = {}
    if args.readout == "nufft":  # the spins sorted by the readout runs' phase, the run tables
        from blochparty_b200 import nufft

        pk, nr, order = nufft.prepare(inp, dev)
        inp = nufft.sorted_inputs(inp, order)
    else:
        pk = engine.pack(inp, dev)
    if args.pulses == "reuse":
        from blochparty_b200.pulses import Reuse

        reuse = Reuse(inp, pk)
        windows, wdev = reuse.plan[0], reuse.plan[1]
    elif args.pulses == "surrogate":
        # one network for the workload's slab pulse (trained before the timed region; speed does not depend on it)
        from blochparty_b200 import surrogate

        is_rf = np.asarray(seq.is_rf, dtype=bool)
        a = int(np.flatnonzero(is_rf)[0])
        k = int(np.flatnonzero(~is_rf[a:])[0])
        sgs = surrogate.pulse_pieces(seq.rf[a:a + k].numpy(), float(seq.dt[a]), float(seq.grad[a, 2]),
                                     float(seq.meta["slab_thickness"]), pieces=args.surrogate_pieces, device=dev)
        t0 = time.perf_counter()
        for sg in sgs:
            sg.train(epochs=args.surrogate_epochs)
        sur_info = {"pieces": args.surrogate_pieces, "epochs": args.surrogate_epochs,
                    "train_s": time.perf_counter() - t0, "network_error_max_rms": [sg.validate() for sg in sgs]}
        sur = surrogate.SurrogateRun(inp, pk, sgs)
        windows, wdev = sur.plan[0], sur.plan[1]
    elif nr is not None:
        windows, wdev = nr.windows, nr.wdev
    elif args.readout == "bf16x3":
        from blochparty_b200.readout_mma import MmaBuffers, run_forward_mma

        mma = MmaBuffers(pk)
        windows, wdev = mma.windows, mma.windows_dev
    else:
        samp = _lib.lib().bp_forward_samp_max(pk.n_coils)
        windows = engine.plan_windows(pk.flags, samp)
        wdev = torch.from_numpy(windows).to(dev)
    state0 = engine.initial_state(inp.pd, None, dev)
    state = torch.empty_like(state0)
    raw = torch.zeros(pk.n_adc, 2 * pk.n_coils, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    n, S = pk.n, len(seq)
    kstart = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kend = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]

    fwd_events = []  # replaced pulses: the forward launches between occurrences, from one untimed pass

    def step(i=None, ev=None):
        state.copy_(state0)
        raw.zero_()
        if i is not None:
            kstart[i].record()
        if reuse is not None:
            reuse.make_maps(pk)
            reuse.run(pk, state, raw, status, events=ev)
        elif sur is not None:
            sur.run(pk, state, raw, status, events=ev)
        elif mma is not None:
            run_forward_mma(pk, mma, state, raw, status)
        elif nr is not None:
            nr.run(state, raw, status)
        else:
            engine.run_forward(pk, state, wdev, 0, windows.shape[0], raw, status)
        if i is not None:
            kend[i].record()
        sig = engine.finish_signal(pk, raw)
        if world > 1:
            dist.reduce(raw, dst=0)
        return sig

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _lib.check_status(status, "bp_forward")
    clocks = Clocks(local)
    elapsed = 0.0
    with clocks:
        for i in range(args.steps):
            flush.zero_()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
            step(i)
            t1.record()
            torch.cuda.synchronize()
            elapsed += t0.elapsed_time(t1)
    _lib.check_status(status, "bp_forward")
    ms = torch.tensor([elapsed / args.steps], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms = float(ms)
    kernel_ms = statistics.mean(kstart[i].elapsed_time(kend[i]) for i in range(args.steps))
    replaced = reuse or sur
    if replaced is not None:  # the forward kernel's own time (the maps or networks excluded), from one more pass
        step(ev=fwd_events)  # whose launches go one by one from Python, each forward launch between two events
        torch.cuda.synchronize()
        kernel_ms = sum(a.elapsed_time(b) for a, b in fwd_events)
    value = world * n * S / (ms * 1e-3)

    # end to end: the public simulate() call with host inputs (packing, copies, kernels, result read-back)
    e2e_ms = []
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        bpb.simulate(ph, seq, coils, readout=args.readout, pulses=args.pulses,
                     **({"surrogate": sur.surrogates} if sur is not None else {}))
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    e2e = world * n * S / (statistics.median(e2e_ms) * 1e-3) if e2e_ms else None
    h2d = sum(t.numel() * t.element_size() for t in (pk.spins, pk.sens, pk.segs, pk.seg64, pk.psi, wdev, state0))
    _lib.check_status(status, "forward")
    d2h = pk.n_coils * pk.n_adc * 8 + state.numel() * 4

    grad_line = None
    if world == 1 and not args.no_grad and replaced is None and mma is None and nr is None:
        grad_line = measure_fwd_adjoint(args, dev, pk, state0, flush, n, S)
        if args.e2e_steps > 0:
            g_ms, g_d2h = e2e_fwd_adjoint(ph, seq, coils)
            grad_line["e2e"] = {"value": n * S / (g_ms * 1e-3), "unit": UNIT, "ms_per_step": g_ms,
                                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h + g_d2h, "runs": 1}

    if rank != 0:
        dist.destroy_process_group() if world > 1 else None
        return
    peak = ffma_peak_tflops(dev)
    stepped = pk.flags
    if replaced is not None:  # the flops of the segments the forward kernel stepped
        keep = np.ones(pk.flags.shape[0], dtype=bool)
        for s0, k in replaced.spans:
            keep[s0:s0 + k] = False
        stepped = pk.flags[keep]
    if sur is not None:  # the networks' signal against plain stepping on the same inputs
        sig_sur = step().clone()
        state.copy_(state0)
        raw.zero_()
        plain = engine.plan_windows(pk.flags, _lib.lib().bp_forward_samp_max(pk.n_coils))
        engine.run_forward(pk, state, torch.from_numpy(plain).to(dev), 0, plain.shape[0], raw, status)
        sig_plain = engine.finish_signal(pk, raw)
        torch.cuda.synchronize()
        sur_info["signal_rel_l2_vs_stepping"] = float(torch.linalg.vector_norm(sig_sur - sig_plain)
                                                      / torch.linalg.vector_norm(sig_plain))
    flops = n * (flops_per_spin(stepped, pk.n_coils) if nr is None else nufft_flops_per_spin(pk.flags, pk.n_coils,
                                                                                            nr.plan))
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    traffic = None  # DRAM bytes per launch, from one ncu capture of the same kernel scaled by spins x segments
    if mma is None and replaced is None:
        per = TRAFFIC_NUFFT_PER_SPIN_SEGMENT if nr is not None else TRAFFIC_FP32_PER_SPIN_SEGMENT
        traffic = {"bytes": per * n * S, "bytes_per_spin_segment": per,
                   "scaled_from": ("ncu capture of bp_forward_kernel with NUFFT runs, head 64^3 x 4 TRs"
                                   if nr is not None else "ncu capture of bp_forward_kernel, head 96^3 x 4 TRs")}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload, "spins_per_gpu": n, "segments": S, "adc_samples": pk.n_adc,
                   "coils": pk.n_coils, "readout": args.readout, "pulses": args.pulses, **({"surrogate": sur_info}
                                                                                               if sur_info else {}),
                   **({"nufft": {"runs": len(nr.plan.runs), "run_samples": nr.plan.L, "grid": nr.plan.G,
                                 "kernel_width": nr.plan.W, "decay_terms": nr.plan.M}} if nr is not None else {}),
                   "ctas": (_lib.lib().bp_forward_mma_grid(n) if mma is not None
                            else _lib.lib().bp_forward_grid(n, pk.n_coils)),
                   "l2": "inputs larger than L2 (state, spins, coils, segments: hundreds of MB per GPU) and a 256 MB L2 "
                         "flush between timed steps"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None if traffic is None else traffic["bytes"],
                     "traffic_source": traffic,
                     "peak_source": "live FFMA probe (bp_ffma_peak) on this GPU; MEASURED_PEAKS.json has no FP32",
                     "kernel": ("bp_forward_mma_kernel" if mma is not None else
                                "bp_forward_kernel (NUFFT runs) + bp_nufft_finish_kernel" if nr is not None
                                else "bp_forward_kernel"),
                     "kernel_ms": kernel_ms,
                     "flops_per_launch": flops},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": statistics.median(e2e_ms) if e2e_ms else None},
        "gpu_launches": ((3 if nr is not None else 2) * args.steps if replaced is None else
                         args.steps * ((len(reuse.pulses) if reuse is not None else 0) + len(replaced.spans)
                                       + len(fwd_events) + 1)),
        "clocks": clocks.summary(),
    }
    if grad_line is not None:
        line["fwd_adjoint"] = grad_line
        line["gpu_launches"] += grad_line["gpu_launches"]
    if world == 1 and not args.no_cpu_baseline:
        case, sample = cpu_sample(ph, seq, coils)
        v, cores = time_cpu(case)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
