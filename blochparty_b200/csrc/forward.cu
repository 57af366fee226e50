// Forward propagation kernel (plain float32 readout) and its C-ABI launcher.
//
// Replaces blochparty's bloch_chunk / bloch_chunk_mma (engines/gpu/cuda/kernels.cu.in:2-185) for static spins
// with PD, T1, T2, dB0, B1+, receive coils and b0_offset (the V=0 variant), driven by
// engines/gpu/driver.py:_forward (:197-756).
//
// Work decomposition (persistent, window-major):
//  * The sequence is cut on the host into windows of consecutive segments (at most BP_SEG_MAX segments and
//    samp_max(NCG) ADC samples each).
//  * A CTA of 128 threads owns every grid-th spin tile from its own index (128 spins each, one spin per thread;
//    the NUFFT kernel a contiguous block of tiles). For every window it stages the window's segment records into
//    shared memory with one TMA bulk copy (double-buffered: window w+1 is in flight while window w runs), then
//    runs each of its tiles through the window: the tile's state is loaded from HBM, propagated in registers,
//    and stored back.
//  * ADC samples: each warp stages the (mx, my) of its 32 spins for 8 samples in shared memory, then contracts
//    them with the spins' coil sensitivities (paired FMAs over the 32 spins per lane: a small matrix product)
//    into its own slice of the window accumulator in shared memory, summed over all of the CTA's tiles. At the
//    window's end the warps' slices are added in fixed order and the CTA's partial is added to the float64 signal
//    with one float64 atomic per (sample, coil, re/im): the cross-block sum is float64 (float32 partials added in
//    float64 are exact in practice, so the result does not depend on the CTAs' order), and the CTA-level sum
//    covers thousands of spins, so the number of atomics does not grow with the spin count.
//  * Readout runs (samples with one segment's factors): the samples come from a float32 recurrence, the state
//    after the run from the float64 merged factors (see bloch_common.cuh), within blocks of BP_ADJ_WIN segments.
//  * Demodulation by exp(-i adc_phase) is the same for every spin and is applied after the sum, in float64
//    (bp_signal_finish).
#include <cuda_runtime.h>

#include <cstdint>

#include "bloch_common.cuh"
#include "physics.cuh"
#include "../../include/blochparty_b200.h"

#define BP_THREADS 128
#define BP_WARPS (BP_THREADS / 32)
#define BP_ACC_SAMPLES 64  // accumulator capacity in samples at 8 coils (one coil group)
#define BP_STAGE 8         // samples staged per warp before they are contracted
#define BP_MB_STRIDE 33    // float2 per staged sample row (32 spins + 1: conflict-free column reads)

// A readout run through the nonuniform FFT (bp_forward_nufft): per spin, the run's samples are z1 q^p (p < L,
// z1 the first sample, q the segment's complex factor), a sum over spins of exp(-2 pi i x p) times a decay; the
// spins spread their weight onto an oversampled grid of G cells (kernel of W cells, exp(beta (sqrt(1 - z^2) - 1)))
// once per term m of the decay's time segmentation (exp(-p dt r2) ~ sum_m a_m(p) exp(-tau_m r2)), and
// bp_nufft_finish turns the grid into the samples. The spins are sorted by x on the host, so a CTA's tiles cover
// a few neighbouring cells.
struct NufArgs {
    const int* run_of;       // [n_windows]: the run a window holds, or -1 (a window of the plain readout)
    const int* base;         // [n]: the spin's first grid cell (floor(x G) - W/2 + 1; may be below 0)
    const float* frac;       // [n]: x G - floor(x G)
    const float2* shift;     // [n]: exp(-2 pi i x floor(L / 2)) (the centred modes' phase)
    const float* decay;      // [M][n]: exp(-tau_m r2)
    const int2* tile_cells;  // [n_tiles]: the cells [lo, hi) the tile's spins reach
    double* grid;            // [runs][G][M][2C] float64, accumulated
    int G, W, M;
    float beta;
};

struct FwdArgs {
    const float* spins;   // [8][n]: px py pz pd r1 r2 db0 b1
    const float* sens;    // [16 ncg][n]: coil c real at row 2c, imaginary at 2c + 1, zero rows to pad
    const SegRec* segs;   // [S]
    const double4* seg64; // [S]: kx ky kz beta in float64
    const int4* windows;  // [n_windows]: first segment, end segment, first ADC row, samples
    int n, n_coils;
    int w_begin, w_end;
    float* state;         // [6][n]: mx my mz and their low parts
    double* raw;          // [n_adc][2C] raw coil sums (float64 atomics), or null: no readout
    float* wstates;       // null, or [(w_end - w_begin) / stride rounded up][6][n]: state at window starts
    int wstate_stride;
    const int* wslot;     // null, or [n_windows]: the slot of wstates that takes window w's start state (-1: none)
    int* status;
    NufArgs nu;           // NUFFT readout runs (bp_forward_nufft only)
    PhysArgs ph;          // the bound pool and the field model (bp_forward_physics only)
};

template <int NCG>
__host__ __device__ constexpr int samp_max() {
    return BP_ACC_SAMPLES / NCG;
}

// The warp's staged samples (mb: [BP_STAGE][BP_MB_STRIDE] (mx, my) of its 32 spins) contracted with the coil
// sensitivities of those spins (st: [32][16 NCG], coils 2q and 2q + 1 of a group at 4q as (re, re', im, im')) and
// added to the warp's accumulator rows acc[row0 + s] (coil c real at 2c, imaginary at 2c + 1). Lane l computes
// sample l & 7, coils 2 (l >> 3) and 2 (l >> 3) + 1 of every coil group, over the 32 spins on paired FMAs (two
// float32 FMAs per instruction, each rounded as one FMA): a = sum mx (re, re'), b = sum my (im, im'),
// c = sum mx (im, im'), d = sum my (re, re'), so that the real parts are a - b and the imaginary ones c + d (the
// coil sum as a small matrix product, no shuffles). Reads are conflict-free: the 8 samples' rows start 33 float2
// apart, and every lane of a sample reads the same spin's sensitivities (a broadcast of 4 float4s).
template <int NCG>
__device__ __forceinline__ void warp_contract(const float2* mb, const float* st, int nslot, float* acc, int row0,
                                              int lane) {
    constexpr int VG = 16 * NCG;
    const int smp = lane & 7, quarter = lane >> 3;
    if (smp >= nslot) return;
    const float2* row = mb + smp * BP_MB_STRIDE;
#pragma unroll
    for (int g = 0; g < NCG; ++g) {
        float2 sa = make_float2(0.f, 0.f), sb = sa, sc = sa, sd = sa;
#pragma unroll 8
        for (int j = 0; j < 32; ++j) {
            const float2 m = row[j];
            const float4 s4 = *reinterpret_cast<const float4*>(st + j * VG + 16 * g + 4 * quarter);
            const float2 re = make_float2(s4.x, s4.y), im = make_float2(s4.z, s4.w);
            const float2 xx = make_float2(m.x, m.x), yy = make_float2(m.y, m.y);
            sa = __ffma2_rn(xx, re, sa);
            sb = __ffma2_rn(yy, im, sb);
            sc = __ffma2_rn(xx, im, sc);
            sd = __ffma2_rn(yy, re, sd);
        }
        float4* dst = reinterpret_cast<float4*>(acc + (row0 + smp) * VG + 16 * g + 4 * quarter);
        float4 d = *dst;
        d.x += sa.x - sb.x, d.y += sc.x + sd.x, d.z += sa.y - sb.y, d.w += sc.y + sd.y;
        *dst = d;
    }
}

// The CTA's NUFFT accumulator rows [0, nrows) (row = (cell - cbase) M + term), summed over the warps' slices in
// fixed order and added to run `run`'s grid with one float64 atomic per value (cells taken modulo G); slots are
// cleared as read. Called by every thread of the CTA between barriers.
template <int NCG>
__device__ __forceinline__ void nuf_flush(const FwdArgs& a, float* acc, int run, int cbase, int nrows, int tid) {
    constexpr int VG = 16 * NCG;
    const int nv = 2 * a.n_coils, M = a.nu.M, G = a.nu.G;
    for (int k = tid; k < nrows * nv; k += BP_THREADS) {
        const int r = k / nv, v = k % nv;
        const int slot = r * VG + v;
        float t = 0.0f;
#pragma unroll
        for (int ww = 0; ww < BP_WARPS; ++ww) {
            t += acc[ww * samp_max<NCG>() * VG + slot];
            acc[ww * samp_max<NCG>() * VG + slot] = 0.0f;
        }
        const int cell = ((cbase + r / M) % G + G) % G, m = r % M;
        atomicAdd(a.nu.grid + (((size_t)run * G + cell) * M + m) * nv + v, (double)t);
    }
}

template <int NCG>
__host__ __device__ constexpr size_t fwd_smem_bytes_t() {
    return 2 * BP_SEG_MAX * sizeof(SegRec)                                   // segment blocks
           + (size_t)BP_WARPS * samp_max<NCG>() * 16 * NCG * sizeof(float)   // window accumulators, one per warp
           + (size_t)BP_WARPS * BP_STAGE * BP_MB_STRIDE * sizeof(float2)     // staged samples
           + (size_t)BP_WARPS * 32 * 16 * NCG * sizeof(float)                // coil sensitivities of the tile
           + 2 * sizeof(uint64_t);
}

// PHYS: the physics variant (bp_forward_physics): every RF segment through the bound pool's step and/or with the
// concomitant field in its offset, the free segments' phase with the concomitant phase and their longitudinal part
// through the exchange step; the rest (windows, readout runs, the coil contraction) as the plain kernel.
template <int NCG, bool NUF, bool PHYS = false>
__global__ void __launch_bounds__(BP_THREADS, NCG == 1 ? 5 : 4) bp_forward_kernel(FwdArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int VG = 16 * NCG;  // accumulator values per sample (coil groups of 8, padded)
    SegRec* segbuf = reinterpret_cast<SegRec*>(smem_raw);                                   // [2][BP_SEG_MAX]
    float* acc = reinterpret_cast<float*>(segbuf + 2 * BP_SEG_MAX);                         // [W][samp][VG]
    float2* mball = reinterpret_cast<float2*>(acc + BP_WARPS * samp_max<NCG>() * VG);       // [W][16][33]
    float* stall = reinterpret_cast<float*>(mball + BP_WARPS * BP_STAGE * BP_MB_STRIDE);    // [W][32][VG]
    uint64_t* bars = reinterpret_cast<uint64_t*>(stall + BP_WARPS * 32 * VG);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = a.n;
    const int n_tiles = (n + BP_THREADS - 1) / BP_THREADS;
    const int nv = 2 * a.n_coils;
    float* my_acc = acc + warp * samp_max<NCG>() * VG;
    float2* mb = mball + warp * BP_STAGE * BP_MB_STRIDE;
    float* st = stall + warp * 32 * VG;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    for (int i = tid; i < BP_WARPS * samp_max<NCG>() * VG; i += BP_THREADS) acc[i] = 0.0f;
    __syncthreads();

    auto issue = [&](int w, int buf) {
        const int4 win = a.windows[w];
        if (!window_ok(win, samp_max<NCG>())) {  // never copy what does not fit: complete the phase without data
            atomicOr(a.status, BP_ERR_BAD_WINDOW);
            mbar_arrive(&bars[buf]);
            return;
        }
        const uint32_t bytes = static_cast<uint32_t>(win.y - win.x) * sizeof(SegRec);
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[buf], bytes);
        tma_load_1d(segbuf + buf * BP_SEG_MAX, a.segs + win.x, bytes, &bars[buf]);
    };
    if (tid == 0) issue(a.w_begin, 0);

    for (int w = a.w_begin; w < a.w_end; ++w) {
        const int i = w - a.w_begin, buf = i & 1;
        const bool ok = mbar_wait_bounded(&bars[buf], (i >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(a.status, BP_ERR_TMA_TIMEOUT);
            return;
        }
        const int4 win = a.windows[w];
        if (!window_ok(win, samp_max<NCG>())) return;  // uniform; the status bit was set where it was staged
        if (tid == 0 && w + 1 < a.w_end) issue(w + 1, buf ^ 1);  // after the check: nothing left in flight
        const SegRec* q0 = segbuf + buf * BP_SEG_MAX;
        const int nseg = win.y - win.x;
        const int nrun = NUF ? a.nu.run_of[w] : -1;  // a NUFFT readout run (the same for the whole CTA)
        const bool readout = a.raw != nullptr && (win.w > 0 || nrun >= 0);
        // the wstates slot that takes this window's start state, or -1
        const int wsl = a.wstates == nullptr                ? -1
                        : a.wslot                           ? a.wslot[w]
                        : (i % a.wstate_stride) == 0 ? i / a.wstate_stride
                                                            : -1;
        const bool save = wsl >= 0;
        // the CTA's tiles: every grid-th tile from its own (measured fastest: 3.07 s against 3.18 s for even
        // contiguous blocks and 3.29 s for blocks of the ceiling on the 1 M-spin GRE, equal to the ceiling's on the
        // 8.4 M-spin head); the NUFFT kernel takes one contiguous block of floor(n_tiles / grid) or one more tiles
        // (the runs' spins are sorted, so a block covers few grid cells)
        const int t_begin = NUF ? (int)((long long)blockIdx.x * n_tiles / gridDim.x) : (int)blockIdx.x;
        const int t_end = NUF ? (int)((long long)(blockIdx.x + 1) * n_tiles / gridDim.x) : n_tiles;
        const int t_step = NUF ? 1 : (int)gridDim.x;
        int cbase = 0, chi = 0;  // NUFFT: the cells the accumulator holds, [cbase, chi) so far
        if (NUF && nrun >= 0 && t_begin < t_end) cbase = chi = a.nu.tile_cells[t_begin].x;

        for (int tile = t_begin; tile < t_end; tile += t_step) {
            if (NUF && nrun >= 0) {
                // the tile's cells must fit the accumulator's rows from cbase: if not, add what it holds to the
                // grid and restart it at this tile (uniform: every warp of the CTA runs the same tiles)
                const int2 tc = a.nu.tile_cells[tile];
                if ((tc.y - cbase) * a.nu.M > samp_max<NCG>()) {
                    __syncthreads();
                    nuf_flush<NCG>(a, acc, nrun, cbase, (chi - cbase) * a.nu.M, tid);
                    __syncthreads();
                    cbase = chi = tc.x;
                }
                chi = max(chi, tc.y);
            }
            const int j0 = tile * BP_THREADS + tid;
            const bool active = j0 < n;
            const int j = active ? j0 : 0;
            const Spin p = load_spin(a.spins, n, j, active);
            float mx = 0.f, my = 0.f, mz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
            // physics variant: the bound pool (inactive lanes read spin 0's, with pd 0: finite, never summed), its
            // state, and the concomitant coefficients
            Pool pb{0.f, 0.f, 1.f, 1.f, 0.f};
            Conc ck{};
            float zb = 0.f, zbl = 0.f, e2h = 0.f;  // the bound pool's Mz (hi, lo)
            if constexpr (PHYS) {
                if (a.ph.mt) {
                    pb = load_pool(a.ph.pool, n, j);
                    if (active) zb = a.ph.bstate[j], zbl = a.ph.bstate[n + j];
                }
                ck = load_conc(a.ph.conc, n, j, a.ph.conc_mode);
            }
            if (active) {
                mx = a.state[j];
                my = a.state[n + j];
                mz = a.state[2 * n + j];
                lx = a.state[3 * n + j];
                ly = a.state[4 * n + j];
                lz = a.state[5 * n + j];
                if (save) {
                    float* ws = a.wstates + (size_t)wsl * 6 * n;
                    ws[j] = mx, ws[n + j] = my, ws[2 * n + j] = mz;
                    ws[3 * n + j] = lx, ws[4 * n + j] = ly, ws[5 * n + j] = lz;
                }
            }
            if (readout) {  // this spin's coil sensitivities into the warp's tile (inactive lanes: zeros), a pair of
                            // coils as (re, re', im, im')
#pragma unroll
                for (int k = 0; k < VG; k += 4) {
                    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (active) v = make_float4(a.sens[k * n + j], a.sens[(k + 2) * n + j], a.sens[(k + 1) * n + j],
                                                a.sens[(k + 3) * n + j]);
                    *reinterpret_cast<float4*>(st + lane * VG + k) = v;
                }
                __syncwarp();
            }
            FreeFactors ff{1.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            RfRelax rr{1.f, 1.f, 0.f, 0.f, 0.f, 0.f};
            float wz = 0.0f;
            int slot = 0, row0 = 0;
            auto stage = [&](float x, float y) {
                mb[slot * BP_MB_STRIDE + lane] = make_float2(x, y);
                if (++slot == BP_STAGE) {
                    __syncwarp();
                    warp_contract<NCG>(mb, st, BP_STAGE, my_acc, row0, lane);
                    __syncwarp();
                    row0 += BP_STAGE;
                    slot = 0;
                }
            };
            if (NUF && nrun >= 0) {
                // the run's first sample z1 = z q, centred by the shift, spread onto the warp's cells for every
                // decay term: the accumulator rows are (cell - cbase) M + m, one staged column per (cell, term),
                // zero where this spin's kernel does not reach
                const SegRec q = q0[0];
                const double4 k64 = a.seg64[win.x];
                ff = free_factors(q, k64, p);
                float zr = mx + lx, zi = my + ly;
                readout_advance(ff, zr, zi);
                const float2 sh = active ? a.nu.shift[j] : make_float2(0.f, 0.f);
                const float w0r = zr * sh.x - zi * sh.y, w0i = zr * sh.y + zi * sh.x;
                const int b = active ? a.nu.base[j] : 0;
                const float fr = active ? a.nu.frac[j] : 0.f;
                const int M = a.nu.M, W = a.nu.W;
                float dec[BP_NUF_MAX_TERMS];
#pragma unroll
                for (int m = 0; m < BP_NUF_MAX_TERMS; ++m) dec[m] = (active && m < M) ? a.nu.decay[(size_t)m * n + j] : 0.f;
                const int wlo = __reduce_min_sync(0xffffffffu, active ? b : 0x7fffffff);
                const int whi = __reduce_max_sync(0xffffffffu, active ? b : -0x7fffffff);
                if (wlo <= whi) {  // (uniform in the warp) some lane is a spin
                    row0 = (wlo - cbase) * M;
                    const float zs = 2.0f / (float)W, half = (float)(W / 2 - 1);
                    for (int c = 0; c < whi - wlo + W; ++c) {
                        const int wi = wlo + c - b;
                        float psi = 0.0f;
                        if (active && wi >= 0 && wi < W) {
                            const float z = zs * ((float)wi - half - fr);
                            psi = expf(a.nu.beta * (sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f))) - 1.0f));
                        }
                        const float vr = w0r * psi, vi = w0i * psi;
#pragma unroll
                        for (int m = 0; m < BP_NUF_MAX_TERMS; ++m)
                            if (m < M) stage(vr * dec[m], vi * dec[m]);
                    }
                }
                // the state after the run: the segment's factors merged over its nseg copies (exact phase)
                const FreeFactors fm = free_factors_merged(q, k64, p, nseg);
                free_step(fm, p, mx, my, mz, lx, ly, lz);
                if (q0[nseg - 1].flags & BP_SPOIL) mx = my = lx = ly = 0.0f;
            }
            for (int s = 0; s < ((NUF && nrun >= 0) ? 0 : nseg); ++s) {
                const SegRec q = q0[s];
                const int f = q.flags;
                if constexpr (PHYS) {
                    if (f & BP_RF) {  // every RF segment alone: the bound pool's step, or the plain one
                        if (s == 0 || !(f & BP_SAME_RFDT)) {
                            rr = rf_relax(q.dt, p);
                            e2h = expm1f(-0.5f * q.dt * p.r2);
                        }
                        if (s == 0 || !(f & BP_SAME_OFF))
                            wz = phys_wz(q, p, a.ph.conc_mode, ck, a.ph.segq + 6 * (size_t)(win.x + s));
                        if (a.ph.mt)
                            rf_step_mt(q, p, pb, e2h, wz, a.ph.rf_freq[win.x + s], a.ph.line, mx, my, mz, lx, ly, lz,
                                       zb, zbl);
                        else
                            rf_step_wz(q, p, rr, wz, mx, my, mz, lx, ly, lz);
                        if ((f & BP_ADC) && readout) stage(mx + lx, my + ly);
                        if (f & BP_SPOIL) mx = my = lx = ly = 0.0f;
                        continue;
                    }
                }
                if (f & BP_RF) {
                    if (s == 0 || !(f & BP_SAME_RFDT)) rr = rf_relax(q.dt, p);
                    if (s == 0 || !(f & BP_SAME_OFF)) wz = rf_wz(q, p);
                    rf_step_wz(q, p, rr, wz, mx, my, mz, lx, ly, lz);
                    if (!(f & (BP_ADC | BP_SPOIL))) {
                        // the rest of a pulse with this dt and offset: only the RF changes from step to step
                        constexpr int kRun = BP_RF | BP_SAME_RFDT | BP_SAME_OFF;
                        if (f & BP_SMALL) {  // (the run's small steps without the factors' tier tests)
                            constexpr int kSmall = kRun | BP_SMALL;
                            while (s + 1 < nseg) {
                                const SegRec& qn = q0[s + 1];
                                if ((qn.flags & (kSmall | BP_ADC | BP_SPOIL)) != kSmall) break;
                                ++s;
                                rf_step_wz<true>(qn, p, rr, wz, mx, my, mz, lx, ly, lz);
                            }
                        }
                        while (s + 1 < nseg) {
                            const SegRec& qn = q0[s + 1];
                            if ((qn.flags & (kRun | BP_ADC | BP_SPOIL)) != kRun) break;
                            ++s;
                            rf_step_wz(qn, p, rr, wz, mx, my, mz, lx, ly, lz);
                        }
                        continue;
                    }
                } else {
                    if (s == 0 || !(f & BP_SAME_FREE)) {
                        if constexpr (PHYS)
                            ff = free_factors_phys(q, a.seg64[win.x + s], p, 1, a.ph.conc_mode, ck,
                                                   a.ph.segq + 6 * (size_t)(win.x + s));
                        else
                            ff = free_factors(q, a.seg64[win.x + s], p);
                    }
                    if (PHYS && a.ph.mt)
                        free_step_mt(ff, zstep(q.dt, p, pb, 0.0f), mx, my, mz, lx, ly, lz, zb, zbl);
                    else
                        free_step(ff, p, mx, my, mz, lx, ly, lz);
                    if ((f & (BP_ADC | BP_SPOIL)) == BP_ADC) {
                        // a readout run: the following samples with this segment's factors (the last may spoil),
                        // within this window and this block of BP_ADJ_WIN segments (so that the runs are cut at
                        // the same segments whatever the window plan). Their values come from a float32
                        // recurrence; the state after the run is this one advanced by the merged factors (exact
                        // phase in float64), as if stepped one by one.
                        const int block_end = min(nseg, (win.x + s) / BP_ADJ_WIN * BP_ADJ_WIN + BP_ADJ_WIN - win.x);
                        // the run's end, from one flag per lane (the candidates s + 1 + lane, at most 31 before the
                        // block's end): the samples that continue the run, up to the first that does not, or
                        // through the first that spoils. Then a tight loop over its samples.
                        const int ec = s + 1 + lane;
                        const int fc = ec < block_end ? q0[ec].flags : 0;
                        const unsigned cont = __ballot_sync(0xffffffffu, ec < block_end &&
                                                                          (fc & ~BP_SPOIL) == (BP_ADC | BP_SAME_FREE));
                        const unsigned spoils = cont & __ballot_sync(0xffffffffu, (fc & BP_SPOIL) != 0);
                        int len = __ffs(~cont) - 1;  // leading continuing samples (cont != ~0: lane 31 is past the block)
                        const unsigned sp = spoils & ((1u << len) - 1u);
                        if (sp) len = __ffs(sp);     // through the first spoiling one
                        const int e = s + 1 + len;
                        if (readout) {
                            float zr = mx + lx, zi = my + ly;
                            stage(zr, zi);
                            for (int t = s + 1; t < e; ++t) {
                                readout_advance(ff, zr, zi);
                                stage(zr, zi);
                            }
                        }
                        if (e > s + 1) {
                            if constexpr (PHYS) {
                                const FreeFactors fr = free_factors_phys(q, a.seg64[win.x + s], p, e - s - 1,
                                                                         a.ph.conc_mode, ck,
                                                                         a.ph.segq + 6 * (size_t)(win.x + s));
                                if (a.ph.mt)
                                    free_step_mt(fr, zstep((float)((double)q.dt * (double)(e - s - 1)), p, pb, 0.0f),
                                                 mx, my, mz, lx, ly, lz, zb, zbl);
                                else
                                    free_step(fr, p, mx, my, mz, lx, ly, lz);
                            } else {
                                const FreeFactors fr = free_factors_merged(q, a.seg64[win.x + s], p, e - s - 1);
                                free_step(fr, p, mx, my, mz, lx, ly, lz);
                            }
                            if (q0[e - 1].flags & BP_SPOIL) mx = my = lx = ly = 0.0f;
                        }
                        s = e - 1;
                        continue;
                    }
                }
                if (f & (BP_ADC | BP_SPOIL)) {
                    if ((f & BP_ADC) && readout) stage(mx + lx, my + ly);
                    if (f & BP_SPOIL) mx = my = lx = ly = 0.0f;
                }
            }
            if (slot > 0) {
                __syncwarp();
                warp_contract<NCG>(mb, st, slot, my_acc, row0, lane);
                __syncwarp();
            }
            if (active) {
                a.state[j] = mx;
                a.state[n + j] = my;
                a.state[2 * n + j] = mz;
                a.state[3 * n + j] = lx;
                a.state[4 * n + j] = ly;
                a.state[5 * n + j] = lz;
                if (PHYS && a.ph.mt) a.ph.bstate[j] = zb, a.ph.bstate[n + j] = zbl;
            }
        }
        __syncthreads();
        if (NUF && nrun >= 0 && readout) {
            nuf_flush<NCG>(a, acc, nrun, cbase, (chi - cbase) * a.nu.M, tid);
            __syncthreads();
        } else if (readout) {
            // the warps' slices in fixed order (the CTA's sum does not depend on timing), then one float64 atomic
            // per value; slots are cleared as read
            for (int k = tid; k < win.w * nv; k += BP_THREADS) {
                const int r = k / nv, v = k % nv;
                const int slot = r * VG + v;
                float t = 0.0f;
#pragma unroll
                for (int ww = 0; ww < BP_WARPS; ++ww) {
                    t += acc[ww * samp_max<NCG>() * VG + slot];
                    acc[ww * samp_max<NCG>() * VG + slot] = 0.0f;
                }
                atomicAdd(a.raw + (size_t)(win.z + r) * nv + v, (double)t);
            }
            __syncthreads();
        }
    }
}

// ---- float64 demodulation of the summed signal: out[c][t] = raw[t][c] exp(-i psi[t]) as complex64 ----
__global__ void bp_signal_finish_kernel(const double* __restrict__ raw, const double* __restrict__ psi, int n_adc,
                                        int n_coils, float2* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)n_adc * n_coils) return;
    const int t = (int)(k % n_adc), c = (int)(k / n_adc);
    const double re = raw[(size_t)t * 2 * n_coils + 2 * c], im = raw[(size_t)t * 2 * n_coils + 2 * c + 1];
    double s, co;
    sincos(psi[t], &s, &co);
    out[k] = make_float2((float)(re * co + im * s), (float)(im * co - re * s));
}

// ---- launch helpers ----
template <int NCG>
static size_t fwd_smem_bytes() {
    return fwd_smem_bytes_t<NCG>();
}

static int g_num_sms[64];

static int num_sms(int dev) {
    if (dev < 0 || dev >= 64) return 148;
    if (!g_num_sms[dev]) cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    return g_num_sms[dev];
}

template <int NCG, bool NUF, bool PHYS = false>
static int forward_grid(int n, int max_ctas, int* grid_out) {
    const size_t smem = fwd_smem_bytes<NCG>();
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_forward_kernel<NCG, NUF, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(bp_forward_kernel<NCG, NUF, PHYS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return BP_E_LAUNCH;
        configured[dev] = true;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_forward_kernel<NCG, NUF, PHYS>, BP_THREADS, smem) !=
        cudaSuccess)
        return BP_E_LAUNCH;
    if (per_sm < 1) per_sm = 1;
    const int n_tiles = (n + BP_THREADS - 1) / BP_THREADS;
    int grid = num_sms(dev) * per_sm;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > n_tiles) grid = n_tiles;
    if (grid < 1) grid = 1;
    *grid_out = grid;
    return BP_OK;
}

template <int NCG, bool NUF, bool PHYS = false>
static int launch_forward(const FwdArgs& a, int max_ctas, cudaStream_t stream) {
    int grid = 0;
    const int code = forward_grid<NCG, NUF, PHYS>(a.n, max_ctas, &grid);
    if (code != BP_OK) return code;
    bp_forward_kernel<NCG, NUF, PHYS><<<grid, BP_THREADS, fwd_smem_bytes<NCG>(), stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

extern "C" int bp_forward_grid(int n, int n_coils) {
    if (n < 1 || n_coils < 1 || n_coils > BP_MAX_COILS) return -BP_E_ARG;
    int grid = 0, code = BP_OK;
    switch ((n_coils + 7) / 8) {
        case 1: code = forward_grid<1, false>(n, 0, &grid); break;
        case 2: code = forward_grid<2, false>(n, 0, &grid); break;
        case 3: code = forward_grid<3, false>(n, 0, &grid); break;
        default: code = forward_grid<4, false>(n, 0, &grid); break;
    }
    return code == BP_OK ? grid : -code;
}

extern "C" int bp_forward_samp_max(int n_coils) {
    if (n_coils < 1 || n_coils > BP_MAX_COILS) return 0;
    const int ncg = (n_coils + 7) / 8;
    switch (ncg) {
        case 1: return samp_max<1>();
        case 2: return samp_max<2>();
        case 3: return samp_max<3>();
        default: return samp_max<4>();
    }
}

static int fill_args(FwdArgs& a, const float* spins, const float* sens, int n, int n_coils, const void* segs,
                     const double* seg64, const int* windows, int w_begin, int w_end, float* state, double* raw,
                     float* wstates, int wstate_stride, int* status) {
    if (n < 1 || n_coils < 1 || n_coils > BP_MAX_COILS || w_begin < 0 || w_end < w_begin) return BP_E_ARG;
    if (!spins || !segs || !seg64 || !windows || !state || !status) return BP_E_ARG;
    if (raw && !sens) return BP_E_ARG;
    if (wstates && wstate_stride < 1) return BP_E_ARG;
    if ((reinterpret_cast<uintptr_t>(segs) & 15) != 0) return BP_E_ALIGN;
    a = FwdArgs{};
    a.spins = spins;
    a.sens = sens;
    a.segs = static_cast<const SegRec*>(segs);
    a.seg64 = reinterpret_cast<const double4*>(seg64);
    a.windows = reinterpret_cast<const int4*>(windows);
    a.n = n;
    a.n_coils = n_coils;
    a.w_begin = w_begin;
    a.w_end = w_end;
    a.state = state;
    a.raw = raw;
    a.wstates = wstates;
    a.wstate_stride = wstate_stride > 0 ? wstate_stride : 1;
    a.status = status;
    return BP_OK;
}

extern "C" int bp_forward(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                          const double* seg64, const int* windows, int w_begin, int w_end, float* state, double* raw,
                          float* wstates, int wstate_stride, int max_ctas, int* status, void* stream) {
    FwdArgs a;
    const int code = fill_args(a, spins, sens, n, n_coils, segs, seg64, windows, w_begin, w_end, state, raw, wstates,
                               wstate_stride, status);
    if (code != BP_OK || w_end == w_begin) return code;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch ((n_coils + 7) / 8) {
        case 1: return launch_forward<1, false>(a, max_ctas, st);
        case 2: return launch_forward<2, false>(a, max_ctas, st);
        case 3: return launch_forward<3, false>(a, max_ctas, st);
        default: return launch_forward<4, false>(a, max_ctas, st);
    }
}

extern "C" int bp_forward_saving(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                 const double* seg64, const int* windows, int w_begin, int w_end, float* state,
                                 double* raw, const int* wslot, float* wstates, int max_ctas, int* status,
                                 void* stream) {
    if (!wslot || !wstates) return BP_E_ARG;
    FwdArgs a;
    const int code = fill_args(a, spins, sens, n, n_coils, segs, seg64, windows, w_begin, w_end, state, raw, wstates,
                               1, status);
    if (code != BP_OK || w_end == w_begin) return code;
    a.wslot = wslot;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch ((n_coils + 7) / 8) {
        case 1: return launch_forward<1, false>(a, max_ctas, st);
        case 2: return launch_forward<2, false>(a, max_ctas, st);
        case 3: return launch_forward<3, false>(a, max_ctas, st);
        default: return launch_forward<4, false>(a, max_ctas, st);
    }
}

extern "C" int bp_forward_nufft(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                const double* seg64, const int* windows, int w_begin, int w_end, float* state,
                                double* raw, int max_ctas, const BpNufft* nu, int* status, void* stream) {
    FwdArgs a;
    const int code = fill_args(a, spins, sens, n, n_coils, segs, seg64, windows, w_begin, w_end, state, raw, nullptr,
                               1, status);
    if (code != BP_OK) return code;
    if (!nu || !raw || !nu->run_of || !nu->base || !nu->frac || !nu->shift || !nu->decay || !nu->tile_cells ||
        !nu->grid || nu->G < 2 || nu->W < 2 || nu->W > nu->G || nu->M < 1 || nu->M > BP_NUF_MAX_TERMS ||
        (reinterpret_cast<uintptr_t>(nu->shift) & 7) != 0 || (reinterpret_cast<uintptr_t>(nu->tile_cells) & 7) != 0)
        return BP_E_ARG;
    const int ncg = (n_coils + 7) / 8;
    // a tile's cells (its spins' kernels: at most W + 1 cells for sorted spins, checked on the host) x terms must
    // fit the accumulator
    if (ncg > 2 || (nu->W + 1) * nu->M > BP_ACC_SAMPLES / ncg) return BP_E_SIZE;
    if (w_end == w_begin) return BP_OK;
    a.nu.run_of = nu->run_of;
    a.nu.base = nu->base;
    a.nu.frac = nu->frac;
    a.nu.shift = static_cast<const float2*>(nu->shift);
    a.nu.decay = nu->decay;
    a.nu.tile_cells = reinterpret_cast<const int2*>(nu->tile_cells);
    a.nu.grid = nu->grid;
    a.nu.G = nu->G, a.nu.W = nu->W, a.nu.M = nu->M;
    a.nu.beta = nu->beta;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return ncg == 1 ? launch_forward<1, true>(a, max_ctas, st) : launch_forward<2, true>(a, max_ctas, st);
}

extern "C" int bp_forward_physics(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                  const double* seg64, const int* windows, int w_begin, int w_end, float* state,
                                  double* raw, int max_ctas, const BpPhysics* ph, int* status, void* stream) {
    FwdArgs a;
    if (!ph) return BP_E_ARG;
    const int code = fill_args(a, spins, sens, n, n_coils, segs, seg64, windows, w_begin, w_end, state, raw,
                               ph->wstates, ph->wstate_stride, status);
    if (code != BP_OK) return code;
    if (ph->conc_mode < 0 || ph->conc_mode > 2 || (ph->wstates && ph->mt)) return BP_E_ARG;
    if (ph->mt && (!ph->pool || !ph->bstate || !ph->rf_freq || !ph->line)) return BP_E_ARG;
    if (ph->conc_mode && !ph->conc) return BP_E_ARG;
    if (ph->conc_mode == 1 && !ph->segq) return BP_E_ARG;
    if (w_end == w_begin) return BP_OK;
    a.ph.mt = ph->mt != 0;
    a.ph.conc_mode = ph->conc_mode;
    a.ph.pool = ph->pool;
    a.ph.bstate = ph->bstate;
    a.ph.rf_freq = ph->rf_freq;
    a.ph.line = ph->line;
    a.ph.conc = ph->conc;
    a.ph.segq = ph->segq;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch ((n_coils + 7) / 8) {
        case 1: return launch_forward<1, false, true>(a, max_ctas, st);
        case 2: return launch_forward<2, false, true>(a, max_ctas, st);
        case 3: return launch_forward<3, false, true>(a, max_ctas, st);
        default: return launch_forward<4, false, true>(a, max_ctas, st);
    }
}

// ---- NUFFT readout runs: grid -> samples (float64) ----
// Block (run r, coil c): the run's grid [G][M] (coil c, re/im) and the twiddles exp(-2 pi i t / G) in shared memory;
// thread p (< L) forms sum_m w[m][p] sum_g grid[g][m] exp(-2 pi i (p - L/2) g / G) and adds it to raw row
// rows[r] + p (rows only these runs own: no other launch writes them).
__global__ void bp_nufft_finish_kernel(const double* __restrict__ grid, const int* __restrict__ rows, int G, int M,
                                       int L, int n_coils, const double* __restrict__ w, double* __restrict__ raw) {
    extern __shared__ double smd[];
    double2* tw = reinterpret_cast<double2*>(smd);  // [G]
    double2* gm = tw + G;                            // [M][G]
    const int r = blockIdx.x, c = blockIdx.y, nv = 2 * n_coils, h = L / 2;
    for (int t = threadIdx.x; t < G; t += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)t / (double)G, &sn, &cs);
        tw[t] = make_double2(cs, -sn);
    }
    for (int k = threadIdx.x; k < G * M; k += blockDim.x) {
        const int g = k / M, m = k % M;
        const double* src = grid + (((size_t)r * G + g) * M + m) * nv + 2 * c;
        gm[m * G + g] = make_double2(src[0], src[1]);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < L; p += blockDim.x) {
        const int kap = p - h;
        const int step = ((kap % G) + G) % G;
        double orr = 0.0, oi = 0.0;
        for (int m = 0; m < M; ++m) {
            double sr = 0.0, si = 0.0;
            int t = 0;
            for (int g = 0; g < G; ++g) {
                const double2 z = gm[m * G + g], e = tw[t];
                sr = fma(z.x, e.x, fma(-z.y, e.y, sr));
                si = fma(z.x, e.y, fma(z.y, e.x, si));
                t += step;
                if (t >= G) t -= G;
            }
            const double wm = w[(size_t)m * L + p];
            orr = fma(wm, sr, orr);
            oi = fma(wm, si, oi);
        }
        double* dst = raw + (size_t)(rows[r] + p) * nv + 2 * c;
        dst[0] += orr;
        dst[1] += oi;
    }
}

extern "C" int bp_nufft_finish(const double* grid, const int* run_rows, int n_runs, int G, int M, int L,
                               int n_coils, const double* weights, double* raw, void* stream) {
    if (n_runs < 0 || G < 2 || M < 1 || M > BP_NUF_MAX_TERMS || L < 1 || n_coils < 1 || n_coils > BP_MAX_COILS)
        return BP_E_ARG;
    if (n_runs == 0) return BP_OK;
    if (!grid || !run_rows || !weights || !raw) return BP_E_ARG;
    const size_t smem = (size_t)G * (M + 1) * sizeof(double2);
    if (smem > 200 * 1024) return BP_E_SIZE;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_nufft_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) !=
            cudaSuccess)
            return BP_E_LAUNCH;
        configured[dev] = true;
    }
    const dim3 blocks((unsigned)n_runs, (unsigned)n_coils);
    const int threads = L < 128 ? 128 : 256;
    bp_nufft_finish_kernel<<<blocks, threads, smem, static_cast<cudaStream_t>(stream)>>>(grid, run_rows, G, M, L,
                                                                                        n_coils, weights, raw);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

extern "C" int bp_signal_finish(const double* raw, const double* psi, int n_adc, int n_coils, void* out,
                                void* stream) {
    if (n_adc < 0 || n_coils < 1) return BP_E_ARG;
    if (n_adc == 0) return BP_OK;
    if (!raw || !psi || !out) return BP_E_ARG;
    const int64_t total = (int64_t)n_adc * n_coils;
    const int threads = 256;
    const int64_t blocks = (total + threads - 1) / threads;
    bp_signal_finish_kernel<<<(unsigned)blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        raw, psi, n_adc, n_coils, static_cast<float2*>(out));
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}
