// Forward propagation with the coil readout on the tensor cores (tcgen05, split bfloat16, float32 accumulation).
//
// The propagation (windows, persistent CTAs over 128-spin tiles, TMA-staged segment blocks, compensated float32
// state) is that of forward.cu. The readout differs: the coil sum of a block of 16 ADC samples over a tile's 128
// spins is one small matrix product on the tensor cores,
//     D[m][t] += sum_k A[m][k] B[t][k],   k = 2 j + {0, 1} (spin j's Mx, My),
// with A the tile's coil sensitivities (row m = 2c: (s_r, -s_i), row 2c + 1: (s_i, s_r) per spin, coil c) and B
// the 16 samples' magnetization. Both are split into bfloat16 high and low parts and D accumulates
// A_hi B_hi + A_hi B_lo + A_lo B_hi in float32 in tensor memory (the dropped A_lo B_lo is ~2^-18 relative).
// Shapes: tcgen05.mma kind::f16, M = 128 (the 2C <= 16 coil rows; rows 16..127 are not read back), N = 16
// samples, K = 256 per tile in 16 steps. D holds the window's (up to 64) samples, summed over all of the CTA's
// tiles; at the window's end warp 0 reads it (tcgen05.ld) and adds it to the float64 signal.
//
// Shared memory (bytes): A hi [0, 8192), A lo [8192, 16384) in the canonical K-major no-swizzle layout (core
// matrices of 8 rows x 16 bytes, K-adjacent core matrices 128 bytes apart, 8-row groups 4096 apart); B: two
// buffers x (hi, lo) of 9216 bytes each from 16384 (K-adjacent core matrices 144 bytes apart so that a warp's
// 4-byte writes of one sample hit 32 different banks, 8-row groups 4608 apart); segment blocks from 53248;
// mbarriers and the tensor-memory address from 73728. The descriptors of A's rows 16..127 address the memory
// after A's 16 rows (B, the segment blocks), so the allocation covers all 128 rows of both A parts (73,728
// bytes); the mbarriers sit after that span.
#include <cuda_runtime.h>

#include <cstdint>

#include "bloch_common.cuh"
#include "tcgen05.cuh"
#include "../../include/blochparty_b200.h"

#define MM_THREADS 128
#define MM_SAMPLES 64   // samples per window (D columns)
#define MM_BLOCK 16     // samples per MMA (N)
#define MM_A_BYTES 8192
#define MM_B_BYTES 9216
#define MM_A_SBO 4096
#define MM_A_LBO 128
#define MM_B_SBO 4608
#define MM_B_LBO 144
#define MM_OFF_B 16384
#define MM_OFF_SEG (MM_OFF_B + 4 * MM_B_BYTES)
#define MM_OFF_BAR 73728  // past the span that A's 128 rows address: mbarriers are touched by mbarrier ops only
#define MM_SMEM 73856
#define MM_TMEM_COLS 64

struct MmaArgs {
    const float* spins;
    const uint8_t* atiles;  // [n_tiles][2][8192]: the tiles' A hi and A lo in shared-memory layout
    const SegRec* segs;
    const double4* seg64;
    const int4* windows;
    int n, n_coils;
    int w_begin, w_end;
    float* state;
    double* raw;
    int* status;
};

// byte offset of element (row r, k) of a K-major operand with the given core-matrix strides
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int lbo, int sbo) {
    return (uint32_t)((r >> 3) * sbo + (k >> 3) * lbo + (r & 7) * 16 + (k & 7) * 2);
}

__global__ void __launch_bounds__(MM_THREADS, 3) bp_forward_mma_kernel(MmaArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    SegRec* segbuf = reinterpret_cast<SegRec*>(sm + MM_OFF_SEG);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + MM_OFF_BAR);  // [0,1] segment blocks, [2,3] MMA, [4] A tile
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + MM_OFF_BAR + 5 * sizeof(uint64_t));
    const int tid = threadIdx.x, warp = tid >> 5;
    const int n = a.n, n_tiles = (n + MM_THREADS - 1) / MM_THREADS;
    const int nv = 2 * a.n_coils;
    const uint32_t sA = smem_u32(sm), sB = smem_u32(sm + MM_OFF_B);
    const uint32_t idesc = umma_idesc_bf16_f32(128, MM_BLOCK);

    if (tid == 0) {
        for (int b = 0; b < 5; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, MM_TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // mbarrier phases, tracked identically by every thread
    uint32_t mma_phase[2] = {0u, 0u}, a_phase = 0u;
    bool mma_pending[2] = {false, false};
    bool fail = false, err = false;  // fail: leave the window loop; err: this thread saw a failed wait
    auto drain = [&](int b) -> bool {  // wait for the MMAs that read B buffer b (and A) to complete
        if (!mma_pending[b]) return true;
        const bool ok = mbar_wait_bounded(&bars[2 + b], mma_phase[b]);
        mma_phase[b] ^= 1u;
        mma_pending[b] = false;
        return ok;
    };
    auto issue_seg = [&](int w, int buf) {
        const int4 win = a.windows[w];
        if (!window_ok(win, MM_SAMPLES)) {  // never copy what does not fit: complete the phase without data
            atomicOr(a.status, BP_ERR_BAD_WINDOW);
            mbar_arrive(&bars[buf]);
            return;
        }
        const uint32_t bytes = static_cast<uint32_t>(win.y - win.x) * sizeof(SegRec);
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[buf], bytes);
        tma_load_1d(segbuf + buf * BP_SEG_MAX, a.segs + win.x, bytes, &bars[buf]);
    };
    int seg_pending = a.w_begin;  // window whose segment block is in flight (-1: none)
    if (tid == 0) issue_seg(a.w_begin, 0);

    for (int w = a.w_begin; w < a.w_end && !fail; ++w) {
        const int i = w - a.w_begin, sbuf = i & 1;
        const bool ok = mbar_wait_bounded(&bars[sbuf], (i >> 1) & 1);
        seg_pending = -1;
        if (__syncthreads_or(!ok)) {
            fail = true;
            break;
        }
        const int4 win = a.windows[w];
        if (!window_ok(win, MM_SAMPLES)) {  // uniform: every thread reads the same record
            fail = true;
            break;
        }
        if (w + 1 < a.w_end) {  // after the check: nothing left in flight on that path
            if (tid == 0) issue_seg(w + 1, sbuf ^ 1);
            seg_pending = w + 1;
        }
        const SegRec* q0 = segbuf + sbuf * BP_SEG_MAX;
        const int nseg = win.y - win.x;
        const bool readout = a.raw != nullptr && win.w > 0;
        bool first_tile = true;

        for (int tile = blockIdx.x; tile < n_tiles && !fail; tile += gridDim.x) {
            // the previous tile's MMAs read A: let them finish, then bring this tile's A in
            bool okd = drain(0);
            okd = drain(1) && okd;
            if (__syncthreads_or(!okd || err)) {
                fail = true;
                break;
            }
            if (readout && tid == 0) {
                fence_proxy_async_smem();
                mbar_expect_tx(&bars[4], 2 * MM_A_BYTES);
                tma_load_1d(sm, a.atiles + (size_t)tile * 2 * MM_A_BYTES, 2 * MM_A_BYTES, &bars[4]);
            }
            bool a_waited = false;
            const int j0 = tile * MM_THREADS + tid;
            const bool active = j0 < n;
            const int j = active ? j0 : 0;
            const Spin p = load_spin(a.spins, n, j, active);
            float mx = 0.f, my = 0.f, mz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
            if (active) {
                mx = a.state[j], my = a.state[n + j], mz = a.state[2 * n + j];
                lx = a.state[3 * n + j], ly = a.state[4 * n + j], lz = a.state[5 * n + j];
            }
            FreeFactors ff{1.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            RfRelax rr{1.f, 1.f, 0.f, 0.f, 0.f, 0.f};
            float wz = 0.0f;
            int slot = 0, grp = 0, row = 0;
            // one sample (x, y) into the B block; a full block (or the window's last sample) goes to the tensor
            // cores. Returns false when a wait failed (the CTA stops).
            auto stage = [&](float x, float y) -> bool {
                const int b = grp & 1;
                // buffer b is free once the MMAs of the block before last have completed (each thread waits; a
                // failed wait is reported at the next barrier)
                if (slot == 0 && !drain(b)) err = true;
                uint16_t xh, xl, yh, yl;
                split_bf16(x, xh, xl);
                split_bf16(y, yh, yl);
                const uint32_t off = kmajor_off(slot, 2 * tid, MM_B_LBO, MM_B_SBO);
                unsigned char* bb = sm + MM_OFF_B + 2 * b * MM_B_BYTES;
                *reinterpret_cast<uint32_t*>(bb + off) = (uint32_t)xh | ((uint32_t)yh << 16);
                *reinterpret_cast<uint32_t*>(bb + MM_B_BYTES + off) = (uint32_t)xl | ((uint32_t)yl << 16);
                ++slot;
                ++row;
                if (slot == MM_BLOCK || row == win.w) {
                    fence_proxy_async_smem();  // this thread's B writes, visible to the tensor cores
                    if (__syncthreads_or(err)) return false;  // the block is complete; every wait so far succeeded
                    if (tid == 0) {
                        if (!a_waited && !mbar_wait_bounded(&bars[4], a_phase)) err = true;
                        if (!err) {
                            tc_fence_after();
                            const uint32_t bh = sB + 2 * b * MM_B_BYTES, bl = bh + MM_B_BYTES;
                            const uint32_t d = tmem + (uint32_t)(grp * MM_BLOCK);
                            // K step kk starts 2 kk core matrices further along K: the descriptors' start field
                            // (address >> 4, low 14 bits) advances by 2 LBO / 16 per step
                            uint64_t ah_d = umma_desc(sA, MM_A_LBO, MM_A_SBO);
                            uint64_t al_d = umma_desc(sA + MM_A_BYTES, MM_A_LBO, MM_A_SBO);
                            uint64_t bh_d = umma_desc(bh, MM_B_LBO, MM_B_SBO);
                            uint64_t bl_d = umma_desc(bl, MM_B_LBO, MM_B_SBO);
#pragma unroll
                            for (int kk = 0; kk < 16; ++kk) {
                                umma_bf16(d, ah_d, bh_d, idesc, (kk == 0 && first_tile) ? 0u : 1u);
                                umma_bf16(d, ah_d, bl_d, idesc, 1u);
                                umma_bf16(d, al_d, bh_d, idesc, 1u);
                                ah_d += 2 * MM_A_LBO / 16, al_d += 2 * MM_A_LBO / 16;
                                bh_d += 2 * MM_B_LBO / 16, bl_d += 2 * MM_B_LBO / 16;
                            }
                            umma_commit(&bars[2 + b]);
                        }
                    }
                    if (!a_waited) a_phase ^= 1u, a_waited = true;
                    mma_pending[b] = true;
                    ++grp;
                    slot = 0;
                }
                return true;
            };
            for (int s = 0; s < nseg && !fail; ++s) {
                const SegRec q = q0[s];
                const int f = q.flags;
                if (f & BP_RF) {
                    if (s == 0 || !(f & BP_SAME_RFDT)) rr = rf_relax(q.dt, p);
                    if (s == 0 || !(f & BP_SAME_OFF)) wz = rf_wz(q, p);
                    rf_step_wz(q, p, rr, wz, mx, my, mz, lx, ly, lz);
                    if (!(f & (BP_ADC | BP_SPOIL))) {  // the rest of the pulse, as in bp_forward
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
                    if (s == 0 || !(f & BP_SAME_FREE)) ff = free_factors(q, a.seg64[win.x + s], p);
                    free_step(ff, p, mx, my, mz, lx, ly, lz);
                    if ((f & (BP_ADC | BP_SPOIL)) == BP_ADC) {
                        // a readout run, as in bp_forward: the samples by a float32 recurrence within this window
                        // and block of BP_ADJ_WIN segments, the state after it from the merged factors
                        const int block_end = min(nseg, (win.x + s) / BP_ADJ_WIN * BP_ADJ_WIN + BP_ADJ_WIN - win.x);
                        int e = s + 1;
                        float zr = mx + lx, zi = my + ly;
                        if (readout && !stage(zr, zi)) fail = true;
                        while (!fail && e < block_end && (q0[e].flags & ~BP_SPOIL) == (BP_ADC | BP_SAME_FREE)) {
                            if (readout) {
                                readout_advance(ff, zr, zi);
                                if (!stage(zr, zi)) {
                                    fail = true;
                                    break;
                                }
                            }
                            if (q0[e++].flags & BP_SPOIL) break;
                        }
                        if (fail) break;
                        if (e > s + 1) {
                            const FreeFactors fr = free_factors_merged(q, a.seg64[win.x + s], p, e - s - 1);
                            free_step(fr, p, mx, my, mz, lx, ly, lz);
                            if (q0[e - 1].flags & BP_SPOIL) mx = my = lx = ly = 0.0f;
                        }
                        s = e - 1;
                        continue;
                    }
                }
                if (f & (BP_ADC | BP_SPOIL)) {
                    if ((f & BP_ADC) && readout && !stage(mx + lx, my + ly)) {
                        fail = true;
                        break;
                    }
                    if (f & BP_SPOIL) mx = my = lx = ly = 0.0f;
                }
            }
            // (on a failure the tile loop ends below, after the A-tile copy has been waited for)
            if (active) {
                a.state[j] = mx, a.state[n + j] = my, a.state[2 * n + j] = mz;
                a.state[3 * n + j] = lx, a.state[4 * n + j] = ly, a.state[5 * n + j] = lz;
            }
            if (readout && !a_waited && tid == 0) mbar_wait_bounded(&bars[4], a_phase);  // only on a failure path
            if (readout && !a_waited) a_phase ^= 1u;
            first_tile = false;
        }
        if (fail) break;
        if (readout) {  // the window's coil sums: D rows 0 .. 2C-1 (TMEM lanes of warp 0), columns = samples
            bool okd = drain(0);
            okd = drain(1) && okd;
            if (__syncthreads_or(!okd || err)) {
                fail = true;
                break;
            }
            tc_fence_after();
            if (warp == 0) {
                for (int c0 = 0; c0 < MM_SAMPLES && c0 < win.w; c0 += 16) {
                    float v[16];
                    tmem_ld16(tmem + (uint32_t)c0, v);
                    tmem_ld_wait();
                    if (tid < nv) {
#pragma unroll
                        for (int t = 0; t < 16; ++t)
                            if (c0 + t < win.w) atomicAdd(a.raw + (size_t)(win.z + c0 + t) * nv + tid, (double)v[t]);
                    }
                }
            }
            tc_fence_before();
            __syncthreads();
        }
    }
    // leave no copy or MMA in flight (failure paths only), then free the tensor memory
    if (seg_pending >= 0 && tid == 0) {
        const int k = seg_pending - a.w_begin;
        mbar_wait_bounded(&bars[k & 1], (k >> 1) & 1);
    }
    drain(0);
    drain(1);
    if ((fail || err) && tid == 0) atomicOr(a.status, BP_ERR_TMA_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, MM_TMEM_COLS);
    }
}

// A tiles from the coil sensitivities ([16][n] float32, coil c real at row 2c, imaginary at 2c + 1): one thread
// per (spin, row), writing the spin's two K entries of that row as bfloat16 high and low parts.
__global__ void bp_mma_atiles_kernel(const float* __restrict__ sens, int n, int n_coils, int n_tiles,
                                     uint8_t* __restrict__ atiles) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n_tiles * MM_THREADS * 16) return;
    const int r = (int)(t & 15), jt = (int)((t >> 4) % MM_THREADS), tile = (int)(t / (16 * MM_THREADS));
    const int j = tile * MM_THREADS + jt;
    float v0 = 0.0f, v1 = 0.0f;  // entries k = 2 jt (multiplies Mx) and 2 jt + 1 (multiplies My)
    if (j < n && r < 2 * n_coils) {
        const int c = r >> 1;
        const float sr = sens[(2 * c) * n + j], si = sens[(2 * c + 1) * n + j];
        if (r & 1) v0 = si, v1 = sr;
        else v0 = sr, v1 = -si;
    }
    uint16_t h0, l0, h1, l1;
    split_bf16(v0, h0, l0);
    split_bf16(v1, h1, l1);
    uint8_t* base = atiles + (size_t)tile * 2 * MM_A_BYTES;
    const uint32_t off = (uint32_t)((r >> 3) * MM_A_SBO + ((2 * jt) >> 3) * MM_A_LBO + (r & 7) * 16 + ((2 * jt) & 7) * 2);
    *reinterpret_cast<uint32_t*>(base + off) = (uint32_t)h0 | ((uint32_t)h1 << 16);
    *reinterpret_cast<uint32_t*>(base + MM_A_BYTES + off) = (uint32_t)l0 | ((uint32_t)l1 << 16);
}

extern "C" int64_t bp_mma_atiles_bytes(int n) {
    if (n < 1) return -1;
    return (int64_t)((n + MM_THREADS - 1) / MM_THREADS) * 2 * MM_A_BYTES;
}

extern "C" int bp_mma_atiles(const float* sens, int n, int n_coils, void* atiles, void* stream) {
    if (!sens || !atiles || n < 1 || n_coils < 1) return BP_E_ARG;
    if (n_coils > BP_MMA_MAX_COILS) return BP_E_SIZE;
    if ((reinterpret_cast<uintptr_t>(atiles) & 15) != 0) return BP_E_ALIGN;
    const int n_tiles = (n + MM_THREADS - 1) / MM_THREADS;
    const int64_t total = (int64_t)n_tiles * MM_THREADS * 16;
    const int threads = 256;
    bp_mma_atiles_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, static_cast<cudaStream_t>(stream)>>>(
        sens, n, n_coils, n_tiles, static_cast<uint8_t*>(atiles));
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// Persistent grid of bp_forward_mma: resident CTAs per SM (shared memory allows 3; tensor memory 512 / 64 = 8)
// times the SM count, capped by max_ctas (> 0) and the tile count.
static int mma_grid(int n, int max_ctas, int* grid_out) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    static bool configured[64] = {false};
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_forward_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MM_SMEM) !=
                cudaSuccess ||
            cudaFuncSetAttribute(bp_forward_mma_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return BP_E_LAUNCH;
        configured[dev] = true;
    }
    // residency from the SM's own limits (the runtime's occupancy query answers 1 for this kernel, while the
    // profiler's limits are 3 by shared memory, 6 by registers): shared memory with the per-block reservation,
    // registers, threads, and tensor memory (512 columns per SM)
    int smem_sm = 0, smem_res = 0, regs_sm = 0, thr_sm = 0;
    cudaFuncAttributes fa;
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, bp_forward_mma_kernel) != cudaSuccess)
        return BP_E_LAUNCH;
    per_sm = smem_sm / (MM_SMEM + smem_res);
    const int regs_block = ((fa.numRegs * 32 + 255) / 256) * 256 * (MM_THREADS / 32);
    if (regs_block > 0 && regs_sm / regs_block < per_sm) per_sm = regs_sm / regs_block;
    if (thr_sm / MM_THREADS < per_sm) per_sm = thr_sm / MM_THREADS;
    if (per_sm > 512 / MM_TMEM_COLS) per_sm = 512 / MM_TMEM_COLS;
    if (per_sm < 1) per_sm = 1;
    const int n_tiles = (n + MM_THREADS - 1) / MM_THREADS;
    int grid = sms * per_sm;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > n_tiles) grid = n_tiles;
    *grid_out = grid;
    return BP_OK;
}

extern "C" int bp_forward_mma_grid(int n) {
    int grid = 0;
    if (n < 1) return -BP_E_ARG;
    const int code = mma_grid(n, 0, &grid);
    return code == BP_OK ? grid : -code;
}

extern "C" int bp_forward_mma(const float* spins, const void* atiles, int n, int n_coils, const void* segs,
                              const double* seg64, const int32_t* windows, int w_begin, int w_end, float* state,
                              double* raw, int max_ctas, int32_t* status, void* stream) {
    if (n < 1 || n_coils < 1 || w_begin < 0 || w_end < w_begin || !spins || !segs || !seg64 || !windows || !state ||
        !status)
        return BP_E_ARG;
    if (n_coils > BP_MMA_MAX_COILS) return BP_E_SIZE;
    if (raw && !atiles) return BP_E_ARG;
    if ((reinterpret_cast<uintptr_t>(segs) & 15) != 0 || (reinterpret_cast<uintptr_t>(atiles) & 15) != 0)
        return BP_E_ALIGN;
    if (w_end == w_begin) return BP_OK;
    int grid = 0;
    const int code = mma_grid(n, max_ctas, &grid);
    if (code != BP_OK) return code;
    MmaArgs a{spins, static_cast<const uint8_t*>(atiles), static_cast<const SegRec*>(segs),
              reinterpret_cast<const double4*>(seg64), reinterpret_cast<const int4*>(windows), n, n_coils,
              w_begin, w_end, state, raw, status};
    bp_forward_mma_kernel<<<grid, MM_THREADS, MM_SMEM, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}
