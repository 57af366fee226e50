// Shared device code of the sm_100a Bloch kernels: the segment record, the compensated (two-sum) state
// arithmetic, the per-segment propagation steps, and the TMA / mbarrier primitives that stage segment blocks
// into shared memory.
//
// Physics and conventions follow blochparty's plain-Bloch GPU path (engines/gpu/shaders/common.metal:10-103)
// and its core (engines/core.py:71-150): dM/dt = gamma M x B with fields in Hz, so a segment's rotation vector
// is w = -2 pi dt (b1 rf_x, b1 rf_y, G.r + dB0 + b0_offset); RF segments relax dt/2, rotate, relax dt/2 (Strang);
// free segments rotate about z exactly and relax exactly. The state is float32 with a float32 low part per
// component: RF increments are added to it by Knuth's two-sum, and free segments are evaluated in float-float
// arithmetic, so a slowly changing magnetization (long RF trains, readouts) accumulates no float32 rounding.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/blochparty_b200.h"

#define BP_TWO_PI_F 6.283185307179586f

// segment flags (host: blochparty_b200/engine.py pack_segments)
#define BP_RF 1          // RF segment
#define BP_ADC 2         // sample at the end of the segment
#define BP_SPOIL 4       // zero Mxy at the end of the segment (after its sample)
#define BP_SAME_FREE 8   // free segment identical (dt, moment, offset) to the free segment just before it
#define BP_SAME_RFDT 16  // RF segment with the dt of the RF segment just before it
#define BP_SAME_OFF 32   // RF segment with the dt, moment and offset of the RF segment just before it (same G.r)
#define BP_SMALL 64      // RF segment whose rotation stays below |w| = 1/4 for every spin (a bound from the spins'
                         // extents, set by the host): the first tier of the Rodrigues factors without tests

// status bits written by the kernels (read by the host after the launch)
#define BP_ERR_TMA_TIMEOUT 1
#define BP_ERR_BAD_WINDOW 2
#define BP_ERR_NO_STATE 4  // the sweep from saved states met a window whose states were not saved (results invalid)

// One segment, 32 bytes: what every spin needs, derived on the host in float64.
struct __align__(16) SegRec {
    float dt;        // [s]
    float wx0, wy0;  // -2 pi dt rf_x, -2 pi dt rf_y [rad per unit B1]
    float kx, ky, kz;  // gradient moment g dt [cycles/m]
    float beta;      // b0_offset dt [cycles]
    int flags;
};

struct Spin {
    float px, py, pz, pd, r1, r2, db0, b1;
};

__device__ __forceinline__ Spin load_spin(const float* __restrict__ spins, int n, int j, bool active) {
    Spin p;
    p.px = spins[j];
    p.py = spins[n + j];
    p.pz = spins[2 * n + j];
    p.pd = active ? spins[3 * n + j] : 0.0f;
    p.r1 = spins[4 * n + j];
    p.r2 = spins[5 * n + j];
    p.db0 = spins[6 * n + j];
    p.b1 = spins[7 * n + j];
    return p;
}

// hi + lo += d with the rounding error of the sum kept in lo (Knuth's two-sum; the __f*_rn intrinsics keep the
// compiler from contracting or reassociating it).
__device__ __forceinline__ void two_sum(float& hi, float& lo, float d) {
    d = __fadd_rn(d, lo);
    const float t = __fadd_rn(hi, d);
    const float bp = __fsub_rn(t, hi);
    lo = __fadd_rn(__fsub_rn(hi, __fsub_rn(t, bp)), __fsub_rn(d, bp));
    hi = t;
}

// hi + lo += d for an increment that does not outgrow hi (an RF step's increment next to the state it turns):
// Dekker's fast two-sum, exact when the exponent of hi is at least that of d + lo (and whenever hi is 0), in four
// operations instead of seven. Where a component crosses zero the condition can fail for a step, and that step's
// rounding error (an ulp of the small increment) is not kept.
__device__ __forceinline__ void quick_two_sum(float& hi, float& lo, float d) {
    d = __fadd_rn(d, lo);
    const float t = __fadd_rn(hi, d);
    lo = __fsub_rn(d, __fsub_rn(t, hi));
    hi = t;
}

// Rodrigues coefficients of a rotation by |w|, from p2 = |w|^2: s1 = sin(phi)/phi, s2 = (1 - cos phi)/phi^2.
// Below phi = 1 both are their Taylor series in p2 (sum_k (-1)^k p2^k / (2k+1)! and / (2k+2)!): truncated after
// p2^3 below phi = 1/4 (the usual RF step; first dropped terms p2^4 / 9! < 4.3e-11) and after p2^5 below phi = 1
// (first dropped terms below 2e-10), far under a float32 ulp, on the FMA pipe with no square root. Above, the
// accurate sine of the angle and of its half.
// The first tier alone (p2 < 1/16 known to the caller).
__device__ __forceinline__ void rodrigues_small(float p2, float& s1, float& s2) {
    s1 = fmaf(p2, fmaf(p2, fmaf(p2, -1.9841269841269841e-04f, 8.3333333333333333e-03f), -1.6666666666666667e-01f), 1.0f);
    s2 = fmaf(p2, fmaf(p2, fmaf(p2, -2.4801587301587302e-05f, 1.3888888888888889e-03f), -4.1666666666666667e-02f), 0.5f);
}

__device__ __forceinline__ void rodrigues_coeffs(float p2, float& s1, float& s2) {
    if (p2 < 0.0625f) {
        rodrigues_small(p2, s1, s2);
    } else if (p2 < 1.0f) {
        s1 = fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, -2.5052108385441720e-08f, 2.7557319223985893e-06f),
                                              -1.9841269841269841e-04f), 8.3333333333333333e-03f),
                           -1.6666666666666667e-01f), 1.0f);
        s2 = fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, -2.0876756987868099e-09f, 2.7557319223985891e-07f),
                                              -2.4801587301587302e-05f), 1.3888888888888889e-03f),
                           -4.1666666666666667e-02f), 0.5f);
    } else {
        const float phi = sqrtf(p2);
        const float inv = 1.0f / phi;
        const float sh = sinf(0.5f * phi) * inv;
        s1 = sinf(phi) * inv;
        s2 = 2.0f * sh * sh;
    }
}

// m += s1 (w x m) + s2 w x (w x m): the rotation about w as an increment, each component added by two_sum.
__device__ __forceinline__ void rotate_inc(float wx, float wy, float wz, float& mx, float& my, float& mz,
                                           float& lx, float& ly, float& lz) {
    const float p2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
    float s1, s2;
    rodrigues_coeffs(p2, s1, s2);
    const float cx = wy * mz - wz * my, cy = wz * mx - wx * mz, cz = wx * my - wy * mx;
    const float dx = wy * cz - wz * cy, dy = wz * cx - wx * cz, dz = wx * cy - wy * cx;
    two_sum(mx, lx, fmaf(s1, cx, s2 * dx));
    two_sum(my, ly, fmaf(s1, cy, s2 * dy));
    two_sum(mz, lz, fmaf(s1, cz, s2 * dz));
}

// Relaxation factors of an RF segment's two half steps (dt/2 each): e = expm1(-dt r / 2), a = 1 + e, and for the
// composed segment d = a^2 - 1 = e (2 + e); cz2 = (a1 + 1)(-pd e1h), the recovery term of both halves.
struct RfRelax {
    float a1, a2, d1, d2, e1h, cz2;
};

__device__ __forceinline__ RfRelax rf_relax(float dt, const Spin& p) {
    RfRelax r;
    r.e1h = expm1f(-0.5f * dt * p.r1);
    const float e2h = expm1f(-0.5f * dt * p.r2);
    r.a1 = 1.0f + r.e1h;
    r.a2 = 1.0f + e2h;
    r.d1 = r.e1h * (2.0f + r.e1h);
    r.d2 = e2h * (2.0f + e2h);
    r.cz2 = -(r.a1 + 1.0f) * p.pd * r.e1h;
    return r;
}

// The z component of an RF segment's rotation vector: -2 pi (k.r + dt dB0 + beta) (its off-resonance in cycles).
__device__ __forceinline__ float rf_wz(const SegRec& q, const Spin& p) {
    return -BP_TWO_PI_F * fmaf(q.kx, p.px, fmaf(q.ky, p.py, fmaf(q.kz, p.pz, fmaf(q.dt, p.db0, q.beta))));
}

// An RF segment: relax dt/2 (m1 = E m + c, E = diag(a2, a2, a1), c = (0, 0, -pd e1h)), rotate about w (n = R m1),
// relax dt/2 (E n + c), composed into one increment of m: (E E - I) m + E (R - I) m1 + (E + I) c, with
// (R - I) m1 = s1 (w x m1) + s2 w x (w x m1). The increment is small next to m and computed from m directly,
// so one (fast) two-sum per component (instead of one per sub-step) keeps the float32 state compensated.
// SMALL: the segment carries BP_SMALL (p2 < 1/16 for every spin).
template <bool SMALL = false>
__device__ __forceinline__ void rf_step_wz(const SegRec& q, const Spin& p, const RfRelax& r, float wz, float& mx,
                                           float& my, float& mz, float& lx, float& ly, float& lz) {
    const float wx = q.wx0 * p.b1, wy = q.wy0 * p.b1;
    const float m1x = mx * r.a2, m1y = my * r.a2, m1z = fmaf(-p.pd, r.e1h, mz * r.a1);
    const float p2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
    float s1, s2;
    if (SMALL)
        rodrigues_small(p2, s1, s2);
    else
        rodrigues_coeffs(p2, s1, s2);
    const float cx = wy * m1z - wz * m1y, cy = wz * m1x - wx * m1z, cz = wx * m1y - wy * m1x;
    const float dx = wy * cz - wz * cy, dy = wz * cx - wx * cz, dz = wx * cy - wy * cx;
    const float qx = fmaf(s1, cx, s2 * dx), qy = fmaf(s1, cy, s2 * dy), qz = fmaf(s1, cz, s2 * dz);
    quick_two_sum(mx, lx, fmaf(r.d2, mx, r.a2 * qx));
    quick_two_sum(my, ly, fmaf(r.d2, my, r.a2 * qy));
    quick_two_sum(mz, lz, fmaf(r.d1, mz, fmaf(r.a1, qz, r.cz2)));
}

__device__ __forceinline__ void rf_step(const SegRec& q, const Spin& p, const RfRelax& r, float& mx, float& my,
                                        float& mz, float& lx, float& ly, float& lz) {
    rf_step_wz(q, p, r, rf_wz(q, p), mx, my, mz, lx, ly, lz);
}

// Free-precession factors of one segment: the rotation (c, s) by -2 pi (k.r + dt dB0 + beta), evaluated in
// float64 from the float64 moments (so a spoiler's hundreds of cycles keep their fraction exactly), reduced to
// [-1/2, 1/2] cycle, and kept as float-float pairs c = ch + cl, s = sh + sl (unit norm to float64 rounding);
// e1, e2: expm1 of the relaxation over dt.
struct FreeFactors {
    float ch, cl, sh, sl, e1, e2;
};

__device__ __forceinline__ FreeFactors free_factors(const SegRec& q, const double4& k64, const Spin& p) {
    FreeFactors f;
    const double cyc = fma(k64.x, (double)p.px,
                           fma(k64.y, (double)p.py, fma(k64.z, (double)p.pz, fma((double)q.dt, (double)p.db0, k64.w))));
    const double fr = cyc - rint(cyc);
    double sd, cd;
    sincospi(-2.0 * fr, &sd, &cd);
    f.ch = (float)cd;
    f.cl = (float)(cd - (double)f.ch);
    f.sh = (float)sd;
    f.sl = (float)(sd - (double)f.sh);
    f.e1 = expm1f(-q.dt * p.r1);
    f.e2 = expm1f(-q.dt * p.r2);
    return f;
}

// The factors of `reps` consecutive copies of one free segment merged into one: the phase of reps x (k.r + dt dB0
// + beta) cycles, taken in float64 before the reduction to [-1/2, 1/2], and the relaxation over reps x dt.
__device__ __forceinline__ FreeFactors free_factors_merged(const SegRec& q, const double4& k64, const Spin& p,
                                                           int reps) {
    FreeFactors f;
    const double cyc = fma(k64.x, (double)p.px,
                           fma(k64.y, (double)p.py, fma(k64.z, (double)p.pz, fma((double)q.dt, (double)p.db0, k64.w))));
    const double tot = cyc * (double)reps;
    const double fr = tot - rint(tot);
    double sd, cd;
    sincospi(-2.0 * fr, &sd, &cd);
    f.ch = (float)cd;
    f.cl = (float)(cd - (double)f.ch);
    f.sh = (float)sd;
    f.sl = (float)(sd - (double)f.sh);
    const float t = (float)((double)q.dt * (double)reps);
    f.e1 = expm1f(-t * p.r1);
    f.e2 = expm1f(-t * p.r2);
    return f;
}

// One sample of a readout run from the previous one: z (e2 + 1) (c + i s), the rotation's low part folded into
// the products and the relaxation applied with one rounding (float32; the run's state is rebuilt exactly after it).
__device__ __forceinline__ void readout_advance(const FreeFactors& f, float& zr, float& zi) {
    const float tr = fmaf(f.cl, zr, -f.sl * zi), ti = fmaf(f.cl, zi, f.sl * zr);
    const float nr = fmaf(f.ch, zr, fmaf(-f.sh, zi, tr));
    const float ni = fmaf(f.ch, zi, fmaf(f.sh, zr, ti));
    zr = fmaf(nr, f.e2, nr);
    zi = fmaf(ni, f.e2, ni);
}

// hi + lo renormalised so that lo is below half an ulp of hi (requires |hi| >= |lo|).
__device__ __forceinline__ void fast_two_sum(float& hi, float& lo) {
    const float t = __fadd_rn(hi, lo);
    lo = __fsub_rn(lo, __fsub_rn(t, hi));
    hi = t;
}

// (ah + al) c - (bh + bl) s in float-float: the two main products exactly (FMA remainders), their difference by
// two-sum, the cross terms with the low parts added to the remainder.
__device__ __forceinline__ void ff_rotate(float ah, float al, float bh, float bl, const float ch, const float cl,
                                         const float sh, const float sl, float& rh, float& rl) {
    const float p = __fmul_rn(ch, ah), pe = fmaf(ch, ah, -p);
    const float q = __fmul_rn(sh, bh), qe = fmaf(sh, bh, -q);
    float t = p, te = 0.0f;
    two_sum(t, te, -q);
    float lo = te + (pe - qe);
    lo += fmaf(ch, al, -sh * bl);
    lo += fmaf(cl, ah, -sl * bh);
    fast_two_sum(t, lo);
    rh = t;
    rl = lo;
}

// A free segment, in float-float: the state (m + l) rotated about z exactly and relaxed exactly. Readout samples
// repeat one rotation tens to hundreds of times; float32 rounding of the state (or of the rotation factors) would
// otherwise drift coherently by ~1e-7 per sample (a measured 1e-5 relative signal error on the 64 x 64 GRE).
__device__ __forceinline__ void free_step(const FreeFactors& f, const Spin& p, float& mx, float& my, float& mz,
                                          float& lx, float& ly, float& lz) {
    float xh, xl, yh, yl;
    ff_rotate(mx, lx, my, ly, f.ch, f.cl, f.sh, f.sl, xh, xl);    // c x - s y
    ff_rotate(my, ly, mx, lx, f.ch, f.cl, -f.sh, -f.sl, yh, yl);  // c y + s x
    two_sum(xh, xl, xh * f.e2);
    two_sum(yh, yl, yh * f.e2);
    two_sum(mz, lz, (mz - p.pd) * f.e1);
    mx = xh, lx = xl, my = yh, ly = yl;
}

// ---- TMA bulk copies into shared memory, completed on an mbarrier ----

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// A window record the kernels can run: segments within one staged block, samples within the accumulator.
__device__ __forceinline__ bool window_ok(const int4& w, int samp_max) {
    return w.x >= 0 && w.y >= w.x && w.y - w.x <= BP_SEG_MAX && w.z >= 0 && w.w >= 0 && w.w <= samp_max;
}

// global -> shared bulk copy (cp.async.bulk, the TMA's untiled form): 16-byte aligned addresses, size a multiple
// of 16 bytes; completion is signalled as transaction bytes on `bar`.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`, giving up after a bounded number of polls (a copy of a few KB lands in
// microseconds; the bound is seconds). Returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

// Eight values per lane summed over the warp and scattered (a butterfly reduce-scatter): afterwards every lane
// holds the warp's total of value index (lane >> 2) & 7. Each stage exchanges the half of the remaining values
// that the partner lane keeps: 4 + 2 + 1 shuffles, then 2 for the last value's four copies (9 instead of the
// 40 of eight separate butterflies).
__device__ __forceinline__ float warp_reduce_scatter8(float* v, int lane) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool up = lane & 16;
        const float send = up ? v[k] : v[k + 4];
        const float keep = up ? v[k + 4] : v[k];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool up = lane & 8;
        const float send = up ? v[k] : v[k + 2];
        const float keep = up ? v[k + 2] : v[k];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    {
        const bool up = lane & 4;
        const float send = up ? v[0] : v[1];
        const float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}
