// Device code of the physics variant of the forward kernel (bp_forward_physics): the rate-model bound pool
// (magnetization transfer) and the scanner field model's concomitant fields, for static spins.
//
// Physics follows blochparty's exchange.py and fields.py and its GPU engine's V=1 step
// (engines/gpu/shaders/common.metal:40-50 offset, :145-208 the bound pool):
//  * the bound pool keeps a longitudinal magnetization Mzb (equilibrium f PD) that exchanges with the water's Mz
//    (exchange.py:1-45): d(Mz, Mzb)/dt = A (Mz, Mzb) + c over a segment, with A = [[-(r1 + k f), k], [k f,
//    -(r1b + k + W)]] and c = (r1 PD, r1b f PD), solved exactly per segment (exchange.z_exchange, :215-244);
//  * RF saturates it at W = w1^2 G(f_rf - bz - dw), w1 = 2 pi b1 |rf| [rad/s], G the absorption lineshape
//    (Lorentzian, or the super-Lorentzian from a table held constant inside a cutoff; exchange.py:146-180);
//  * the concomitant field adds to a segment's off-resonance bz: at leading order a quadratic form of the gradient
//    with per-spin coefficients, c . (gx^2, gy^2, gz^2, gx gy, gx gz, gy gz); exactly, |B| - f0 - lin
//    = t^2 / (sqrt(u^2 + t^2) + u), t the transverse field (ax . g, ay . g), u = f0 + lin (fields.py:207-245).
#pragma once
#include "bloch_common.cuh"

// BP_BOUND_ONLY (the header): an RF segment only the bound pool feels; the water precesses, the pool saturates.

// The physics inputs a launch of the variant reads (device pointers; see bp_forward_physics in the header).
struct PhysArgs {
    int mt;                // a bound pool is present
    int conc_mode;         // 0 none, 1 leading order, 2 exact
    const float* pool;     // [5][n]: f, k [1/s], r1b = 1/T1b [1/s], T2b [s], dw [Hz]
    float* bstate;         // [2][n]: Mzb and its low part, in/out
    const float* rf_freq;  // [S] the RF's frequency [Hz]
    const float* line;     // lineshape: kind (1 Lorentzian, 2 super-Lorentzian), cutoff [Hz], ln x0, step, x_min,
                           // size; then `size` values ln F at ln x0 + i step (super-Lorentzian)
    const float* conc;     // [7][n]: mode 1: the quadratic form's coefficients (6); mode 2: ax (3), ay (3), f0
    const double* segq;    // [S][6] mode 1: dt (gx^2, gy^2, gz^2, gx gy, gx gz, gy gz) in float64
};

struct Pool {
    float f, k, r1b, t2b, dw;
};

__device__ __forceinline__ Pool load_pool(const float* __restrict__ pool, int n, int j) {
    return Pool{pool[j], pool[n + j], pool[2 * n + j], pool[3 * n + j], pool[4 * n + j]};
}

// The per-spin coefficients of the concomitant field (7 values; unused ones 0).
struct Conc {
    float c[7];
};

__device__ __forceinline__ Conc load_conc(const float* __restrict__ conc, int n, int j, int mode) {
    Conc k;
#pragma unroll
    for (int i = 0; i < 7; ++i) k.c[i] = (mode && (i < 6 || mode == 2)) ? conc[i * n + j] : 0.0f;
    return k;
}

// The exact longitudinal exchange step over a time t with saturation w, as an increment of (Mz, Mzb) from the
// steady state z: exp(A t) = e^{m t} (cosh(q t) I + sinh(q t) / q (A - m I)) with m, h the half sum and half
// difference of A's diagonal and q = sqrt(h^2 + a12 a21); e^{mt} cosh(qt) - 1 comes from expm1 of the two
// eigenvalues, so a short step (an RF raster of microseconds) keeps its small increment to float32 precision.
struct ZStep {
    float chm1, sh, z1, z2, h, a12, a21;
};

__device__ __forceinline__ ZStep zstep(float t, const Spin& p, const Pool& b, float w) {
    const float kf = b.k * b.f;
    const float a11 = -(p.r1 + kf), a12 = b.k, a21 = kf, a22 = -(b.r1b + b.k + w);
    const float c1 = p.r1 * p.pd, c2 = b.r1b * b.f * p.pd;
    const float det = a11 * a22 - a12 * a21;
    ZStep z;
    z.z1 = -(a22 * c1 - a12 * c2) / det;
    z.z2 = -(a11 * c2 - a21 * c1) / det;
    const float m = 0.5f * (a11 + a22), h = 0.5f * (a11 - a22);
    const float q = sqrtf(h * h + a12 * a21);
    z.chm1 = 0.5f * (expm1f((m + q) * t) + expm1f((m - q) * t));
    if (2.0f * q * t < 1.0f)
        z.sh = q > 0.0f ? expf((m - q) * t) * 0.5f * expm1f(2.0f * q * t) / q : t * expf(m * t);
    else
        z.sh = 0.5f * (expf((m + q) * t) - expf((m - q) * t)) / q;
    z.h = h;
    z.a12 = a12;
    z.a21 = a21;
    return z;
}

// (Mz, Mzb) advanced by a step, each increment added to its compensated (hi, lo) pair.
__device__ __forceinline__ void zapply(const ZStep& z, float& mz, float& lz, float& mb, float& lb) {
    const float d1 = mz - z.z1, d2 = mb - z.z2;
    const float n1 = fmaf(z.chm1, d1, z.sh * fmaf(z.h, d1, z.a12 * d2));
    const float n2 = fmaf(z.chm1, d2, z.sh * fmaf(z.a21, d1, -z.h * d2));
    two_sum(mz, lz, n1);
    two_sum(mb, lb, n2);
}

// The absorption lineshape G(2 pi delta) [s] of a bound pool with T2b = t2b (exchange.lorentzian and
// exchange.superlorentzian): Lorentzian t2b / (1 + x^2), x = 2 pi delta t2b; super-Lorentzian t2b F(x) with
// x = 2 pi max(|delta|, cutoff) t2b, ln F interpolated linearly in ln x on the table (clamped to its ends), and 0
// beyond x = 30.
__device__ __forceinline__ float lineshape(float delta, float t2b, const float* __restrict__ line) {
    if (line[0] < 1.5f) {
        const float x = BP_TWO_PI_F * delta * t2b;
        return t2b / fmaf(x, x, 1.0f);
    }
    const float x = BP_TWO_PI_F * fmaxf(fabsf(delta), line[1]) * t2b;
    if (x > 30.0f) return 0.0f;
    const int size = (int)line[5];
    const float pos = fminf(fmaxf((logf(fmaxf(x, line[4])) - line[2]) / line[3], 0.0f), (float)(size - 1));
    const int i = min((int)floorf(pos), size - 2);
    const float a = pos - (float)i;
    const float* lf = line + 6;
    return t2b * expf(fmaf(lf[i + 1], a, lf[i] * (1.0f - a)));
}

// The concomitant field's phase over a segment [cycles], in float32 (RF segments): mode 1 c . Q, Q = segq[s] the
// segment's dt-weighted gradient monomials; mode 2 dt (|B| - f0 - lin) = T2 / (sqrt(U^2 + T2) + U) with
// U = f0 dt + lin dt and T2 = (ax . k)^2 + (ay . k)^2 (k = g dt; the segment's dt cancels), lin_cyc = lin dt.
__device__ __forceinline__ float conc_cycles(int mode, const Conc& k, const SegRec& q, const double* __restrict__ sq,
                                             float lin_cyc) {
    if (mode == 1) {
        float acc = 0.0f;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc = fmaf(k.c[i], (float)sq[i], acc);
        return acc;
    }
    const float tx = fmaf(k.c[0], q.kx, fmaf(k.c[1], q.ky, k.c[2] * q.kz));
    const float ty = fmaf(k.c[3], q.kx, fmaf(k.c[4], q.ky, k.c[5] * q.kz));
    const float t2 = fmaf(tx, tx, ty * ty);
    const float u = fmaf(k.c[6], q.dt, lin_cyc);
    return t2 > 0.0f ? t2 / (sqrtf(fmaf(u, u, t2)) + u) : 0.0f;
}

// The same in float64 (the free segments' phase, taken in float64 like the rest of it).
__device__ __forceinline__ double conc_cycles64(int mode, const Conc& k, const SegRec& q, const double4& k64,
                                                const double* __restrict__ sq, double lin_cyc) {
    if (mode == 1) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) acc = fma((double)k.c[i], sq[i], acc);
        return acc;
    }
    const double tx = fma((double)k.c[0], k64.x, fma((double)k.c[1], k64.y, (double)k.c[2] * k64.z));
    const double ty = fma((double)k.c[3], k64.x, fma((double)k.c[4], k64.y, (double)k.c[5] * k64.z));
    const double t2 = fma(tx, tx, ty * ty);
    const double u = fma((double)k.c[6], (double)q.dt, lin_cyc);
    return t2 > 0.0 ? t2 / (sqrt(fma(u, u, t2)) + u) : 0.0;
}

// An RF segment's rotation about z with the field model: -2 pi (lin + concomitant) cycles.
__device__ __forceinline__ float phys_wz(const SegRec& q, const Spin& p, int mode, const Conc& k,
                                         const double* __restrict__ sq) {
    const float lin = fmaf(q.kx, p.px, fmaf(q.ky, p.py, fmaf(q.kz, p.pz, fmaf(q.dt, p.db0, q.beta))));
    return -BP_TWO_PI_F * (mode ? lin + conc_cycles(mode, k, q, sq, lin) : lin);
}

// free_factors_merged (reps = 1: free_factors) with the concomitant phase added before the reduction mod 1.
__device__ __forceinline__ FreeFactors free_factors_phys(const SegRec& q, const double4& k64, const Spin& p, int reps,
                                                         int mode, const Conc& k, const double* __restrict__ sq) {
    FreeFactors f;
    double cyc = fma(k64.x, (double)p.px,
                     fma(k64.y, (double)p.py, fma(k64.z, (double)p.pz, fma((double)q.dt, (double)p.db0, k64.w))));
    if (mode) cyc += conc_cycles64(mode, k, q, k64, sq, cyc);
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

// A free segment with the bound pool: the transverse part as free_step (float-float rotation, exact relaxation),
// the longitudinal part by the exchange step z (no saturation).
__device__ __forceinline__ void free_step_mt(const FreeFactors& f, const ZStep& z, float& mx, float& my, float& mz,
                                             float& lx, float& ly, float& lz, float& mb, float& lb) {
    float xh, xl, yh, yl;
    ff_rotate(mx, lx, my, ly, f.ch, f.cl, f.sh, f.sl, xh, xl);
    ff_rotate(my, ly, mx, lx, f.ch, f.cl, -f.sh, -f.sl, yh, yl);
    two_sum(xh, xl, xh * f.e2);
    two_sum(yh, yl, yh * f.e2);
    mx = xh, lx = xl, my = yh, ly = yl;
    zapply(z, mz, lz, mb, lb);
}

// An RF segment with the bound pool (Strang, as the plain step): half a step of transverse relaxation and of the
// saturated exchange, the water's rotation about its effective field (about z alone for a bound-only segment),
// the other half; every increment added by two-sum. e2h = expm1(-dt r2 / 2); wz from phys_wz.
__device__ __forceinline__ void rf_step_mt(const SegRec& q, const Spin& p, const Pool& b, float e2h, float wz,
                                           float f_rf, const float* __restrict__ line, float& mx, float& my,
                                           float& mz, float& lx, float& ly, float& lz, float& mb, float& lb) {
    const bool bound_only = (q.flags & BP_BOUND_ONLY) != 0;
    // W = w1^2 G(f_rf - bz - dw): w1^2 = b1^2 (wx0^2 + wy0^2) / dt^2, bz = -wz / (2 pi dt)
    const float inv_dt = q.dt > 0.0f ? 1.0f / q.dt : 0.0f;
    const float w1sq = p.b1 * p.b1 * fmaf(q.wx0, q.wx0, q.wy0 * q.wy0) * inv_dt * inv_dt;
    const float delta = f_rf + wz * inv_dt * (1.0f / BP_TWO_PI_F) - b.dw;
    const float w = w1sq > 0.0f ? w1sq * lineshape(delta, b.t2b, line) : 0.0f;
    const ZStep z = zstep(0.5f * q.dt, p, b, w);
    two_sum(mx, lx, mx * e2h);
    two_sum(my, ly, my * e2h);
    zapply(z, mz, lz, mb, lb);
    if (bound_only)
        rotate_inc(0.0f, 0.0f, wz, mx, my, mz, lx, ly, lz);
    else
        rotate_inc(q.wx0 * p.b1, q.wy0 * p.b1, wz, mx, my, mz, lx, ly, lz);
    two_sum(mx, lx, mx * e2h);
    two_sum(my, ly, my * e2h);
    zapply(z, mz, lz, mb, lb);
}
