// Learned RF surrogate: a 14 -> 64 -> 64 -> 64 -> 16 GELU network standing in for the sub-stepped integration of
// one shaped RF pulse, mapping (off-resonance in the slice gradient, B1 scale) to the pulse's rotation and its
// first-order relaxation terms.
//
// No counterpart in the reference (its nearest part is the exact per-spin map of a reused pulse,
// engines/gpu/cuda/pulse.cu.in:3-32). Kernels here:
//  * bp_pulse_targets: training targets from the plain integrator: per sample, the pulse's per-step rotations
//    w = -2 pi dt (b1 rf_x, b1 rf_y, G z + df) composed as unit quaternions in float64, reduced by the free
//    precession (R = Rz(wz/2) R~ Rz(wz/2), wz = -2 pi (G z + df) T) so that the target is smooth in z, with the
//    first-order relaxation terms the whole-pulse splitting misses;
//  * bp_mlp_grad: fused forward + backward of the network over a batch (per-CTA gradient partials), then
//    bp_mlp_reduce (fixed-order sum over CTAs) and bp_adam (the optimiser step): training on the GPU;
//  * bp_surrogate_pulse: one pulse occurrence applied to every spin's state: inside the training domain, the
//    network's rotation wrapped by half-pulse relaxations (relax T/2, rotate, relax T/2) with its first-order
//    relaxation correction; outside it, the plain sub-stepped integration of the pulse's segments (the fallback).
// Quaternions: (q0, q1, q2, q3) = (cos |w|/2, sin |w|/2 w/|w|), composition "q1 then q2" = q2 q1 (Hamilton
// product); the Cayley-Klein pair of q is alpha = q0 - i q3, beta = -i (q1 + i q2).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "bloch_common.cuh"
#include "../../include/blochparty_b200.h"

#define MLP_H 64
#define MLP_X 2                        // the inputs (f^, b^)
#define MLP_NF 6                       // Fourier orders of f^
#define MLP_IN (MLP_X + 2 * MLP_NF)    // the first layer's features
#define MLP_OUT 16  // the reduced quaternion (4), dA~ / T (9) and dC~ / T (3)
// flat parameter layout: W1 (64 x 14), b1 (64), W2 (64 x 64), b2, W3 (64 x 64), b3, W4 (16 x 64), b4 (16)
#define P_W1 0
#define P_B1 (P_W1 + MLP_H * MLP_IN)
#define P_W2 (P_B1 + MLP_H)
#define P_B2 (P_W2 + MLP_H * MLP_H)
#define P_W3 (P_B2 + MLP_H)
#define P_B3 (P_W3 + MLP_H * MLP_H)
#define P_W4 (P_B3 + MLP_H)
#define P_B4 (P_W4 + MLP_OUT * MLP_H)
#define N_PARAMS (P_B4 + MLP_OUT)  // 10320

static_assert(N_PARAMS == BP_MLP_PARAMS, "parameter count");

// The training domain of a network is |df| <= dom_df [Hz], |b1 - 1| <= dom_b1, |z_rel| <= dom_z [slice widths]
// (the caller's choice). The pulse acts on a spin through its off-resonance in the slice gradient,
// f = df + G (z - z0) [Hz], and its B1 scale alone, so the inputs are f^ = f / F with F = dom_df + |G| dom_z
// thickness (the largest |f| in the domain) and b^ = (b1 - 1) / dom_b1; the first layer sees them with the
// Fourier features sin(k pi f^), cos(k pi f^), k = 1..6, which let a small network follow the slice profile's sharp
// edges (Tancik et al., "Fourier features let networks learn high frequency functions", 2020).

struct dq4 {
    double w, x, y, z;
};

__device__ __forceinline__ dq4 dq_mul(const dq4& a, const dq4& b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}

__device__ __forceinline__ dq4 dq_rotvec(double wx, double wy, double wz) {
    const double phi = sqrt(wx * wx + wy * wy + wz * wz);
    double s, c;
    sincos(0.5 * phi, &s, &c);
    const double k = phi > 1e-300 ? s / phi : 0.5;
    return {c, k * wx, k * wy, k * wz};
}

__device__ __forceinline__ dq4 dq_z(double angle) {
    double s, c;
    sincos(0.5 * angle, &s, &c);
    return {c, 0.0, 0.0, s};
}

// 3 x 3 float64 matrices, row-major
struct dm3 {
    double m[9];
};

__device__ __forceinline__ dm3 dm_of_quat(const dq4& q) {
    const double s = q.w, x = q.x, y = q.y, z = q.z;
    return {{1 - 2 * (y * y + z * z), 2 * (x * y - s * z), 2 * (x * z + s * y),
             2 * (x * y + s * z), 1 - 2 * (x * x + z * z), 2 * (y * z - s * x),
             2 * (x * z - s * y), 2 * (y * z + s * x), 1 - 2 * (x * x + y * y)}};
}

__device__ __forceinline__ dm3 dm_mul(const dm3& a, const dm3& b) {
    dm3 c;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            c.m[3 * r + k] = a.m[3 * r] * b.m[k] + a.m[3 * r + 1] * b.m[3 + k] + a.m[3 * r + 2] * b.m[6 + k];
    return c;
}

// Targets: samples [n][3] (df [Hz], b1, z_rel [slice widths]) -> targets [n][16] float32 (and q [n][4] if not null):
// the reduced rotation q~ (4), dA~ / T (9, row-major) and dC~ / T (3), from the plain integrator's Strang steps
// E(h) R_k E(h), h = dt / 2, expanded to first order in the relaxation rates:
//   A <- R_k A + h (P R_k + R_k P) R,  C <- R_k C + h (R_k e_z + e_z),  R <- R_k R   (P = diag(1, 1, 0)),
// then dA = A - (T/2)(P R + R P), dC = C - (T/2)(R e_z + e_z), reduced by Rz(-wz/2) like the rotation.
__global__ void bp_pulse_targets_kernel(const double2* __restrict__ rf, int k_steps, double dt, double gz,
                                        double thickness, double z0, const float* __restrict__ samples, int n,
                                        float* __restrict__ targets, float* __restrict__ qfull) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double df = samples[3 * i], b1 = samples[3 * i + 1], zr = samples[3 * i + 2];
    const double z = z0 + zr * thickness;
    const double w = -2.0 * M_PI * dt, wz = w * (gz * z + df), h = 0.5 * dt;
    dq4 q{1.0, 0.0, 0.0, 0.0};
    dm3 R{{1, 0, 0, 0, 1, 0, 0, 0, 1}}, A{{0, 0, 0, 0, 0, 0, 0, 0, 0}};
    double C[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < k_steps; ++k) {
        const double2 r = rf[k];
        const dq4 qk = dq_rotvec(w * b1 * r.x, w * b1 * r.y, wz);
        const dm3 Rk = dm_of_quat(qk);
        // (P R_k + R_k P) R: P zeroes row 2 of R_k (left) or column 2 of R_k (right)
        dm3 S;
#pragma unroll
        for (int e = 0; e < 9; ++e) S.m[e] = Rk.m[e] * ((e / 3 < 2 ? 1.0 : 0.0) + (e % 3 < 2 ? 1.0 : 0.0));
        const dm3 RA = dm_mul(Rk, A), SR = dm_mul(S, R);
#pragma unroll
        for (int e = 0; e < 9; ++e) A.m[e] = RA.m[e] + h * SR.m[e];
        const double c0 = Rk.m[0] * C[0] + Rk.m[1] * C[1] + Rk.m[2] * C[2];
        const double c1 = Rk.m[3] * C[0] + Rk.m[4] * C[1] + Rk.m[5] * C[2];
        const double c2 = Rk.m[6] * C[0] + Rk.m[7] * C[1] + Rk.m[8] * C[2];
        C[0] = c0 + h * Rk.m[2], C[1] = c1 + h * Rk.m[5], C[2] = c2 + h * (Rk.m[8] + 1.0);
        R = dm_mul(Rk, R);
        q = dq_mul(qk, q);
    }
    const double T = k_steps * dt;
    dm3 dA;
#pragma unroll
    for (int e = 0; e < 9; ++e)  // (P R + R P)_{rc} = R_{rc} ((r < 2) + (c < 2))
        dA.m[e] = A.m[e] - 0.5 * T * R.m[e] * ((e / 3 < 2 ? 1.0 : 0.0) + (e % 3 < 2 ? 1.0 : 0.0));
    const double dC[3] = {C[0] - 0.5 * T * R.m[2], C[1] - 0.5 * T * R.m[5], C[2] - 0.5 * T * (R.m[8] + 1.0)};
    const dq4 hq = dq_z(-0.5 * wz * k_steps);
    const dq4 qr = dq_mul(dq_mul(hq, q), hq);
    const dm3 Rh = dm_of_quat(hq);
    const dm3 dAr = dm_mul(dm_mul(Rh, dA), Rh);
    float* t = targets + 16 * (size_t)i;
    t[0] = (float)qr.w, t[1] = (float)qr.x, t[2] = (float)qr.y, t[3] = (float)qr.z;
#pragma unroll
    for (int e = 0; e < 9; ++e) t[4 + e] = (float)(dAr.m[e] / T);
#pragma unroll
    for (int r = 0; r < 3; ++r)
        t[13 + r] = (float)((Rh.m[3 * r] * dC[0] + Rh.m[3 * r + 1] * dC[1] + Rh.m[3 * r + 2] * dC[2]) / T);
    if (qfull) qfull[4 * i] = (float)q.w, qfull[4 * i + 1] = (float)q.x, qfull[4 * i + 2] = (float)q.y, qfull[4 * i + 3] = (float)q.z;
}

extern "C" int bp_pulse_targets(const double* rf, int k_steps, double dt, double gz, double thickness, double z0,
                                const float* samples, int n, float* targets, float* qfull, void* stream) {
    if (!rf || !samples || !targets || k_steps < 1 || n < 0 || dt <= 0 || thickness <= 0) return BP_E_ARG;
    if (n == 0) return BP_OK;
    bp_pulse_targets_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const double2*>(rf), k_steps, dt, gz, thickness, z0, samples, n, targets, qfull);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// GELU in its tanh form, 0.5 x (1 + tanh(u)), u = c (x + 0.044715 x^3), c = sqrt(2/pi) (Hendrycks and Gimpel),
// evaluated as the identical x sigma(2u) = x / (1 + exp(-2u)) with the fast exponential and divide (absolute error
// of sigma ~1e-7); the derivative is sigma(2u) + x s (1 - s) 2 du/dx. exp(-2u) overflowing to inf gives 0, the limit.
__device__ __forceinline__ float gelu_sig(float x) {
    const float c2 = 2.0f * 0.7978845608028654f;
    return __fdividef(1.0f, 1.0f + __expf(-c2 * fmaf(0.044715f * x, x * x, x)));
}

__device__ __forceinline__ float gelu_f(float x) { return x * gelu_sig(x); }

__device__ __forceinline__ float gelu_d(float x) {
    const float c2 = 2.0f * 0.7978845608028654f;
    const float s = gelu_sig(x);
    return fmaf(x * s * (1.0f - s), c2 * fmaf(3.0f * 0.044715f * x, x, 1.0f), s);
}

// ---- training: forward + backward over a batch ----
#define TR_T 128          // samples per CTA (one per thread)
#define TR_LD 65          // row stride (floats) of the per-sample activation arrays [TR_T][TR_LD]
#define TR_ARR (TR_T * TR_LD)

// The first layer's features of inputs (f^, b^): f^, b^, then sin(k pi f^), cos(k pi f^) for k = 1..6 (from
// sincospi(f^), the higher orders by the angle-addition formulas: about k float32 roundings each).
__device__ __forceinline__ void mlp_features(float fh, float bh, float g[MLP_IN]) {
    float s1, c1;
    sincospif(fh, &s1, &c1);
    g[0] = fh, g[1] = bh;
    float s = s1, c = c1;
#pragma unroll
    for (int k = 0; k < MLP_NF; ++k) {
        g[MLP_X + 2 * k] = s, g[MLP_X + 2 * k + 1] = c;
        const float sn = fmaf(s, c1, c * s1), cn = fmaf(c, c1, -s * s1);
        s = sn, c = cn;
    }
}

// The network's output for inputs x = (f^, b^), and (train) its pre-activations into z1, z2, z3 rows.
__device__ __forceinline__ void mlp_forward_row(const float* __restrict__ P, const float x[MLP_X], float* z1,
                                                float* z2, float* z3, float y[MLP_OUT]) {
    float g[MLP_IN];
    mlp_features(x[0], x[1], g);
    float a[MLP_H];
#pragma unroll
    for (int k = 0; k < MLP_H; ++k) {
        float v = P[P_B1 + k];
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) v = fmaf(P[P_W1 + MLP_IN * k + i], g[i], v);
        if (z1) z1[k] = v;
        a[k] = gelu_f(v);
    }
    float b[MLP_H];
    for (int k = 0; k < MLP_H; ++k) {
        float v = P[P_B2 + k];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) v = fmaf(P[P_W2 + MLP_H * k + i], a[i], v);
        if (z2) z2[k] = v;
        b[k] = gelu_f(v);
    }
    for (int k = 0; k < MLP_H; ++k) {
        float v = P[P_B3 + k];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) v = fmaf(P[P_W3 + MLP_H * k + i], b[i], v);
        if (z3) z3[k] = v;
        a[k] = gelu_f(v);
    }
#pragma unroll
    for (int j = 0; j < MLP_OUT; ++j) {
        float v = P[P_B4 + j];
#pragma unroll
        for (int i = 0; i < MLP_H; ++i) v = fmaf(P[P_W4 + MLP_H * j + i], a[i], v);
        y[j] = v;
    }
}

// Sum over the CTA's samples of dz[t][k] * act[t][i] -> grad[o_w + k * n_in + i], and of dz[t][k] -> grad[o_b + k]:
// thread (kb, ib) owns an 8 x 4 block of (k, i).
__device__ __forceinline__ void weight_grads(const float* dz, const float* act, int n_in, int nt, float* grad,
                                             int o_w, int o_b, int tid) {
    const int kb = tid >> 4, ib = tid & 15;
    if (4 * ib < n_in) {
        float acc[8][4];
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = 0.0f;
        for (int t = 0; t < nt; ++t) {
            float d[8], v[4];
#pragma unroll
            for (int r = 0; r < 8; ++r) d[r] = dz[t * TR_LD + 8 * kb + r];
#pragma unroll
            for (int c = 0; c < 4; ++c) v[c] = (4 * ib + c < n_in) ? act[t * TR_LD + 4 * ib + c] : 0.0f;
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(d[r], v[c], acc[r][c]);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (4 * ib + c < n_in) grad[o_w + (8 * kb + r) * n_in + 4 * ib + c] = acc[r][c];
    }
    if (tid < MLP_H) {
        float s = 0.0f;
        for (int t = 0; t < nt; ++t) s += dz[t * TR_LD + tid];
        grad[o_b + tid] = s;
    }
}

// Per CTA: samples [blockIdx.x * 128, +128) of x [n][2] (inputs f^, b^) and targets [n][16]; writes the CTA's
// gradient sum (not yet divided by the batch) to gpart[blockIdx.x][N_PARAMS] and its loss sum to lpart.
__global__ void __launch_bounds__(TR_T, 1) bp_mlp_grad_kernel(const float* __restrict__ params,
                                                              const float* __restrict__ x, const float* __restrict__ target,
                                                              int n, float vw, float cw, float* __restrict__ gpart,
                                                              float* __restrict__ lpart) {
    extern __shared__ __align__(16) float sm[];
    float* P = sm;                       // N_PARAMS (padded to a multiple of 4)
    float* z1 = P + ((N_PARAMS + 3) & ~3);
    float* z2 = z1 + TR_ARR;
    float* z3 = z2 + TR_ARR;
    float* buf = z3 + TR_ARR;            // activations of the layer below, then x
    __shared__ float dyb[TR_T][MLP_OUT];
    __shared__ float lsum[TR_T];
    const int tid = threadIdx.x;
    const int t0 = blockIdx.x * TR_T;
    const int nt = min(TR_T, n - t0);
    for (int i = tid; i < N_PARAMS; i += TR_T) P[i] = params[i];
    __syncthreads();
    float* g = gpart + (size_t)blockIdx.x * N_PARAMS;
    const bool live = tid < nt;
    float xin[MLP_X] = {0.f, 0.f}, y[MLP_OUT];
#pragma unroll
    for (int j = 0; j < MLP_OUT; ++j) y[j] = 0.0f;
    if (live) {
        xin[0] = x[MLP_X * (t0 + tid)], xin[1] = x[MLP_X * (t0 + tid) + 1];
        mlp_forward_row(P, xin, z1 + tid * TR_LD, z2 + tid * TR_LD, z3 + tid * TR_LD, y);
    }
    // loss (q0 - t0)^2 + vw |q_vec - t_vec|^2 + cw |c - t_c|^2 with q = y[0:4]/|y[0:4]| (vw weights the vector
    // part: relative precision for small rotations) and c = y[4:16] the first-order corrections;
    // dL/dy[0:4] = (dL/dq - q (q . dL/dq)) / |y[0:4]|, dL/dy[4:16] = 2 cw (c - t_c)
    float dy[MLP_OUT], loss = 0.0f;
#pragma unroll
    for (int j = 0; j < MLP_OUT; ++j) dy[j] = 0.0f;
    if (live) {
        const float* tg = target + (size_t)MLP_OUT * (t0 + tid);
        const float r = sqrtf(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
        const float inv = 1.0f / r;
        float q[4], gq[4], qg = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            q[j] = y[j] * inv;
            const float e = q[j] - tg[j];
            const float w = j == 0 ? 1.0f : vw;
            loss = fmaf(w * e, e, loss);
            gq[j] = 2.0f * w * e;
            qg = fmaf(q[j], gq[j], qg);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) dy[j] = (gq[j] - q[j] * qg) * inv;
#pragma unroll
        for (int j = 4; j < MLP_OUT; ++j) {
            const float e = y[j] - tg[j];
            loss = fmaf(cw * e, e, loss);
            dy[j] = 2.0f * cw * e;
        }
    }
#pragma unroll
    for (int j = 0; j < MLP_OUT; ++j) dyb[tid][j] = dy[j];
    lsum[tid] = loss;
    // a3 = gelu(z3) into buf (own row)
    for (int k = 0; k < MLP_H; ++k) buf[tid * TR_LD + k] = live ? gelu_f(z3[tid * TR_LD + k]) : 0.0f;
    __syncthreads();
    if (tid == 0) {
        float s = 0.0f;
        for (int t = 0; t < nt; ++t) s += lsum[t];
        lpart[blockIdx.x] = s;
    }
    // layer 4: dW4[j][k] = sum_t dy[t][j] a3[t][k], db4[j] = sum_t dy[t][j]
    for (int o = tid; o < MLP_OUT * MLP_H + MLP_OUT; o += TR_T) {
        float s = 0.0f;
        if (o < MLP_OUT * MLP_H) {
            const int j = o / MLP_H, k = o % MLP_H;
            for (int t = 0; t < nt; ++t) s = fmaf(dyb[t][j], buf[t * TR_LD + k], s);
            g[P_W4 + o] = s;
        } else {
            const int j = o - MLP_OUT * MLP_H;
            for (int t = 0; t < nt; ++t) s += dyb[t][j];
            g[P_B4 + j] = s;
        }
    }
    // dz3 = (W4^T dy) gelu'(z3), in place of z3
    if (live) {
        for (int k = 0; k < MLP_H; ++k) {
            float d = 0.0f;
#pragma unroll
            for (int j = 0; j < MLP_OUT; ++j) d = fmaf(P[P_W4 + MLP_H * j + k], dy[j], d);
            z3[tid * TR_LD + k] = d * gelu_d(z3[tid * TR_LD + k]);
        }
    } else {
        for (int k = 0; k < MLP_H; ++k) z3[tid * TR_LD + k] = 0.0f;
    }
    __syncthreads();  // buf (a3) consumed; dz3 complete
    for (int k = 0; k < MLP_H; ++k) buf[tid * TR_LD + k] = live ? gelu_f(z2[tid * TR_LD + k]) : 0.0f;  // a2
    __syncthreads();
    weight_grads(z3, buf, MLP_H, nt, g, P_W3, P_B3, tid);
    // dz2 = (W3^T dz3) gelu'(z2), in place of z2
    if (live) {
        float d3[MLP_H];
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) d3[k] = z3[tid * TR_LD + k];
        for (int i = 0; i < MLP_H; ++i) {
            float d = 0.0f;
#pragma unroll
            for (int k = 0; k < MLP_H; ++k) d = fmaf(P[P_W3 + MLP_H * k + i], d3[k], d);
            z2[tid * TR_LD + i] = d * gelu_d(z2[tid * TR_LD + i]);
        }
    } else {
        for (int k = 0; k < MLP_H; ++k) z2[tid * TR_LD + k] = 0.0f;
    }
    __syncthreads();  // buf (a2) consumed by the layer-3 gradients; dz2 complete
    for (int k = 0; k < MLP_H; ++k) buf[tid * TR_LD + k] = live ? gelu_f(z1[tid * TR_LD + k]) : 0.0f;  // a1
    __syncthreads();
    weight_grads(z2, buf, MLP_H, nt, g, P_W2, P_B2, tid);
    if (live) {
        float d2[MLP_H];
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) d2[k] = z2[tid * TR_LD + k];
        for (int i = 0; i < MLP_H; ++i) {
            float d = 0.0f;
#pragma unroll
            for (int k = 0; k < MLP_H; ++k) d = fmaf(P[P_W2 + MLP_H * k + i], d2[k], d);
            z1[tid * TR_LD + i] = d * gelu_d(z1[tid * TR_LD + i]);
        }
    } else {
        for (int k = 0; k < MLP_H; ++k) z1[tid * TR_LD + k] = 0.0f;
    }
    __syncthreads();  // buf (a1) consumed; dz1 complete
    {
        float gf[MLP_IN];
        mlp_features(xin[0], xin[1], gf);
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) buf[tid * TR_LD + i] = live ? gf[i] : 0.0f;
    }
    __syncthreads();
    weight_grads(z1, buf, MLP_IN, nt, g, P_W1, P_B1, tid);
}

// grad[p] = scale * sum over CTAs (in order) of gpart[cta][p]; loss = scale * sum of lpart (float64 sums)
__global__ void bp_mlp_reduce_kernel(const float* __restrict__ gpart, const float* __restrict__ lpart, int n_cta,
                                     float scale, float* __restrict__ grad, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N_PARAMS) {
        double s = 0.0;
        for (int c = 0; c < n_cta; ++c) s += (double)gpart[(size_t)c * N_PARAMS + p];
        grad[p] = (float)(s * scale);
    }
    if (p == 0 && loss) {
        double s = 0.0;
        for (int c = 0; c < n_cta; ++c) s += (double)lpart[c];
        *loss = (float)(s * scale);
    }
}

// Adam (Kingma and Ba): m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2, p -= lr mhat / (sqrt(vhat) + eps) with
// the bias corrections of step `step` (1-based).
__global__ void bp_adam_kernel(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                               float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N_PARAMS) return;
    const float g = grad[p];
    const float mm = fmaf(b1, m[p], (1.0f - b1) * g), vv = fmaf(b2, v[p], (1.0f - b2) * g * g);
    m[p] = mm, v[p] = vv;
    params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

extern "C" int bp_mlp_grad_ctas(int n) { return n < 1 ? 0 : (n + TR_T - 1) / TR_T; }

static size_t mlp_grad_smem() { return (((size_t)N_PARAMS + 3) & ~(size_t)3) * 4 + 4 * (size_t)TR_ARR * 4; }

extern "C" int bp_mlp_grad(const float* params, const float* x, const float* target, int n, float vweight,
                           float cweight, float* gpart, float* lpart, void* stream) {
    if (!params || !x || !target || !gpart || !lpart || n < 1 || !(vweight > 0) || !(cweight >= 0)) return BP_E_ARG;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mlp_grad_smem()) != cudaSuccess)
            return BP_E_LAUNCH;
        configured[dev] = true;
    }
    bp_mlp_grad_kernel<<<bp_mlp_grad_ctas(n), TR_T, mlp_grad_smem(), static_cast<cudaStream_t>(stream)>>>(
        params, x, target, n, vweight, cweight, gpart, lpart);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

extern "C" int bp_mlp_reduce(const float* gpart, const float* lpart, int n_cta, float scale, float* grad, float* loss,
                             void* stream) {
    if (!gpart || !lpart || !grad || n_cta < 1) return BP_E_ARG;
    bp_mlp_reduce_kernel<<<(N_PARAMS + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(gpart, lpart, n_cta,
                                                                                              scale, grad, loss);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

extern "C" int bp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
                       float eps, int step, void* stream) {
    if (!params || !grad || !m || !v || step < 1) return BP_E_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    bp_adam_kernel<<<(N_PARAMS + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grad, m, v, lr, beta1,
                                                                                       beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// Network outputs for inputs x [n][2] (f^, b^) -> y [n][16] (the quaternion part normalised to unit length):
// inference for checks.
__global__ void __launch_bounds__(128) bp_mlp_eval_kernel(const float* __restrict__ params, const float* __restrict__ x,
                                                         int n, float* __restrict__ y) {
    __shared__ float P[N_PARAMS];
    for (int i = threadIdx.x; i < N_PARAMS; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float xin[MLP_X] = {x[MLP_X * t], x[MLP_X * t + 1]};
    float o[MLP_OUT];
    mlp_forward_row(P, xin, nullptr, nullptr, nullptr, o);
    const float inv = rsqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2] + o[3] * o[3]);
#pragma unroll
    for (int j = 0; j < MLP_OUT; ++j) y[MLP_OUT * (size_t)t + j] = j < 4 ? o[j] * inv : o[j];
}

extern "C" int bp_mlp_eval(const float* params, const float* x, int n, float* y, void* stream) {
    if (!params || !x || !y || n < 0) return BP_E_ARG;
    if (n == 0) return BP_OK;
    bp_mlp_eval_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(params, x, n, y);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// ---- inference: one pulse occurrence applied to every spin's state ----
struct PulseArgs {
    const float* spins;   // [8][n]
    float* state;         // [6][n] in/out
    const float* params;  // the pulse's network
    const SegRec* segs;   // the occurrence's segments for the fallback: segs[seg0 .. seg0 + k_steps)
    int seg0, k_steps, n;
    double T, gz, thickness, z0, phi0;  // duration [s], slice gradient [Hz/m], thickness [m], centre [m], RF phase
    float b0off;          // the occurrence's uniform off-resonance [Hz]
    int* counts;          // null or [2]: spins through the network, spins through the fallback
    float dom_df, dom_b1, dom_z;  // the network's training domain
    double fmax;                  // dom_df + |gz| dom_z thickness: the scale of the input f^
};

// The network's inputs (f^, b^) of a spin (f^ clamped to [-1, 1]: rows outside the domain, whose outputs are not
// used, stay finite).
__device__ __forceinline__ void pulse_inputs(const PulseArgs& a, const Spin& p, float df, float x[MLP_X]) {
    const float fh = (float)(((double)df + a.gz * ((double)p.pz - a.z0)) / a.fmax);
    x[0] = fminf(fmaxf(fh, -1.f), 1.f);
    x[1] = fminf(fmaxf((p.b1 - 1.0f) / a.dom_b1, -1.f), 1.f);
}

// The plain sub-stepped pulse for spin j (the fallback outside the domain).
__device__ __forceinline__ void fallback_spin(const PulseArgs& a, int j) {
    const Spin p = load_spin(a.spins, a.n, j, true);
    float mx = a.state[j], my = a.state[a.n + j], mz = a.state[2 * a.n + j];
    float lx = a.state[3 * a.n + j], ly = a.state[4 * a.n + j], lz = a.state[5 * a.n + j];
    RfRelax rr{1.f, 1.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < a.k_steps; ++k) {
        const SegRec q = a.segs[a.seg0 + k];
        if (k == 0 || !(q.flags & BP_SAME_RFDT)) rr = rf_relax(q.dt, p);
        rf_step(q, p, rr, mx, my, mz, lx, ly, lz);
    }
    a.state[j] = mx, a.state[a.n + j] = my, a.state[2 * a.n + j] = mz;
    a.state[3 * a.n + j] = lx, a.state[4 * a.n + j] = ly, a.state[5 * a.n + j] = lz;
}

// sin and cos of a float64 angle to float32: reduced to [-pi, pi] in float64, then sincosf.
__device__ __forceinline__ void sincos_reduced(double x, float* s, float* c) {
    sincosf((float)(x - 2.0 * M_PI * rint(x * (0.5 / M_PI))), s, c);
}

__device__ __forceinline__ void quat_mul_f(const float a[4], const float b[4], float o[4]) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

// The network's outputs y (the reduced quaternion, dA~ / T, dC~ / T) applied to one spin's state (m + l):
// R = Rz(a1) R~ Rz(a2), dA = Rz(a1) dA~ Rz(a2), dC = Rz(a1) dC~ with a1 = wz/2 + phi0, a2 = wz/2 - phi0 and
// wz = -2 pi (G z + df) T (half angles in float64); then m -> E (R - (r2 - r1) dA)(E m + c) + c + r1 pd dC, E and c
// the exact relaxation and recovery of half the pulse: the pulse's map to first order in the relaxation rates
// beyond the relax / rotate / relax splitting (exact in the splitting's exponentials).
__device__ __forceinline__ void apply_pulse_map(const float* y, const PulseArgs& a, const Spin& p, float df,
                                                float& mx, float& my, float& mz, float& lx, float& ly, float& lz) {
    const float inv = rsqrtf(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
    const float qr[4] = {y[0] * inv, y[1] * inv, y[2] * inv, y[3] * inv};
    const double half = -M_PI * ((double)a.gz * (double)p.pz + (double)df) * a.T;
    float s1, c1, s2, c2;
    sincos_reduced(0.5 * (half + a.phi0), &s1, &c1);
    sincos_reduced(0.5 * (half - a.phi0), &s2, &c2);
    const float qa[4] = {c1, 0.f, 0.f, s1}, qb[4] = {c2, 0.f, 0.f, s2};
    float t4[4], q[4];
    quat_mul_f(qa, qr, t4);
    quat_mul_f(t4, qb, q);
    const float s = q[0], x = q[1], yq = q[2], z = q[3];
    float R[9] = {1 - 2 * (yq * yq + z * z), 2 * (x * yq - s * z), 2 * (x * z + s * yq),
                  2 * (x * yq + s * z), 1 - 2 * (x * x + z * z), 2 * (yq * z - s * x),
                  2 * (x * z - s * yq), 2 * (yq * z + s * x), 1 - 2 * (x * x + yq * yq)};
    // the full angles' cos / sin from the half angles
    const float C1 = fmaf(c1, c1, -s1 * s1), S1 = 2.0f * s1 * c1, C2 = fmaf(c2, c2, -s2 * s2), S2 = 2.0f * s2 * c2;
    const float T = (float)a.T;
    const float k = -(p.r2 - p.r1) * T;  // M = R + k dA~' (dA~' = Rz(a1) (dA~ / T) Rz(a2))
    float X[9];  // X = (dA~ / T) Rz(a2): columns 0 and 1 turn
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float d0 = y[4 + 3 * r], d1 = y[5 + 3 * r];
        X[3 * r] = fmaf(d0, C2, d1 * S2);
        X[3 * r + 1] = fmaf(-d0, S2, d1 * C2);
        X[3 * r + 2] = y[6 + 3 * r];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {  // Rz(a1) X: rows 0 and 1 turn; M = R + k Rz(a1) X
        const float a0 = fmaf(C1, X[c], -S1 * X[3 + c]), a1 = fmaf(S1, X[c], C1 * X[3 + c]);
        R[c] = fmaf(k, a0, R[c]);
        R[3 + c] = fmaf(k, a1, R[3 + c]);
        R[6 + c] = fmaf(k, X[6 + c], R[6 + c]);
    }
    const float th = 0.5f * T;
    const float e1 = expm1f(-th * p.r1), e2 = expm1f(-th * p.r2);
    const float ax = (mx + lx) * (1.0f + e2), ay = (my + ly) * (1.0f + e2);
    const float az = fmaf((mz + lz) - p.pd, e1, mz + lz);
    const float nx = fmaf(R[0], ax, fmaf(R[1], ay, R[2] * az));
    const float ny = fmaf(R[3], ax, fmaf(R[4], ay, R[5] * az));
    const float nz = fmaf(R[6], ax, fmaf(R[7], ay, R[8] * az));
    const float g = p.r1 * p.pd * T;  // r1 pd dC = r1 pd T Rz(a1) (dC~ / T)
    mx = fmaf(g, fmaf(C1, y[13], -S1 * y[14]), nx * (1.0f + e2));
    my = fmaf(g, fmaf(S1, y[13], C1 * y[14]), ny * (1.0f + e2));
    mz = fmaf(g, y[15], fmaf(nz - p.pd, e1, nz));
    lx = ly = lz = 0.0f;
}

__global__ void __launch_bounds__(128) bp_surrogate_pulse_kernel(PulseArgs a) {
    __shared__ float P[N_PARAMS];
    for (int i = threadIdx.x; i < N_PARAMS; i += blockDim.x) P[i] = a.params[i];
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = j < a.n;
    const int jj = active ? j : 0;
    const Spin p = load_spin(a.spins, a.n, jj, active);
    const float df = p.db0 + a.b0off;
    const float zr = (float)(((double)p.pz - a.z0) / a.thickness);
    const bool inside = fabsf(df) <= a.dom_df && fabsf(p.b1 - 1.0f) <= a.dom_b1 && fabsf(zr) <= a.dom_z;
    if (a.counts) {
        const unsigned in_mask = __ballot_sync(0xffffffffu, active && inside);
        const unsigned out_mask = __ballot_sync(0xffffffffu, active && !inside);
        if ((threadIdx.x & 31) == 0) {
            if (in_mask) atomicAdd(&a.counts[0], __popc(in_mask));
            if (out_mask) atomicAdd(&a.counts[1], __popc(out_mask));
        }
    }
    if (!active) return;
    float mx = a.state[j], my = a.state[a.n + j], mz = a.state[2 * a.n + j];
    float lx = a.state[3 * a.n + j], ly = a.state[4 * a.n + j], lz = a.state[5 * a.n + j];
    if (inside) {
        float xin[MLP_X];
        pulse_inputs(a, p, df, xin);
        float y[MLP_OUT];
        mlp_forward_row(P, xin, nullptr, nullptr, nullptr, y);
        apply_pulse_map(y, a, p, df, mx, my, mz, lx, ly, lz);
    } else {  // the fallback: the plain sub-stepped pulse
        RfRelax rr{1.f, 1.f, 0.f, 0.f, 0.f, 0.f};
        for (int k = 0; k < a.k_steps; ++k) {
            const SegRec q = a.segs[a.seg0 + k];
            if (k == 0 || !(q.flags & BP_SAME_RFDT)) rr = rf_relax(q.dt, p);
            rf_step(q, p, rr, mx, my, mz, lx, ly, lz);
        }
    }
    a.state[j] = mx, a.state[a.n + j] = my, a.state[2 * a.n + j] = mz;
    a.state[3 * a.n + j] = lx, a.state[4 * a.n + j] = ly, a.state[5 * a.n + j] = lz;
}

extern "C" int bp_surrogate_pulse(const float* spins, float* state, int n, const float* params, const void* segs,
                                  int seg0, int k_steps, double T, double gz, double thickness, double z0, double phi0,
                                  float b0off, float dom_df, float dom_b1, float dom_z, int32_t* counts,
                                  void* stream) {
    if (!spins || !state || !params || !segs || n < 1 || seg0 < 0 || k_steps < 1 || T <= 0 || thickness <= 0 ||
        !(dom_df > 0) || !(dom_b1 > 0) || !(dom_z > 0))
        return BP_E_ARG;
    PulseArgs a{spins, state, params, static_cast<const SegRec*>(segs), seg0, k_steps, n, T, gz, thickness, z0, phi0,
                b0off, counts, dom_df, dom_b1, dom_z, dom_df + fabs(gz) * dom_z * thickness};
    bp_surrogate_pulse_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// ---- inference on the tensor cores: all four layers as tcgen05 matrix products ----
//
// Per CTA tile of 128 spins (thread t = spin row t = tensor-memory lane t), four rounds, one per layer: every
// thread stores its row of the layer's input, split into bfloat16 high and low parts, as the A operand (K-major),
// one thread issues D = A_hi W_hi^T + A_hi W_lo^T + A_lo W_hi^T (M = 128, float32 accumulation in tensor memory),
// and every thread reads its row of D back (tcgen05.ld) and adds the bias (and GELU for layers 1 to 3):
//   layer 1: the 14 input features, zero-padded to K = 16 (one K step), N = 64, D in columns [0, 64);
//   layers 2 and 3: K = 64 (4 steps), N = 64, D in columns [0, 64);
//   layer 4: K = 64, N = 16, D in columns [64, 80).
// Shared memory: W2 hi, W2 lo, W3 hi, W3 lo (8192 bytes each, [0, 32768)), W1 hi, W1 lo ([32768, 36864)), W4 hi,
// W4 lo ([36864, 40960)), A hi and A lo (16384 each, [40960, 73728)), the fallback queue, mbarriers. The biases
// travel in the kernel's arguments (the constant bank). Layout of every operand: core matrices of 8 rows x 16
// bytes, K-adjacent ones 128 bytes apart, 8-row groups 1024 bytes apart (W1: 256, its rows being 16 wide); a thread
// writes its row 16 bytes at a time, so the 8 lanes of each store phase fill one 128-byte line.
#include "tcgen05.cuh"

#define SI_W_BYTES 8192                         // W2 or W3, one half (hi or lo)
#define SI_W1_BYTES 2048                        // W1 (64 x 16), one half
#define SI_W4_BYTES 2048                        // W4 (16 x 64), one half
#define SI_OFF_W1 (4 * SI_W_BYTES)              // 32768
#define SI_OFF_W4 (SI_OFF_W1 + 2 * SI_W1_BYTES) // 36864
#define SI_WT_BYTES (SI_OFF_W4 + 2 * SI_W4_BYTES)  // 40960: every weight tile, one bulk copy
#define SI_OFF_A SI_WT_BYTES
#define SI_A_BYTES 16384
#define SI_OFF_LIST (SI_OFF_A + 2 * SI_A_BYTES)  // queued fallback spins (256 ints), after the A operand
#define SI_LIST 256
#define SI_OFF_BAR (SI_OFF_LIST + SI_LIST * 4)
#define SI_SMEM (SI_OFF_BAR + 64)
#define SI_LBO 128
#define SI_SBO 1024
#define SI_SBO_W1 256
#define SI_COLS 128   // tensor-memory columns: D of layers 1 to 3 in [0, 64), of layer 4 in [64, 80)
#define SI_D4 64
#define SI_K1 16      // layer 1's K: the features, zero-padded

static_assert(SI_OFF_A % 1024 == 0 && SI_OFF_W1 % 16 == 0 && SI_OFF_W4 % 16 == 0, "operand alignment");
static_assert(MLP_IN <= SI_K1, "layer 1 fits one K step");

// NCH x 8 values of this thread's row -> A hi and A lo rows, chunks [chunk0, chunk0 + NCH) (16-byte stores)
template <int NCH>
__device__ __forceinline__ void store_row_bf16x2(unsigned char* ahi, unsigned char* alo, int row, const float* v,
                                                 int chunk0) {
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {  // a pair: hi = bf16(v) (nearest), lo = bf16(v - hi), two values per conversion
            const float v0 = v[8 * c + 2 * w], v1 = v[8 * c + 2 * w + 1];
            const __nv_bfloat162 hp = __floats2bfloat162_rn(v0, v1);
            const float2 hf = __bfloat1622float2(hp);
            const __nv_bfloat162 lp = __floats2bfloat162_rn(v0 - hf.x, v1 - hf.y);
            h[w] = *reinterpret_cast<const uint32_t*>(&hp);
            l[w] = *reinterpret_cast<const uint32_t*>(&lp);
        }
        const uint32_t off = (uint32_t)((row >> 3) * SI_SBO + (chunk0 + c) * SI_LBO + (row & 7) * 16);
        *reinterpret_cast<uint4*>(ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

// The network's biases, passed by value in the kernel's arguments (832 bytes of the constant bank; every thread
// reads the same bias at the same time): b1, b2, b3 (64 each), then b4 (16).
struct SmallNet {
    float bias[3 * MLP_H + MLP_OUT];
};

struct PulseMmaArgs {
    PulseArgs p;            // (p.params unused: the biases are in net, the weights in wtiles)
    const uint8_t* wtiles;  // SI_WT_BYTES: W2 hi, W2 lo, W3 hi, W3 lo, W1 hi, W1 lo, W4 hi, W4 lo (bp_mlp_wtiles)
    int* status;
    SmallNet net;
};

// (__grid_constant__: the biases are indexed in place in the parameter space, not copied to the stack)
__global__ void __launch_bounds__(128, 3) bp_surrogate_pulse_mma_kernel(const __grid_constant__ PulseMmaArgs args) {
    extern __shared__ __align__(1024) unsigned char smb[];
    const PulseArgs& a = args.p;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smb + SI_OFF_BAR);  // [0] weights, [1] MMA
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smb + SI_OFF_BAR + 2 * sizeof(uint64_t));
    int* queued = reinterpret_cast<int*>(smb + SI_OFF_BAR + 3 * sizeof(uint64_t));
    int* flist = reinterpret_cast<int*>(smb + SI_OFF_LIST);
    unsigned char* ahi = smb + SI_OFF_A;
    unsigned char* alo = smb + SI_OFF_A + SI_A_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sW = smem_u32(smb), sA = smem_u32(ahi);

    const float* bias = args.net.bias;
    if (tid == 0) {
        *queued = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[0], SI_WT_BYTES);
        tma_load_1d(smb, args.wtiles, SI_WT_BYTES, &bars[0]);
    }
    if (warp == 0) tmem_alloc(tmem_slot, SI_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);

    uint32_t mma_phase = 0;
    bool w_ready = false, fail = false, err = false, mma_out = false;
    const int n_tiles = (a.n + 127) / 128;

    for (int tile = blockIdx.x; tile < n_tiles && !fail; tile += gridDim.x) {
        const int j0 = tile * 128 + tid;
        const bool active = j0 < a.n;
        const int j = active ? j0 : 0;
        const Spin p = load_spin(a.spins, a.n, j, active);
        const float df = p.db0 + a.b0off;
        const float zr = (float)(((double)p.pz - a.z0) / a.thickness);
        const bool inside = active && fabsf(df) <= a.dom_df && fabsf(p.b1 - 1.0f) <= a.dom_b1 && fabsf(zr) <= a.dom_z;
        float y[MLP_OUT];
        {   // layer 1's input: the features, zero-padded to 16, as the A operand's first two chunks
            float xin[MLP_X], g[SI_K1];
            pulse_inputs(a, p, df, xin);
            mlp_features(xin[0], xin[1], g);
#pragma unroll
            for (int i = MLP_IN; i < SI_K1; ++i) g[i] = 0.0f;
            store_row_bf16x2<SI_K1 / 8>(ahi, alo, tid, g, 0);
        }
#pragma unroll 1
        for (int layer = 0; layer < 4; ++layer) {  // a real loop: one copy of the code serves the four layers
            fence_proxy_async_smem();
            tc_fence_before();
            if (__syncthreads_or(err)) {
                fail = true;
                break;
            }
            if (tid == 0) {
                if (!w_ready && !mbar_wait_bounded(&bars[0], 0)) err = true;
                w_ready = true;
                if (!err) {
                    tc_fence_after();
                    const uint32_t wh = layer == 0 ? sW + SI_OFF_W1
                                      : layer == 3 ? sW + SI_OFF_W4
                                                   : sW + (uint32_t)(2 * (layer - 1)) * SI_W_BYTES;
                    const uint32_t wl = wh + (layer == 0 ? SI_W1_BYTES : layer == 3 ? SI_W4_BYTES : SI_W_BYTES);
                    const uint32_t sbo_w = layer == 0 ? SI_SBO_W1 : SI_SBO;
                    const uint32_t idesc = umma_idesc_bf16_f32(128, layer == 3 ? MLP_OUT : MLP_H);
                    const uint32_t d = tmem + (layer == 3 ? SI_D4 : 0u);
                    uint64_t ah_d = umma_desc(sA, SI_LBO, SI_SBO), al_d = umma_desc(sA + SI_A_BYTES, SI_LBO, SI_SBO);
                    uint64_t bh_d = umma_desc(wh, SI_LBO, sbo_w), bl_d = umma_desc(wl, SI_LBO, sbo_w);
                    const int k_steps = layer == 0 ? SI_K1 / 16 : MLP_H / 16;
                    for (int kk = 0; kk < k_steps; ++kk) {
                        umma_bf16(d, ah_d, bh_d, idesc, kk > 0 ? 1u : 0u);
                        umma_bf16(d, ah_d, bl_d, idesc, 1u);
                        umma_bf16(d, al_d, bh_d, idesc, 1u);
                        ah_d += 2 * SI_LBO / 16, al_d += 2 * SI_LBO / 16, bh_d += 2 * SI_LBO / 16, bl_d += 2 * SI_LBO / 16;
                    }
                    umma_commit(&bars[1]);
                }
            }
            mma_out = true;
            if (mbar_wait_bounded(&bars[1], mma_phase)) {
                mma_phase ^= 1u;
                mma_out = false;
            } else {
                err = true;
            }
            if (__syncthreads_or(err)) {
                fail = true;
                break;
            }
            tc_fence_after();
            if (layer < 3) {
                // the layer's output 16 columns at a time: bias and GELU, split straight into the next A operand
                // (the MMA that read the A operand has completed)
                const float* b = bias + layer * MLP_H;
#pragma unroll 1
                for (int c0 = 0; c0 < MLP_H; c0 += 16) {
                    float d[16];
                    tmem_ld16(lane_addr + (uint32_t)c0, d);
                    tmem_ld_wait();
#pragma unroll
                    for (int i = 0; i < 16; ++i) d[i] = gelu_f(d[i] + b[c0 + i]);
                    store_row_bf16x2<2>(ahi, alo, tid, d, c0 / 8);
                }
            } else {
                float d[16];
                tmem_ld16(lane_addr + (uint32_t)SI_D4, d);
                tmem_ld_wait();
#pragma unroll
                for (int o = 0; o < MLP_OUT; ++o) y[o] = d[o] + bias[3 * MLP_H + o];
            }
            tc_fence_before();
        }
        if (fail) break;
        if (inside) {
            float mx = a.state[j], my = a.state[a.n + j], mz = a.state[2 * a.n + j];
            float lx = a.state[3 * a.n + j], ly = a.state[4 * a.n + j], lz = a.state[5 * a.n + j];
            apply_pulse_map(y, a, p, df, mx, my, mz, lx, ly, lz);
            a.state[j] = mx, a.state[a.n + j] = my, a.state[2 * a.n + j] = mz;
            a.state[3 * a.n + j] = lx, a.state[4 * a.n + j] = ly, a.state[5 * a.n + j] = lz;
        }
        // spins outside the domain join the CTA's queue; whenever it holds 128, all threads step them (full warps
        // whatever the spins' order)
        const unsigned in_mask = __ballot_sync(0xffffffffu, inside);
        const unsigned out_mask = __ballot_sync(0xffffffffu, active && !inside);
        if (a.counts && (tid & 31) == 0) {
            if (in_mask) atomicAdd(&a.counts[0], __popc(in_mask));
            if (out_mask) atomicAdd(&a.counts[1], __popc(out_mask));
        }
        if (out_mask) {
            int base = 0;
            if ((tid & 31) == 0) base = atomicAdd(queued, __popc(out_mask));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (active && !inside) flist[base + __popc(out_mask & ((1u << (tid & 31)) - 1u))] = j;
        }
        __syncthreads();
        const int nq = *queued;
        if (nq >= 128) {
            fallback_spin(a, flist[nq - 128 + tid]);
            __syncthreads();
            if (tid == 0) *queued = nq - 128;
        }
        __syncthreads();
    }
    if (!fail && tid < *queued) fallback_spin(a, flist[tid]);
    // leave no copy or MMA in flight (failure paths), then free the tensor memory
    if (tid == 0 && !w_ready) mbar_wait_bounded(&bars[0], 0);
    if (mma_out) mbar_wait_bounded(&bars[1], mma_phase);
    if ((fail || err) && tid == 0 && args.status) atomicOr(args.status, BP_ERR_TMA_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, SI_COLS);
    }
}

// The weights -> bfloat16 high / low tiles in the operand layout, row n (output unit), column k (input unit):
//   W2, W3 (64 x 64): element (n / 8) 512 + (k / 8) 64 + (n % 8) 8 + k % 8 of tiles 0-1 (W2 hi, lo) and 2-3 (W3);
//   W1 (64 x 16, columns 14 and 15 zero): element (n / 8) 128 + (k / 8) 64 + (n % 8) 8 + k % 8 of tiles 4-5;
//   W4 (16 x 64): as W2, of tiles 6-7.
#define WT_N23 (2 * MLP_H * MLP_H)
#define WT_N1 (MLP_H * SI_K1)
#define WT_N4 (MLP_OUT * MLP_H)
__global__ void bp_mlp_wtiles_kernel(const float* __restrict__ params, uint16_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= WT_N23 + WT_N1 + WT_N4) return;
    uint16_t h, lo;
    int base, half, e;
    if (i < WT_N23) {
        const int l = i / (MLP_H * MLP_H), r = i % (MLP_H * MLP_H), n = r / MLP_H, k = r % MLP_H;
        split_bf16(params[(l ? P_W3 : P_W2) + r], h, lo);
        base = 2 * l * (SI_W_BYTES / 2), half = SI_W_BYTES / 2;
        e = (n >> 3) * 512 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
    } else if (i < WT_N23 + WT_N1) {
        const int r = i - WT_N23, n = r / SI_K1, k = r % SI_K1;
        split_bf16(k < MLP_IN ? params[P_W1 + MLP_IN * n + k] : 0.0f, h, lo);
        base = SI_OFF_W1 / 2, half = SI_W1_BYTES / 2;
        e = (n >> 3) * 128 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
    } else {
        const int r = i - WT_N23 - WT_N1, n = r / MLP_H, k = r % MLP_H;
        split_bf16(params[P_W4 + r], h, lo);
        base = SI_OFF_W4 / 2, half = SI_W4_BYTES / 2;
        e = (n >> 3) * 512 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
    }
    out[base + e] = h;
    out[base + half + e] = lo;
}

extern "C" int bp_mlp_wtiles_bytes(void) { return SI_WT_BYTES; }

extern "C" int bp_mlp_wtiles(const float* params, void* tiles, void* stream) {
    if (!params || !tiles) return BP_E_ARG;
    if ((reinterpret_cast<uintptr_t>(tiles) & 15) != 0) return BP_E_ALIGN;
    bp_mlp_wtiles_kernel<<<(WT_N23 + WT_N1 + WT_N4 + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        params, static_cast<uint16_t*>(tiles));
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// CTAs of bp_surrogate_pulse_mma for n spins: one per 128-spin tile up to the SMs x the residency by shared memory
// (with the per-block reservation), registers, threads and tensor memory (512 columns per SM).
static int pulse_mma_grid(int n, int max_ctas, int* grid_out) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    static bool configured[64] = {false};
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_surrogate_pulse_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SI_SMEM) != cudaSuccess ||
            cudaFuncSetAttribute(bp_surrogate_pulse_mma_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return BP_E_LAUNCH;
        configured[dev] = true;
    }
    int smem_sm = 0, smem_res = 0, regs_sm = 0, thr_sm = 0;
    cudaFuncAttributes fa;
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, bp_surrogate_pulse_mma_kernel) != cudaSuccess)
        return BP_E_LAUNCH;
    int per_sm = smem_sm / (SI_SMEM + smem_res);
    const int regs_block = ((fa.numRegs * 32 + 255) / 256) * 256 * 4;
    if (regs_block > 0 && regs_sm / regs_block < per_sm) per_sm = regs_sm / regs_block;
    if (thr_sm / 128 < per_sm) per_sm = thr_sm / 128;
    if (per_sm > 512 / SI_COLS) per_sm = 512 / SI_COLS;
    if (per_sm < 1) per_sm = 1;
    const int n_tiles = (n + 127) / 128;
    int grid = sms * per_sm;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid > n_tiles) grid = n_tiles;
    *grid_out = grid;
    return BP_OK;
}

extern "C" int bp_surrogate_pulse_mma_grid(int n) {
    int grid = 0;
    if (n < 1) return -BP_E_ARG;
    const int code = pulse_mma_grid(n, 0, &grid);
    return code == BP_OK ? grid : -code;
}

extern "C" int bp_surrogate_pulse_mma(const float* spins, float* state, int n, const float* params_host,
                                      const void* wtiles, const void* segs, int seg0, int k_steps, double T, double gz,
                                      double thickness, double z0, double phi0, float b0off, float dom_df,
                                      float dom_b1, float dom_z, int32_t* counts, int32_t* status, int max_ctas,
                                      void* stream) {
    if (!spins || !state || !params_host || !wtiles || !segs || !status || n < 1 || seg0 < 0 || k_steps < 1 ||
        T <= 0 || thickness <= 0 || !(dom_df > 0) || !(dom_b1 > 0) || !(dom_z > 0))
        return BP_E_ARG;
    if ((reinterpret_cast<uintptr_t>(wtiles) & 15) != 0) return BP_E_ALIGN;
    int grid = 0;
    const int code = pulse_mma_grid(n, max_ctas, &grid);
    if (code != BP_OK) return code;
    PulseMmaArgs a{{spins, state, nullptr, static_cast<const SegRec*>(segs), seg0, k_steps, n, T, gz, thickness, z0,
                    phi0, b0off, counts, dom_df, dom_b1, dom_z, dom_df + fabs(gz) * dom_z * thickness},
                   static_cast<const uint8_t*>(wtiles), status, {}};
    std::memcpy(a.net.bias, params_host + P_B1, MLP_H * sizeof(float));
    std::memcpy(a.net.bias + MLP_H, params_host + P_B2, MLP_H * sizeof(float));
    std::memcpy(a.net.bias + 2 * MLP_H, params_host + P_B3, MLP_H * sizeof(float));
    std::memcpy(a.net.bias + 3 * MLP_H, params_host + P_B4, MLP_OUT * sizeof(float));
    bp_surrogate_pulse_mma_kernel<<<grid, 128, SI_SMEM, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}
