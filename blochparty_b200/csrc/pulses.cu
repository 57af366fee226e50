// Reused pulses (simulate(..., pulses="reuse")): a pulse of two or more RF segments that recurs, up to a global
// RF phase, is composed once per spin into its affine map m -> M m + v and applied at every occurrence, turned
// about z by the occurrence's phase phi: m -> Rz(phi) (M Rz(-phi) m + v). Relaxation and its recovery commute
// with rotations about z, and the rotation axes of the phase-shifted pulse are the original ones turned by phi,
// so the turned map is exact.
//
// Replaces blochparty's pulse maps (engines/gpu/cuda/pulse.cu.in:3-32 and the reuse branch of bloch_chunk_mma,
// engines/gpu/cuda/kernels.cu.in:141-165; occurrences found by engines/gpu/driver.py:112-164). Here the map is
// composed in float64 (the plain RF step: relax dt/2, Rodrigues rotation about w = -2 pi dt (b1 rf_x, b1 rf_y,
// G.r + dB0 + b0_offset), relax dt/2, with the phase of G.r from the float64 moments) and kept in float64, and the
// application works on the compensated state in float64: one occurrence costs 96 bytes of map and 48 bytes of
// state per spin (HBM-bound) instead of K RF steps.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "bloch_common.cuh"
#include "../../include/blochparty_b200.h"

// x += s1 (w x x) + s2 w x (w x x): the rotation about w of a float64 3-vector
__device__ __forceinline__ void rot_d(double wx, double wy, double wz, double s1, double s2, double& x, double& y,
                                      double& z) {
    const double cx = wy * z - wz * y, cy = wz * x - wx * z, cz = wx * y - wy * x;
    const double dx = wy * cz - wz * cy, dy = wz * cx - wx * cz, dz = wx * cy - wy * cx;
    x += s1 * cx + s2 * dx;
    y += s1 * cy + s2 * dy;
    z += s1 * cz + s2 * dz;
}

// Per spin: the affine map of segments [seg0, seg0 + k_steps) (all RF, a spoil zeroing the transverse part after its
// segment), maps [12][n] float64: M row-major, then v.
__global__ void bp_pulse_maps_kernel(const float* __restrict__ spins, int n, const SegRec* __restrict__ segs,
                                     const double4* __restrict__ seg64, int seg0, int k_steps,
                                     double* __restrict__ maps) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const Spin p = load_spin(spins, n, j, true);
    // columns of M (linear part) and v (the image of the zero state)
    double m[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};  // m[c] = column c
    double vx = 0.0, vy = 0.0, vz = 0.0;
    double a1 = 1.0, a2 = 1.0, e1h = 0.0;
    for (int k = 0; k < k_steps; ++k) {
        const SegRec q = segs[seg0 + k];
        const double4 k64 = seg64[seg0 + k];
        if (k == 0 || !(q.flags & BP_SAME_RFDT)) {
            e1h = expm1(-0.5 * (double)q.dt * (double)p.r1);
            a1 = 1.0 + e1h;
            a2 = 1.0 + expm1(-0.5 * (double)q.dt * (double)p.r2);
        }
        const double cz = -(double)p.pd * e1h;  // recovery of one half step
        const double cyc = fma(k64.x, (double)p.px,
                               fma(k64.y, (double)p.py, fma(k64.z, (double)p.pz, fma((double)q.dt, (double)p.db0, k64.w))));
        const double wx = (double)q.wx0 * (double)p.b1, wy = (double)q.wy0 * (double)p.b1;
        const double wz = -2.0 * M_PI * cyc;
        const double p2 = wx * wx + wy * wy + wz * wz;
        double s1, s2;
        if (p2 < 1e-8) {
            s1 = 1.0 - p2 / 6.0;
            s2 = 0.5 - p2 / 24.0;
        } else {
            const double phi = sqrt(p2);
            const double sh = sin(0.5 * phi) / phi;
            s1 = sin(phi) / phi;
            s2 = 2.0 * sh * sh;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double x = m[c][0] * a2, y = m[c][1] * a2, z = m[c][2] * a1;
            rot_d(wx, wy, wz, s1, s2, x, y, z);
            m[c][0] = x * a2, m[c][1] = y * a2, m[c][2] = z * a1;
        }
        double x = vx * a2, y = vy * a2, z = vz * a1 + cz;
        rot_d(wx, wy, wz, s1, s2, x, y, z);
        vx = x * a2, vy = y * a2, vz = z * a1 + cz;
        if (q.flags & BP_SPOIL) {  // the segment's spoil: no transverse magnetization leaves it
#pragma unroll
            for (int c = 0; c < 3; ++c) m[c][0] = m[c][1] = 0.0;
            vx = vy = 0.0;
        }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) maps[(size_t)(3 * r + c) * n + j] = m[c][r];
    maps[(size_t)9 * n + j] = vx, maps[(size_t)10 * n + j] = vy, maps[(size_t)11 * n + j] = vz;
}

// state (hi + lo) -> Rz(phi) (M Rz(-phi) m + v), in float64, written back as float32 hi + lo.
__global__ void bp_pulse_apply_kernel(const double* __restrict__ maps, int n, float* __restrict__ state, double c,
                                      double s) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double mx = (double)state[j] + (double)state[3 * n + j];
    const double my = (double)state[n + j] + (double)state[4 * n + j];
    const double mz = (double)state[2 * n + j] + (double)state[5 * n + j];
    const double ux = c * mx + s * my, uy = c * my - s * mx;  // Rz(-phi)
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        t[r] = fma(maps[(size_t)(3 * r) * n + j], ux,
                   fma(maps[(size_t)(3 * r + 1) * n + j], uy, fma(maps[(size_t)(3 * r + 2) * n + j], mz,
                                                                 maps[(size_t)(9 + r) * n + j])));
    const double ox = c * t[0] - s * t[1], oy = s * t[0] + c * t[1], oz = t[2];  // Rz(phi)
    const float hx = (float)ox, hy = (float)oy, hz = (float)oz;
    state[j] = hx, state[n + j] = hy, state[2 * n + j] = hz;
    state[3 * n + j] = (float)(ox - (double)hx), state[4 * n + j] = (float)(oy - (double)hy);
    state[5 * n + j] = (float)(oz - (double)hz);
}

extern "C" int bp_pulse_maps(const float* spins, int n, const void* segs, const double* seg64, int seg0, int k_steps,
                             double* maps, void* stream) {
    if (!spins || !segs || !seg64 || !maps || n < 1 || seg0 < 0 || k_steps < 1) return BP_E_ARG;
    bp_pulse_maps_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        spins, n, static_cast<const SegRec*>(segs), reinterpret_cast<const double4*>(seg64), seg0, k_steps, maps);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

extern "C" int bp_pulse_apply(const double* maps, int n, float* state, double phase, void* stream) {
    if (!maps || !state || n < 1) return BP_E_ARG;
    const double s = std::sin(phase), c = std::cos(phase);
    bp_pulse_apply_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(maps, n, state, c, s);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}
