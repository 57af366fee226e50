// Hand-written adjoint (reverse sweep) of the forward kernel, and the fixed-order reduction of its segment
// gradients. Replaces blochparty's bloch_replay / bloch_adjoint_c<NC> / seg_reduce
// (engines/gpu/cuda/replay.cu.in:3-33, adjoint.cu.in:5-121, seg_reduce.cu:3-11; the reverse of one segment is
// shaders/adjoint_common.metal:212-315) for static spins.
//
// Checkpointing has three levels. The forward stores the state at the start of every checkpoint interval. The
// backward replays one interval at a time with the forward kernel (no readout), storing the state at the start
// of every adjoint window (<= BP_ADJ_WIN segments, also cut at every run of like segments). This kernel then
// sweeps the interval's windows in reverse: per window it recomputes the window forward from its start state in
// plain float32, keeping the state after every segment in shared memory (one slot per segment and spin), and runs
// the segments backward from them. A window that is one RF run or one readout run takes a sweep without
// per-segment tests.
//
// Segment s maps the magnetization affinely, m_s = A_s m_{s-1} + b_s. With lambda = dL/dm after segment s
// (after its spoil), the sweep is lambda_{s-1} = A_s^T (P_s lambda + dL/dm of the sample), P_s the spoil
// projection; the parameter gradients of segment s follow from lambda and m_{s-1} (for an RF segment's rotation,
// through the rotation's left Jacobian). Per-spin gradients are running totals in registers through the interval;
// per-segment gradients are reduced over the warp by shuffles, over the CTA's warps in fixed order in shared
// memory, and written as one float32 partial per CTA and segment; bp_seg_reduce adds the CTAs' partials in fixed
// order in float64. No atomics: every run gives the same bits.
//
// Without per-spin gradients (the RF waveform's alone) the variant SG = false keeps no state slots: its windows of
// free segments carry lambda alone, its windows of RF segments integrate their states backward from the state
// after them (from the replay, or, in bp_adjoint_saved, from the state the forward saved after the pulse, carried
// from window to window of the pulse in registers), a sample's coil sum runs on paired FMAs over cotangent rows
// staged by TMA one window ahead, and its per-window shared buffers alternate by the window's parity, so a readout
// window needs a single barrier.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "bloch_common.cuh"
#include "physics.cuh"
#include "../../include/blochparty_b200.h"

#define ADJ_THREADS 128
#define ADJ_WARPS (ADJ_THREADS / 32)
#define ADJ_SLOTS (BP_ADJ_WIN + 1)
// !SG: the RF gradient of an interval of at most this many segments is summed over the CTA's tiles in shared memory
// ([ADJ_SACC_MAX][2] floats) and written to gseg once, instead of added to gseg after every window
#define ADJ_SACC_MAX 2048
// the sweep's own bits in a staged record's flags (above the record's): the segment before it (in the window)
// spoils; the segment after it (in the window, swept just before) shares its RF relaxation, its RF off-resonance,
// or its free factors, so the sweep keeps them
#define A_PREV_SPOIL (1 << 8)
#define A_KEEP_RELAX (1 << 9)
#define A_KEEP_WZ (1 << 10)
#define A_KEEP_FREE (1 << 11)
// (bits 0-6 are the record's own flags; BP_SMALL, bit 6, is not used by the sweep, which tests per warp)

// per-spin gradient rows of `gs`
enum { G_PX, G_PY, G_PZ, G_DB0, G_PD, G_R1, G_R2, G_B1, N_GS };
// per-segment gradient columns: with respect to the record's dt (its direct uses), -2 pi dt rf_x, -2 pi dt rf_y,
// the moments g dt, and b0_offset dt
enum { S_DT, S_WX, S_WY, S_KX, S_KY, S_KZ, S_BETA, N_SG = 8 };

struct AdjArgs {
    const float* spins;
    const float* sens;    // [16 ncg][n]
    const SegRec* segs;
    const double4* seg64;
    const int4* windows;  // adjoint windows
    int n, n_coils;
    int wa, wb;           // this interval's adjoint windows
    int seg0, seg_len;    // first segment of the interval, segments in it
    const float* wstates; // [wb - wa + 1][6][n] state at every window start, then after the last window (replay)
    const float* h;       // [n_adc][2C] dL/d(raw coil sums), or null
    int n_adc;            // rows of h
    float* lam;           // [3][n] in: dL/dm at the interval's end; out: at its start
    float* gs;            // [N_GS][n] += per-spin gradients
    float* gc;            // [2C][n] += coil gradients (rows 2c real, 2c+1 imaginary), or null
    float* gseg;          // [gridDim.x][seg_len][N_SG] per-CTA segment gradients, or null
    int seg_mask;         // which of the N_SG segment gradients are reduced (bit k: component k)
    int* status;          // |= BP_ERR_BAD_WINDOW for a window outside the interval (skipped)
    int grid_rows;        // rows of gseg (bp_adjoint's `grid`): a variant that launches fewer CTAs clears the rest
    // the field model (bp_adjoint_physics, variant PH): concomitant mode, per-spin coefficients [7][n], the segments'
    // dt-weighted gradient monomials [S][6] (mode 1), and the coefficients' gradient [7][n] (+=, or null)
    int conc_mode;
    const float* conc;
    const double* segq;
    float* gconc;
    // the sweep from saved states (bp_adjoint_saved; variant !SG): wstates holds states by slot and wslot[w] is the
    // slot of the state at window w's start (-1: not saved). A window of RF segments takes the state after it from
    // the window after it when that one was integrated backward too (its start state, carried in registers: the
    // chain), else from the slot of the next window's start. chain [3][n] carries the chain between calls: read at
    // the start when chain_in (window wb was integrated backward), written at the end (window wa's start state).
    const int* wslot;
    float* chain;
    int chain_in;
};

// Rodrigues factors of the rotation by |w| (p2 = |w|^2) with the third factor of its left Jacobian:
// c = cos phi, s1 = sin(phi)/phi, s2 = (1 - cos phi)/phi^2, s3 = (phi - sin phi)/phi^3 = (1 - s1)/p2. Below
// phi = 1 all are Taylor series in p2 (s3 = sum_k (-1)^k p2^k / (2k+3)!), truncated like rodrigues_coeffs (first
// dropped terms below 4e-13 under phi = 1/4, below 2e-10 under phi = 1).
// SMALL: the caller knows p2 < 1/16 (the first tier, no tests).
template <bool SMALL>
__device__ __forceinline__ void rot_factors(float p2, float& c, float& s1, float& s2, float& s3) {
    if (SMALL)
        rodrigues_small(p2, s1, s2);
    else
        rodrigues_coeffs(p2, s1, s2);
    c = fmaf(-s2, p2, 1.0f);
    if (SMALL || p2 < 0.0625f) {
        s3 = fmaf(p2, fmaf(p2, fmaf(p2, -2.7557319223985893e-06f, 1.9841269841269841e-04f), -8.3333333333333333e-03f),
                  1.6666666666666667e-01f);
    } else if (p2 < 1.0f) {
        s3 = fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, -1.6059043836821615e-10f, 2.5052108385441720e-08f),
                                              -2.7557319223985893e-06f), 1.9841269841269841e-04f),
                           -8.3333333333333333e-03f), 1.6666666666666667e-01f);
    } else {
        s3 = (1.0f - s1) / p2;
    }
}

struct SegGrad {
    float v[N_SG];
};

// dL/d(offset in cycles) `gc` of a segment: per-spin and per-segment parts (cyc = k.r + dt dB0 + beta)
__device__ __forceinline__ void offset_grads(float gcyc, const SegRec& q, const Spin& p, float* g, SegGrad& sg) {
    g[G_PX] = fmaf(gcyc, q.kx, g[G_PX]);
    g[G_PY] = fmaf(gcyc, q.ky, g[G_PY]);
    g[G_PZ] = fmaf(gcyc, q.kz, g[G_PZ]);
    g[G_DB0] = fmaf(gcyc, q.dt, g[G_DB0]);
    sg.v[S_KX] += gcyc * p.px;
    sg.v[S_KY] += gcyc * p.py;
    sg.v[S_KZ] += gcyc * p.pz;
    sg.v[S_BETA] += gcyc;
    sg.v[S_DT] += gcyc * p.db0;
}

// The field model in the sweep (variant PH): the spin's concomitant coefficients and the running totals of their
// gradients.
struct PhysSpin {
    int mode;
    Conc c;
    float gk[7];
};

// dL/d(segment phase in cycles) `gcyc` with the field model: the concomitant field's share goes to the spin's
// coefficients and to the segment's moments and dt, the rest (through the phase's dependence on the linear offset)
// to offset_grads. Leading order: phase = lin + c . Q, Q = (kx^2, ky^2, kz^2, kx ky, kx kz, ky kz) / dt, so
// dQ/dk and dQ/ddt (at fixed k) are the gradient monomials' derivatives; exact: phase = lin + E, E = sqrt(U^2 + T2)
// - U with U = f0 dt + lin and T2 = (ax . k)^2 + (ay . k)^2, dE/dU = -E / S, dE/dT = T / S (S = sqrt(U^2 + T2)).
// `sq`: the segment's dt-weighted monomials (mode 1).
template <bool PH>
__device__ __forceinline__ void phase_grads(float gcyc, const SegRec& q, const Spin& p, float* g, SegGrad& sg,
                                            PhysSpin* ps, const double* __restrict__ sq) {
    if constexpr (PH) {
        const Conc& c = ps->c;
        if (ps->mode == 1) {
            float conc = 0.0f;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const float qi = (float)sq[i];
                conc = fmaf(c.c[i], qi, conc);
                ps->gk[i] = fmaf(gcyc, qi, ps->gk[i]);
            }
            const float idt = q.dt > 0.0f ? 1.0f / q.dt : 0.0f;
            const float gx = q.kx * idt, gy = q.ky * idt, gz = q.kz * idt;
            sg.v[S_KX] += gcyc * fmaf(2.0f * c.c[0], gx, fmaf(c.c[3], gy, c.c[4] * gz));
            sg.v[S_KY] += gcyc * fmaf(2.0f * c.c[1], gy, fmaf(c.c[3], gx, c.c[5] * gz));
            sg.v[S_KZ] += gcyc * fmaf(2.0f * c.c[2], gz, fmaf(c.c[4], gx, c.c[5] * gy));
            sg.v[S_DT] -= gcyc * conc * idt;
        } else if (ps->mode == 2) {
            const float lin = fmaf(q.kx, p.px, fmaf(q.ky, p.py, fmaf(q.kz, p.pz, fmaf(q.dt, p.db0, q.beta))));
            const float tx = fmaf(c.c[0], q.kx, fmaf(c.c[1], q.ky, c.c[2] * q.kz));
            const float ty = fmaf(c.c[3], q.kx, fmaf(c.c[4], q.ky, c.c[5] * q.kz));
            const float t2 = fmaf(tx, tx, ty * ty);
            const float u = fmaf(c.c[6], q.dt, lin);
            const float sr = sqrtf(fmaf(u, u, t2));
            const float e = t2 > 0.0f ? t2 / (sr + u) : 0.0f;
            const float isr = sr > 0.0f ? 1.0f / sr : 0.0f;
            const float de_du = -e * isr, rx = tx * isr, ry = ty * isr;
            ps->gk[0] = fmaf(gcyc * rx, q.kx, ps->gk[0]);
            ps->gk[1] = fmaf(gcyc * rx, q.ky, ps->gk[1]);
            ps->gk[2] = fmaf(gcyc * rx, q.kz, ps->gk[2]);
            ps->gk[3] = fmaf(gcyc * ry, q.kx, ps->gk[3]);
            ps->gk[4] = fmaf(gcyc * ry, q.ky, ps->gk[4]);
            ps->gk[5] = fmaf(gcyc * ry, q.kz, ps->gk[5]);
            ps->gk[6] = fmaf(gcyc * de_du, q.dt, ps->gk[6]);
            sg.v[S_KX] += gcyc * fmaf(rx, c.c[0], ry * c.c[3]);
            sg.v[S_KY] += gcyc * fmaf(rx, c.c[1], ry * c.c[4]);
            sg.v[S_KZ] += gcyc * fmaf(rx, c.c[2], ry * c.c[5]);
            sg.v[S_DT] += gcyc * de_du * c.c[6];
            gcyc *= 1.0f + de_du;  // the linear offset's share
        }
    }
    offset_grads(gcyc, q, p, g, sg);
}

// The half-step relaxation of an RF segment as the sweep uses it: e1h = expm1(-dt r1 / 2), a1 = 1 + e1h (and
// e2h, a2 likewise), the inverses of a1 and a2, and whether they are safe to divide by (a >= 1/2: T1, T2 above
// 0.72 dt; otherwise the rotated state is formed from the segment's input instead).
struct RevRelax {
    float e1h, e2h, a1, a2, ia1, ia2;
    bool invert;
};

__device__ __forceinline__ RevRelax rev_relax(float dt, const Spin& p) {
    RevRelax r;
    r.e1h = expm1f(-0.5f * dt * p.r1);
    r.e2h = expm1f(-0.5f * dt * p.r2);
    r.a1 = 1.0f + r.e1h;
    r.a2 = 1.0f + r.e2h;
    r.invert = r.a1 >= 0.5f && r.a2 >= 0.5f;
    r.ia1 = r.invert ? 1.0f / r.a1 : 0.0f;
    r.ia2 = r.invert ? 1.0f / r.a2 : 0.0f;
    return r;
}

// An RF segment of the recompute in plain float32 (the states only feed the gradients, which need no
// compensated sums): m1 = E m + c, n = R m1 = c m1 + s1 (w x m1) + s2 w (w . m1), m = E n + c.
template <bool SMALL>
__device__ __forceinline__ void rf_step_plain(const SegRec& q, const Spin& p, const RevRelax& r, float wz, float& mx,
                                              float& my, float& mz) {
    const float wx = q.wx0 * p.b1, wy = q.wy0 * p.b1;
    const float m1x = mx * r.a2, m1y = my * r.a2, m1z = fmaf(mz - p.pd, r.e1h, mz);
    const float p2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
    float s1, s2;
    if (SMALL)
        rodrigues_small(p2, s1, s2);
    else
        rodrigues_coeffs(p2, s1, s2);
    const float c = fmaf(-s2, p2, 1.0f);
    const float k = s2 * fmaf(wx, m1x, fmaf(wy, m1y, wz * m1z));
    const float nx = fmaf(c, m1x, fmaf(s1, wy * m1z - wz * m1y, k * wx));
    const float ny = fmaf(c, m1y, fmaf(s1, wz * m1x - wx * m1z, k * wy));
    const float nz = fmaf(c, m1z, fmaf(s1, wx * m1y - wy * m1x, k * wz));
    mx = nx * r.a2, my = ny * r.a2, mz = fmaf(nz - p.pd, r.e1h, nz);
}

// A free segment of the recompute in plain float32: rotation about z by the factors' (float32) phase, relaxation.
__device__ __forceinline__ void free_step_plain(const FreeFactors& f, const Spin& p, float& mx, float& my, float& mz) {
    const float x = fmaf(f.ch, mx, -f.sh * my), y = fmaf(f.sh, mx, f.ch * my);
    mx = fmaf(x, f.e2, x), my = fmaf(y, f.e2, y), mz = fmaf(mz - p.pd, f.e1, mz);
}

// Reverse of an RF segment from its input state (x0, y0, z0) and output state (ox, oy, oz): lambda in/out,
// gradients accumulated. The rotated state n = R m1 comes from the output, m2 = E n + c, by E's inverse (or, with
// strong relaxation, from the input). dL/dw = J^T (n x a), a = dL/dn and J the rotation's left Jacobian
// (R(w + d) = exp([J d]x) R(w)): J^T u = s1 u - s2 (w x u) + s3 (w . u) w.
template <bool SMALL, bool OG, bool SG = true, bool PH = false>
__device__ __forceinline__ void rf_reverse(const SegRec& q, const Spin& p, const RevRelax& r, float wz, float x0,
                                           float y0, float z0, float ox, float oy, float oz, float& lx, float& ly,
                                           float& lz, float* g, SegGrad& sg, PhysSpin* ps = nullptr,
                                           const double* sq = nullptr) {
    const float h = 0.5f * q.dt;
    const float wx = q.wx0 * p.b1, wy = q.wy0 * p.b1;
    const float p2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
    float c, s1, s2, s3;
    rot_factors<SMALL>(p2, c, s1, s2, s3);
    const float a2 = r.a2, a1 = r.a1, e1h = r.e1h;
    float nx, ny, nz;
    if (r.invert) {
        nx = ox * r.ia2, ny = oy * r.ia2, nz = fmaf(p.pd, e1h, oz) * r.ia1;
    } else {
        const float m1x = x0 * a2, m1y = y0 * a2, m1z = fmaf(z0 - p.pd, e1h, z0);
        const float k = s2 * fmaf(wx, m1x, fmaf(wy, m1y, wz * m1z));
        nx = fmaf(c, m1x, fmaf(s1, wy * m1z - wz * m1y, k * wx));
        ny = fmaf(c, m1y, fmaf(s1, wz * m1x - wx * m1z, k * wy));
        nz = fmaf(c, m1z, fmaf(s1, wx * m1y - wy * m1x, k * wz));
    }
    // second half relaxation: m2 = (n a2, n a2, nz + (nz - pd) e1h)
    float gd2 = fmaf(lx, nx, ly * ny), gd1 = lz * (nz - p.pd), gpd = -lz * e1h;
    const float ax = lx * a2, ay = ly * a2, az = lz * a1;  // dL/dn
    // rotation: b = R^T a = c a - s1 (w x a) + s2 w (w . a)
    const float k2 = s2 * fmaf(wx, ax, fmaf(wy, ay, wz * az));
    const float bx = fmaf(c, ax, fmaf(-s1, wy * az - wz * ay, k2 * wx));
    const float by = fmaf(c, ay, fmaf(-s1, wz * ax - wx * az, k2 * wy));
    const float bz = fmaf(c, az, fmaf(-s1, wx * ay - wy * ax, k2 * wz));
    // gw = J^T u, u = n x a
    const float ux = ny * az - nz * ay, uy = nz * ax - nx * az, uz = nx * ay - ny * ax;
    const float k3 = s3 * fmaf(wx, ux, fmaf(wy, uy, wz * uz));
    const float gwx = fmaf(s1, ux, fmaf(-s2, wy * uz - wz * uy, k3 * wx));
    const float gwy = fmaf(s1, uy, fmaf(-s2, wz * ux - wx * uz, k3 * wy));
    const float gwz = OG ? fmaf(s1, uz, fmaf(-s2, wx * uy - wy * ux, k3 * wz)) : 0.0f;
    // first half relaxation
    gd2 = fmaf(bx, x0, fmaf(by, y0, gd2));
    gd1 = fmaf(bz, z0 - p.pd, gd1);
    gpd = fmaf(-bz, e1h, gpd);
    lx = bx * a2, ly = by * a2, lz = bz * a1;
    // e1h = expm1(-h r1): d/dr1 = -h (1 + e1h), d/d(dt) = -(r1 / 2)(1 + e1h)
    if (SG) {
        g[G_R1] = fmaf(-gd1 * h, a1, g[G_R1]);
        g[G_R2] = fmaf(-gd2 * h, a2, g[G_R2]);
        g[G_PD] += gpd;
        g[G_B1] = fmaf(gwx, q.wx0, fmaf(gwy, q.wy0, g[G_B1]));
    }
    sg.v[S_WX] += gwx * p.b1;
    sg.v[S_WY] += gwy * p.b1;
    if (OG) {  // the offset's and dt's gradients (position, dB0, segment dt, moments, b0_offset)
        sg.v[S_DT] -= 0.5f * (gd1 * p.r1 * a1 + gd2 * p.r2 * a2);
        phase_grads<PH>(-BP_TWO_PI_F * gwz, q, p, g, sg, ps, sq);
    }
}

// Reverse of an RF segment without per-spin or offset gradients, from its output state alone (ox, oy, oz), which
// it turns into the segment's input state: n = E^-1 (out - c) (the half-step relaxation undone), lambda and the
// rotation's gradient as rf_reverse forms them, then m1 = R^T n and in = E^-1 (m1 - c). Needs the relaxation to be
// invertible (r.invert). A window swept this way needs no recompute of its states: it integrates them backward
// from the state after the window.
template <bool SMALL>
__device__ __forceinline__ void rf_back(const SegRec& q, const Spin& p, const RevRelax& r, float wz, float& ox,
                                        float& oy, float& oz, float& lx, float& ly, float& lz, SegGrad& sg) {
    const float wx = q.wx0 * p.b1, wy = q.wy0 * p.b1;
    const float p2 = fmaf(wx, wx, fmaf(wy, wy, wz * wz));
    float c, s1, s2, s3;
    rot_factors<SMALL>(p2, c, s1, s2, s3);
    const float nx = ox * r.ia2, ny = oy * r.ia2, nz = fmaf(p.pd, r.e1h, oz) * r.ia1;
    const float ax = lx * r.a2, ay = ly * r.a2, az = lz * r.a1;  // dL/dn
    const float k2 = s2 * fmaf(wx, ax, fmaf(wy, ay, wz * az));
    const float bx = fmaf(c, ax, fmaf(-s1, wy * az - wz * ay, k2 * wx));
    const float by = fmaf(c, ay, fmaf(-s1, wz * ax - wx * az, k2 * wy));
    const float bz = fmaf(c, az, fmaf(-s1, wx * ay - wy * ax, k2 * wz));
    const float ux = ny * az - nz * ay, uy = nz * ax - nx * az, uz = nx * ay - ny * ax;
    const float k3 = s3 * fmaf(wx, ux, fmaf(wy, uy, wz * uz));
    const float gwx = fmaf(s1, ux, fmaf(-s2, wy * uz - wz * uy, k3 * wx));
    const float gwy = fmaf(s1, uy, fmaf(-s2, wz * ux - wx * uz, k3 * wy));
    lx = bx * r.a2, ly = by * r.a2, lz = bz * r.a1;
    sg.v[S_WX] += gwx * p.b1;
    sg.v[S_WY] += gwy * p.b1;
    const float k4 = s2 * fmaf(wx, nx, fmaf(wy, ny, wz * nz));
    const float m1x = fmaf(c, nx, fmaf(-s1, wy * nz - wz * ny, k4 * wx));
    const float m1y = fmaf(c, ny, fmaf(-s1, wz * nx - wx * nz, k4 * wy));
    const float m1z = fmaf(c, nz, fmaf(-s1, wx * ny - wy * nx, k4 * wz));
    ox = m1x * r.ia2, oy = m1y * r.ia2, oz = fmaf(p.pd, r.e1h, m1z) * r.ia1;
}

// Reverse of a free segment (rotation about z by phi = -2 pi cyc, then exact relaxation). OG: the offset's and dt's
// gradients are wanted.
template <bool OG, bool SG = true, bool PH = false>
__device__ __forceinline__ void free_reverse(const SegRec& q, const Spin& p, const FreeFactors& f, float x0, float y0,
                                             float z0, float& lx, float& ly, float& lz, float* g, SegGrad& sg,
                                             PhysSpin* ps = nullptr, const double* sq = nullptr) {
    const float c = f.ch, s = f.sh, a2 = 1.0f + f.e2, a1 = 1.0f + f.e1;
    if (!SG && !OG) {  // lambda alone: no gradient of this segment is wanted (and the input state is not read)
        const float nlx = a2 * fmaf(c, lx, s * ly), nly = a2 * fmaf(-s, lx, c * ly);
        lx = nlx, ly = nly, lz *= a1;
        return;
    }
    const float ux = fmaf(c, x0, -s * y0), uy = fmaf(s, x0, c * y0);
    const float gd2 = fmaf(lx, ux, ly * uy);
    const float gphi = OG ? a2 * fmaf(ly, ux, -lx * uy) : 0.0f;
    const float nlx = a2 * fmaf(c, lx, s * ly), nly = a2 * fmaf(-s, lx, c * ly);
    const float gd1 = lz * (z0 - p.pd);
    g[G_PD] = fmaf(-lz, f.e1, g[G_PD]);
    lz = lz * a1;
    lx = nlx, ly = nly;
    g[G_R2] = fmaf(-gd2 * q.dt, a2, g[G_R2]);
    g[G_R1] = fmaf(-gd1 * q.dt, a1, g[G_R1]);
    if (OG) {
        sg.v[S_DT] -= gd2 * p.r2 * a2 + gd1 * p.r1 * a1;
        phase_grads<PH>(-BP_TWO_PI_F * gphi, q, p, g, sg, ps, sq);
    }
}

template <int K>
struct KindTag {
    static constexpr int value = K;
};

// A window the sweep can run: at most BP_ADJ_WIN segments (the slots and staging buffers), inside the interval (the
// rows of gseg), its samples (at most one per segment) inside h.
__device__ __forceinline__ bool adj_window_ok(const int4& win, const AdjArgs& a) {
    const int nseg = win.y - win.x;
    return !(nseg < 0 || nseg > BP_ADJ_WIN || win.x < a.seg0 || win.y > a.seg0 + a.seg_len || win.z < 0 ||
             win.w < 0 || win.w > nseg || (a.h != nullptr && win.z + win.w > a.n_adc));
}

// NCG: groups of 8 coils; CG: whether the coil gradients are wanted (a.gc not null); OG: whether the gradients
// of the spins' offsets (position, dB0) or of the segments' dt, moments or b0_offset are wanted (otherwise their
// rows of gs and columns of gseg are left as they were); SG: whether any per-spin gradient is wanted (without them,
// and without CG and OG, gs is left as it was and a window of free segments only carries lambda back, with no
// recompute: only the RF segments' gradients and lambda are formed).
//
// Without per-spin gradients (SG false) the variant keeps no state slots: its windows of free segments carry lambda
// alone and its windows of RF segments integrate their states backward, and the rare window that needs its states
// recomputed (a spoil at its end, relaxation too strong to invert, RF and free segments mixed) recomputes each
// segment's input from the window start in registers (n(n+1)/2 steps instead of n). Its shared memory holds the
// window's cotangent rows instead, so a sample's coil sum reads shared memory, and five CTAs fit on an SM.
template <int NCG, bool CG, bool OG, bool SG, bool PH>
__global__ void __launch_bounds__(ADJ_THREADS, SG ? (NCG == 1 ? 4 : 3) : (NCG == 1 ? 5 : 4))
    bp_adjoint_kernel(AdjArgs a) {
    static_assert(SG || (!CG && !OG), "coil and offset gradients are per-spin gradients");
    extern __shared__ __align__(16) float sm[];
    float* slots = sm;                                              // SG: [ADJ_SLOTS][3][ADJ_THREADS]
    // the warps' segment partials [ADJ_WARPS][BP_ADJ_WIN][SGW] and the window's records [BP_ADJ_WIN]: one of
    // each (SG), or two (!SG: window w uses buffer w's parity, so a window's staging never waits for the last
    // reads of the window before it). !SG forms the RF's two components alone: SGW = 2 (S_WX, S_WY)
    constexpr int NBUF = SG ? 1 : 2, SGW = SG ? N_SG : 2;
    constexpr int PERBUF = ADJ_WARPS * BP_ADJ_WIN * SGW + BP_ADJ_WIN * (int)(sizeof(SegRec) / sizeof(float));
    float* wbuf0 = sm + (SG ? ADJ_SLOTS * 3 * ADJ_THREADS : 0);  // [NBUF]: segacc, then the records
    double4* wk64 = reinterpret_cast<double4*>(wbuf0 + NBUF * PERBUF);  // SG: the window's moments
    // !SG: two staging buffers, each the raw records, the moments and the cotangent rows ([BP_ADJ_WIN][8 NCG]) of a
    // window, filled by TMA bulk copies one window ahead; wk64 and hs point into the current one
    SegRec* rawrec = reinterpret_cast<SegRec*>(wk64 + (SG ? BP_ADJ_WIN : 0));      // !SG: [2][BP_ADJ_WIN]
    double4* wk64b = reinterpret_cast<double4*>(rawrec + 2 * BP_ADJ_WIN);          // !SG: [2][BP_ADJ_WIN]
    float2* hsb = reinterpret_cast<float2*>(wk64b + 2 * BP_ADJ_WIN);               // !SG: [2][BP_ADJ_WIN][8 NCG]
    uint64_t* bars = reinterpret_cast<uint64_t*>(hsb + 2 * BP_ADJ_WIN * 8 * NCG);  // !SG: [2]
    float2* iacc = reinterpret_cast<float2*>(bars + 2);  // !SG: [ADJ_SACC_MAX] the interval's RF gradient (x, y)
    float* mes = reinterpret_cast<float*>(iacc + ADJ_SACC_MAX);  // !SG: [2][6][ADJ_THREADS] the states after windows
    // !SG: the cotangent rows expanded for paired FMAs, (h_re, h_im, h_im, -h_re) per coil: [2][BP_ADJ_WIN][8 NCG]
    float4* hs4b = reinterpret_cast<float4*>(mes + 2 * 6 * ADJ_THREADS);
    float2* hs = hsb;
    float4* hs4 = hs4b;
    __shared__ float wmax[2];  // the window's largest wx0^2 + wy0^2 (by the window's parity, as wkind)
    __shared__ unsigned wkind[2][ADJ_WARPS];  // per warp: a copy timed out (1), not all RF (2), not all free (4)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = a.n, n_tiles = (n + ADJ_THREADS - 1) / ADJ_THREADS;
    const int nv = 2 * a.n_coils;
    const bool need_seg = a.gseg != nullptr;
    const bool rf_only = need_seg && (a.seg_mask & BP_SEG_ALL & ~((1 << S_WX) | (1 << S_WY))) == 0;
    for (int b = 0; b < NBUF; ++b)
        for (int i = tid; i < ADJ_WARPS * BP_ADJ_WIN * SGW; i += ADJ_THREADS) wbuf0[b * PERBUF + i] = 0.0f;
    // !SG (only the RF's two components): the interval's sums in shared memory when they fit, in the order the
    // global adds would take (tile by tile), so the bits are the same
    const bool sacc = !SG && need_seg && a.seg_len <= ADJ_SACC_MAX;
    if (sacc)
        for (int i = tid; i < a.seg_len; i += ADJ_THREADS) iacc[i] = make_float2(0.0f, 0.0f);
    if (need_seg)  // this CTA's rows of gseg, and those of CTAs this launch does not have
        for (int r = blockIdx.x; r < a.grid_rows; r += gridDim.x)
            for (int i = tid; i < a.seg_len * N_SG; i += ADJ_THREADS) a.gseg[(size_t)r * a.seg_len * N_SG + i] = 0.0f;
    // !SG: the cotangent rows come by TMA when they are whole coil groups on a 16-byte aligned base (else the
    // threads copy them, zero-padded); issue(w, b) stages window w into buffer b (thread 0): a window the sweep
    // cannot run, or one without segments, completes the buffer's phase with no data
    const bool h_tma = !SG && a.h != nullptr && 2 * a.n_coils == 16 * NCG && (reinterpret_cast<uintptr_t>(a.h) & 15) == 0;
    // the tile's state after the window (its six rows of the replay's window states: 128 spins each) comes by TMA
    // too when every row starts on a 16-byte boundary (n a multiple of 4, the array 16-byte aligned)
    const bool me_tma = !SG && (n & 3) == 0 && (reinterpret_cast<uintptr_t>(a.wstates) & 15) == 0;
    // !SG: the rows of the state after window w (the next window's start), or null where it was not saved
    auto after_state = [&](int w) -> const float* {
        if (a.wslot) {
            const int sl = a.wslot[w + 1];
            return sl >= 0 ? a.wstates + (size_t)sl * 6 * n : nullptr;
        }
        return a.wstates + (size_t)(w - a.wa + 1) * 6 * n;
    };
    auto issue = [&](int w, int b, int t) {
        const int4 win = a.windows[w];
        const int ns = win.y - win.x;
        if (!adj_window_ok(win, a) || ns == 0) {
            mbar_arrive(&bars[b]);
            return;
        }
        const bool th = h_tma && win.w > 0;
        const uint32_t rec_bytes = (uint32_t)ns * sizeof(SegRec), hbytes = th ? (uint32_t)win.w * 64u * NCG : 0u;
        const int t0 = t * ADJ_THREADS, cnt = min(ADJ_THREADS, n - t0);
        const float* we = after_state(w);
        const uint32_t me_bytes = (me_tma && we) ? (uint32_t)cnt * 4u : 0u;  // (a multiple of 16: n, t0 are of 4)
        fence_proxy_async_smem();
        mbar_expect_tx(&bars[b], 2 * rec_bytes + hbytes + 6 * me_bytes);
        tma_load_1d(rawrec + b * BP_ADJ_WIN, a.segs + win.x, rec_bytes, &bars[b]);
        tma_load_1d(wk64b + b * BP_ADJ_WIN, a.seg64 + win.x, rec_bytes, &bars[b]);
        if (th) tma_load_1d(hsb + b * BP_ADJ_WIN * 8 * NCG, a.h + (size_t)win.z * 16 * NCG, hbytes, &bars[b]);
        if (me_bytes)
            for (int k = 0; k < 6; ++k)
                tma_load_1d(mes + (b * 6 + k) * ADJ_THREADS, we + t0 + (size_t)k * n, me_bytes, &bars[b]);
    };
    int seq = 0;  // !SG: windows this CTA has staged so far (buffer seq & 1, its phase (seq >> 1) & 1)
    if (!SG && tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (!SG && tid == 0 && blockIdx.x < n_tiles && a.wb > a.wa) issue(a.wb - 1, 0, blockIdx.x);

    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int j0 = tile * ADJ_THREADS + tid;
        const bool active = j0 < n;
        const int j = active ? j0 : 0;
        const Spin p = load_spin(a.spins, n, j, active);
        // PH: the spin's concomitant coefficients and their gradients' running totals (as g)
        PhysSpin ps{};
        if constexpr (PH) {
            ps.mode = a.conc_mode;
            ps.c = load_conc(a.conc, n, j, a.conc_mode);
#pragma unroll
            for (int k = 0; k < 7; ++k) ps.gk[k] = (SG && active && a.gconc) ? a.gconc[k * n + j] : 0.0f;
        }
        // the segment's rotation about z and free factors (PH: with the concomitant field), s its index in the
        // sequence
        auto wz_of = [&](const SegRec& q, int s) -> float {
            if constexpr (PH) return phys_wz(q, p, ps.mode, ps.c, a.segq + 6 * (size_t)s);
            return rf_wz(q, p);
        };
        auto ff_of = [&](const SegRec& q, const double4& k64, int s) -> FreeFactors {
            if constexpr (PH) return free_factors_phys(q, k64, p, 1, ps.mode, ps.c, a.segq + 6 * (size_t)s);
            return free_factors(q, k64, p);
        };
        float lx = active ? a.lam[j] : 0.0f, ly = active ? a.lam[n + j] : 0.0f, lz = active ? a.lam[2 * n + j] : 0.0f;
        // from saved states: the chain (the start state of the window swept last, when it was integrated backward)
        const bool saved = !SG && a.wslot != nullptr;
        bool chain_ok = saved && a.chain_in != 0, no_state = false;
        float cx = 0.f, cy = 0.f, cz = 0.f;
        if (chain_ok && active) cx = a.chain[j], cy = a.chain[n + j], cz = a.chain[2 * n + j];
        // per-spin gradients: running totals carried in registers through the interval (loaded here, stored after
        // its last window): every contribution is added to the total in segment order, so the results do not
        // depend on where the checkpoint intervals fall
        float g[N_GS];
#pragma unroll
        for (int k = 0; k < N_GS; ++k) g[k] = (SG && active) ? a.gs[k * n + j] : 0.0f;
        const bool want_gc = CG && active;
        // the spin's coil sensitivities: SG as two arrays, !SG as (re, im) pairs (the operands of paired FMAs)
        float gcr[CG ? 8 * NCG : 1], gci[CG ? 8 * NCG : 1], sr[SG ? 8 * NCG : 1], si[SG ? 8 * NCG : 1];
        float2 sp[SG ? 1 : 8 * NCG];
#pragma unroll
        for (int c = 0; c < 8 * NCG; ++c) {
            if (CG) {
                gcr[c] = (want_gc && c < a.n_coils) ? a.gc[(2 * c) * n + j] : 0.0f;
                gci[c] = (want_gc && c < a.n_coils) ? a.gc[(2 * c + 1) * n + j] : 0.0f;
            }
            const float re = active ? a.sens[(2 * c) * n + j] : 0.0f, im = active ? a.sens[(2 * c + 1) * n + j] : 0.0f;
            if constexpr (SG)
                sr[c] = re, si[c] = im;
            else
                sp[c] = make_float2(re, im);
        }
        for (int w = a.wb - 1; w >= a.wa; --w) {
            const int4 win = a.windows[w];
            // a window the sweep can run (adj_window_ok); anything else is skipped (the same for the whole CTA) and
            // reported, after the barrier below
            const bool good = adj_window_ok(win, a);
            const int buf = seq & 1;
            bool ok = true;
            if constexpr (!SG) {
                ok = mbar_wait_bounded(&bars[buf], (seq >> 1) & 1);  // (a copy of a few KB: never this long)
                ++seq;
                wk64 = wk64b + buf * BP_ADJ_WIN;
                hs = hsb + buf * BP_ADJ_WIN * 8 * NCG;
                hs4 = hs4b + buf * BP_ADJ_WIN * 8 * NCG;
            }
            const int nseg = (good && ok) ? win.y - win.x : 0;  // (nothing is read of a window that is not run)
            float* segacc = wbuf0 + buf * PERBUF;  // (SG: buf is 0)
            SegRec* wrec = reinterpret_cast<SegRec*>(segacc + ADJ_WARPS * BP_ADJ_WIN * SGW);
            // the window's states from the replay (in DRAM for long intervals), loaded first so that their latency
            // overlaps the staging below: SG its start (the recompute's); !SG the state after it (the next window's
            // start, or the interval's end: RF windows integrate backward from it), its start only where a window
            // recomputes (loaded there)
            float m0x = 0.f, m0y = 0.f, m0z = 0.f, mex = 0.f, mey = 0.f, mez = 0.f;
            const float* we = SG ? nullptr : after_state(w);
            const bool chain_in_w = chain_ok;  // the window after this one was integrated backward (saved states)
            chain_ok = false;
            if (active && nseg > 0) {
                if (SG) {
                    const float* ws = a.wstates + (size_t)(w - a.wa) * 6 * n;
                    m0x = ws[j] + ws[3 * n + j], m0y = ws[n + j] + ws[4 * n + j], m0z = ws[2 * n + j] + ws[5 * n + j];
                } else if (we && me_tma) {  // staged with the window's records
                    const float* me = mes + buf * 6 * ADJ_THREADS + tid;
                    mex = me[0] + me[3 * ADJ_THREADS], mey = me[ADJ_THREADS] + me[4 * ADJ_THREADS];
                    mez = me[2 * ADJ_THREADS] + me[5 * ADJ_THREADS];
                } else if (we) {
                    mex = we[j] + we[3 * n + j], mey = we[n + j] + we[4 * n + j], mez = we[2 * n + j] + we[5 * n + j];
                }
            }
            // the window's records into shared memory (every warp of the CTA sweeps the same window); the barrier
            // at the end of the previous window ended its reads. The flags word of record s is written by thread s
            // alone, with the sweep's own bits added: SG from the global records, !SG from the staging buffer (read
            // only), so no thread reads a word another writes
            const SegRec* gw = SG ? a.segs + win.x : rawrec + buf * BP_ADJ_WIN;
            for (int i = tid; i < nseg * 8; i += ADJ_THREADS)
                if ((i & 7) != 7) reinterpret_cast<float*>(wrec)[i] = reinterpret_cast<const float*>(gw)[i];
            for (int i = tid; i < nseg; i += ADJ_THREADS) {
                const int f = gw[i].flags, fn = i + 1 < nseg ? gw[i + 1].flags : 0;
                int x = f;
                if (i > 0 && (gw[i - 1].flags & BP_SPOIL)) x |= A_PREV_SPOIL;
                if ((f & BP_RF) && (fn & BP_RF) && (fn & BP_SAME_RFDT)) x |= A_KEEP_RELAX;
                if ((f & BP_RF) && (fn & BP_RF) && (fn & BP_SAME_OFF)) x |= A_KEEP_WZ;
                if (!(f & BP_RF) && i + 1 < nseg && !(fn & BP_RF) && (fn & BP_SAME_FREE)) x |= A_KEEP_FREE;
                wrec[i].flags = x;
            }
            if (SG)
                for (int i = tid; i < nseg * 4; i += ADJ_THREADS)
                    reinterpret_cast<double*>(wk64)[i] = reinterpret_cast<const double*>(a.seg64 + win.x)[i];
            if (!SG && a.h != nullptr && nseg > 0) {  // cotangent rows, expanded, zero-padded to 8 NCG coils
                for (int i = tid; i < win.w * 8 * NCG; i += ADJ_THREADS) {
                    const int r = i / (8 * NCG), c = i - r * (8 * NCG);
                    const float2 v = h_tma ? hs[i]  // (staged by TMA)
                                     : c < a.n_coils
                                         ? reinterpret_cast<const float2*>(a.h + (size_t)(win.z + r) * nv)[c]
                                         : make_float2(0.0f, 0.0f);
                    hs4[i] = make_float4(v.x, v.y, v.y, -v.x);
                }
            }
            // the window's kind (the same for the whole CTA): every segment RF with the dt and offset of the first,
            // no sample (the steps of an RF pulse); or every segment free with the factors of the first (a
            // readout's samples); in either, a spoil at most after the last segment. Their sweeps skip the
            // per-segment tests.
            bool rf_ok = true, free_ok = true;
            if (tid < nseg) {
                const int f = gw[tid].flags;
                const bool spoil_ok = !(f & BP_SPOIL) || tid == nseg - 1;
                rf_ok = (f & BP_RF) && !(f & BP_ADC) && spoil_ok && (tid == 0 || (f & BP_SAME_OFF));
                free_ok = !(f & BP_RF) && spoil_ok && (tid == 0 || (f & BP_SAME_FREE));
            }
            if (warp == 0) {  // the window's largest wx0^2 + wy0^2 (non-negative floats order as their bits)
                const float v = lane < nseg ? fmaf(gw[lane].wx0, gw[lane].wx0, gw[lane].wy0 * gw[lane].wy0) : 0.0f;
                const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(v));
                if (lane == 0) wmax[buf] = __uint_as_float(m);
            }
            // one barrier for the staging, the copy's bounded wait (any thread gave up) and the window's kind (every
            // thread agrees): each warp's OR of its threads' bits, then the warps' words
            const unsigned bits = (ok ? 0u : 1u) | (rf_ok ? 0u : 2u) | (free_ok ? 0u : 4u);
            const unsigned wbits = __reduce_or_sync(0xffffffffu, bits);
            if (lane == 0) wkind[buf][warp] = wbits;
            __syncthreads();
            // !SG: the next window (this tile's, or the next tile's first) into the other buffer, now that every
            // thread is past the barrier: its reads of that buffer (the window before this one's) have ended
            if (!SG && tid == 0) {
                if (w > a.wa)
                    issue(w - 1, buf ^ 1, tile);
                else if (tile + (int)gridDim.x < n_tiles)
                    issue(a.wb - 1, buf ^ 1, tile + (int)gridDim.x);
            }
            unsigned kind_bits = 0;
#pragma unroll
            for (int k = 0; k < ADJ_WARPS; ++k) kind_bits |= wkind[buf][k];
            if (kind_bits & 1u) {  // a staging copy did not land within the bound: report and stop
                if (tid == 0) {
                    atomicOr(a.status, BP_ERR_TMA_TIMEOUT);
                    if (!SG) mbar_wait_bounded(&bars[buf ^ 1], (seq >> 1) & 1);  // the other buffer's copy, if any
                }
                return;
            }
            if (!good) {
                if (tid == 0) atomicOr(a.status, BP_ERR_BAD_WINDOW);
                __syncthreads();  // (every thread has read wkind before the next window writes it)
                continue;
            }
            const bool all_rf = !(kind_bits & 2u), all_free = !(kind_bits & 4u);
            // the segment's partial gradients summed over the warp into its slice of segacc
            auto reduce_seg = [&](int s, const SegGrad& sg) {
                if (rf_only) {  // only the RF's two components: a reduce-scatter of 2 values (lanes 0, 16 hold them)
                    const bool up = lane & 16;
                    const float v0 = sg.v[S_WX], v1 = sg.v[S_WY];  // (0 for a padding row: its lambda is 0)
                    float t = (up ? v1 : v0) + __shfl_xor_sync(0xffffffffu, up ? v0 : v1, 16);
#pragma unroll
                    for (int o = 8; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                    const int col = SG ? (up ? S_WY : S_WX) : (up ? 1 : 0);
                    if ((lane & 15) == 0) segacc[(warp * BP_ADJ_WIN + s) * SGW + col] = t;
                } else if (SG && need_seg) {  // the warp's sums of the N_SG (= 8) values, one per group of four lanes
                    float v[N_SG];
#pragma unroll
                    for (int k = 0; k < N_SG; ++k) v[k] = sg.v[k];
                    const float t = warp_reduce_scatter8(v, lane);
                    if ((lane & 3) == 0) segacc[(warp * BP_ADJ_WIN + s) * SGW + ((lane >> 2) & 7)] = t;
                }
            };
            auto sweep = [&](auto kind_tag) {
                // 0: any segments, 1: uniform RF, 2: uniform free, 3: uniform RF with every |w| < 1/4 in the warp
                constexpr int KIND = decltype(kind_tag)::value;
                constexpr bool URF = KIND == 1 || KIND == 3;
                // a uniform free window without gradients of its own carries lambda alone: no states needed
                constexpr bool LAMBDA_ONLY = KIND == 2 && !SG && !OG;
                // a uniform RF window without per-spin gradients integrates its states backward from the state
                // after it, when that state is unspoiled and every lane's relaxation is invertible
                if constexpr (URF && !SG && !OG) {
                    const RevRelax rb = rev_relax(wrec[0].dt, p);
                    const float wzb = wz_of(wrec[0], win.x);
                    const bool from_chain = saved && chain_in_w;
                    if (!(wrec[nseg - 1].flags & BP_SPOIL) && __all_sync(0xffffffffu, rb.invert) &&
                        (from_chain || we != nullptr)) {
                        float ox = from_chain ? cx : mex, oy = from_chain ? cy : mey, oz = from_chain ? cz : mez;
                        for (int s = nseg - 1; s >= 0; --s) {
                            SegGrad sg;
#pragma unroll
                            for (int k = 0; k < N_SG; ++k) sg.v[k] = 0.0f;
                            rf_back<KIND == 3>(wrec[s], p, rb, wzb, ox, oy, oz, lx, ly, lz, sg);
                            reduce_seg(s, sg);
                        }
                        if (saved) cx = ox, cy = oy, cz = oz, chain_ok = true;  // the state after the window before
                        return;
                    }
                }
                // recompute the window in plain float32 from its (compensated) start state: slot k = state after
                // segment k-1 (before its spoil), slot 0 = window start
                if constexpr (!SG && !LAMBDA_ONLY) {  // (loaded only here: the windows that recompute)
                    if (saved) {  // no window start states were saved: this window cannot be swept (reported)
                        no_state = true;
                        return;
                    }
                    if (active) {
                        const float* ws = a.wstates + (size_t)(w - a.wa) * 6 * n;
                        m0x = ws[j] + ws[3 * n + j], m0y = ws[n + j] + ws[4 * n + j];
                        m0z = ws[2 * n + j] + ws[5 * n + j];
                    }
                }
                float mx = m0x, my = m0y, mz = m0z;
                if (SG && !LAMBDA_ONLY) slots[tid] = mx, slots[ADJ_THREADS + tid] = my, slots[2 * ADJ_THREADS + tid] = mz;
                FreeFactors ff{1.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                RevRelax rr{0.f, 0.f, 1.f, 1.f, 1.f, 1.f, true};
                float wz = 0.f;
                if (URF) rr = rev_relax(wrec[0].dt, p), wz = wz_of(wrec[0], win.x);
                if (KIND == 2) ff = ff_of(wrec[0], wk64[0], win.x);
                // !SG: the state after segments 0 .. upto-1 of the window (before the last one's spoil), recomputed
                // from the window start with factors of its own (the sweep's are kept)
                auto state_at = [&](int upto, float& x, float& y, float& z) {
                    x = m0x, y = m0y, z = m0z;
                    FreeFactors f2 = ff;
                    RevRelax r2 = rr;
                    float w2 = wz;
                    for (int s = 0; s < upto; ++s) {
                        const SegRec q = wrec[s];
                        if (URF || (KIND == 0 && (q.flags & BP_RF))) {
                            if (KIND == 0) {
                                if (s == 0 || !(q.flags & BP_SAME_RFDT)) r2 = rev_relax(q.dt, p);
                                if (s == 0 || !(q.flags & BP_SAME_OFF)) w2 = wz_of(q, win.x + s);
                            }
                            rf_step_plain<KIND == 3>(q, p, r2, w2, x, y, z);
                        } else {
                            if (KIND == 0 && (s == 0 || !(q.flags & BP_SAME_FREE))) f2 = ff_of(q, wk64[s], win.x + s);
                            free_step_plain(f2, p, x, y, z);
                        }
                        if (KIND == 0 && s + 1 < upto && (q.flags & BP_SPOIL)) x = y = 0.0f;
                    }
                };
                for (int s = 0; s < ((LAMBDA_ONLY || !SG) ? 0 : nseg); ++s) {
                    const SegRec q = wrec[s];
                    if (URF || (KIND == 0 && (q.flags & BP_RF))) {
                        if (KIND == 0) {
                            if (s == 0 || !(q.flags & BP_SAME_RFDT)) rr = rev_relax(q.dt, p);
                            if (s == 0 || !(q.flags & BP_SAME_OFF)) wz = wz_of(q, win.x + s);
                        }
                        rf_step_plain<KIND == 3>(q, p, rr, wz, mx, my, mz);
                    } else {
                        if (KIND == 0 && (s == 0 || !(q.flags & BP_SAME_FREE))) ff = ff_of(q, wk64[s], win.x + s);
                        free_step_plain(ff, p, mx, my, mz);
                    }
                    float* sl = slots + (s + 1) * 3 * ADJ_THREADS;
                    sl[tid] = mx, sl[ADJ_THREADS + tid] = my, sl[2 * ADJ_THREADS + tid] = mz;
                    if (KIND == 0 && (q.flags & BP_SPOIL)) mx = my = 0.0f;
                }
                // sweep back
                int row = win.z + win.w;
                // (a uniform window spoils at most after its last segment, where the sweep starts)
                if (KIND != 0 && (wrec[nseg - 1].flags & BP_SPOIL)) lx = ly = 0.0f;
                // the cotangent rows as (re, im) pairs: 8-byte aligned (rows of 2 C floats on an 8-byte aligned
                // base, checked by bp_adjoint). A readout window loads each sample's row one sample ahead, so the
                // loads' latency overlaps the sweep of the sample before (rows [win.z, win.z + win.w) only)
                float2 hnext[8 * NCG];
                if (SG && KIND == 2 && a.h != nullptr && win.w > 0) {
                    const float2* hr = reinterpret_cast<const float2*>(a.h + (size_t)(row - 1) * nv);
#pragma unroll
                    for (int c = 0; c < 8 * NCG; ++c) hnext[c] = c < a.n_coils ? hr[c] : make_float2(0.f, 0.f);
                }
                // the state after the segment being swept (its output, before its spoil): slot s + 1, which the
                // previous iteration read as its input
                float outx = 0.f, outy = 0.f, outz = 0.f;
                if (!LAMBDA_ONLY) {
                    if (SG) {
                        outx = slots[nseg * 3 * ADJ_THREADS + tid], outy = slots[(nseg * 3 + 1) * ADJ_THREADS + tid];
                        outz = slots[(nseg * 3 + 2) * ADJ_THREADS + tid];
                    } else {
                        state_at(nseg, outx, outy, outz);
                    }
                }
                for (int s = nseg - 1; s >= 0; --s) {
                    const SegRec q = wrec[s];
                    const int f = q.flags;
                    if (KIND == 0 && (f & BP_SPOIL)) lx = ly = 0.0f;
                    const float ox = outx, oy = outy, oz = outz;
                    if (!URF && (f & BP_ADC) && a.h != nullptr) {
                        --row;
                        if constexpr (!SG) {
                            // the staged row (zero-padded coils) by paired FMAs: u = sum (h_re, h_im) (s_re, s_im),
                            // v = sum (h_im, -h_re) (s_re, s_im); dL/dm_x = u.x + u.y, dL/dm_y = v.x + v.y
                            const float4* hr = hs4 + (row - win.z) * 8 * NCG;
                            float2 u = make_float2(0.0f, 0.0f), v = make_float2(0.0f, 0.0f);
#pragma unroll
                            for (int c = 0; c < 8 * NCG; ++c) {
                                const float4 h4 = hr[c];
                                u = __ffma2_rn(make_float2(h4.x, h4.y), sp[c], u);
                                v = __ffma2_rn(make_float2(h4.z, h4.w), sp[c], v);
                            }
                            lx += u.x + u.y, ly += v.x + v.y;
                        } else {
                        float2 hrow[8 * NCG];
                        if (KIND == 2) {
#pragma unroll
                            for (int c = 0; c < 8 * NCG; ++c) hrow[c] = hnext[c];
                            if (row > win.z) {
                                const float2* hr = reinterpret_cast<const float2*>(a.h + (size_t)(row - 1) * nv);
#pragma unroll
                                for (int c = 0; c < 8 * NCG; ++c)
                                    if (c < a.n_coils) hnext[c] = hr[c];
                            }
                        } else {
                            const float2* hr = reinterpret_cast<const float2*>(a.h + (size_t)row * nv);
#pragma unroll
                            for (int c = 0; c < 8 * NCG; ++c)
                                if (c < a.n_coils) hrow[c] = hr[c];
                        }
                        float dx = 0.0f, dy = 0.0f;
#pragma unroll
                        for (int c = 0; c < 8 * NCG; ++c) {
                            if (c < a.n_coils) {
                                const float2 hc = hrow[c];
                                const float h0 = hc.x, h1 = hc.y;
                                dx = fmaf(h0, sr[c], fmaf(h1, si[c], dx));
                                dy = fmaf(-h0, si[c], fmaf(h1, sr[c], dy));
                                if (CG) {
                                    gcr[c] = fmaf(h0, ox, fmaf(h1, oy, gcr[c]));
                                    gci[c] = fmaf(-h0, oy, fmaf(h1, ox, gci[c]));
                                }
                            }
                        }
                        lx += dx, ly += dy;
                        }
                    }
                    // the segment's input state: slot s, spoiled by segment s-1 if it spoils
                    float x0 = 0.f, y0 = 0.f, z0 = 0.f;
                    if (!LAMBDA_ONLY) {
                        if (SG) {
                            const float* in = slots + s * 3 * ADJ_THREADS;
                            x0 = in[tid], y0 = in[ADJ_THREADS + tid], z0 = in[2 * ADJ_THREADS + tid];
                        } else {
                            state_at(s, x0, y0, z0);
                        }
                    }
                    outx = x0, outy = y0, outz = z0;
                    if (KIND == 0 && (f & A_PREV_SPOIL)) x0 = y0 = 0.0f;
                    SegGrad sg;
#pragma unroll
                    for (int k = 0; k < N_SG; ++k) sg.v[k] = 0.0f;
                    if (URF || (KIND == 0 && (f & BP_RF))) {
                        // the factors of the segment after this one (swept just before) when they are the same
                        if (KIND == 0) {
                            if (!(f & A_KEEP_RELAX)) rr = rev_relax(q.dt, p);
                            if (!(f & A_KEEP_WZ)) wz = wz_of(q, win.x + s);
                        }
                        rf_reverse<KIND == 3, OG, SG, PH>(q, p, rr, wz, x0, y0, z0, ox, oy, oz, lx, ly, lz, g, sg, &ps,
                                                          PH ? a.segq + 6 * (size_t)(win.x + s) : nullptr);
                    } else {
                        if (KIND == 0 && !(f & A_KEEP_FREE)) ff = ff_of(q, wk64[s], win.x + s);
                        free_reverse<OG, SG, PH>(q, p, ff, x0, y0, z0, lx, ly, lz, g, sg, &ps,
                                                 PH ? a.segq + 6 * (size_t)(win.x + s) : nullptr);
                    }
                    if (!(rf_only && KIND == 2)) reduce_seg(s, sg);  // (a uniform free window's RF partials are 0)
                }
            };
            if (all_rf) {
                // every rotation of the window below |w| = 1/4 for every spin of the warp: |w|^2 <= b1^2 max(wx0^2 +
                // wy0^2) + wz^2 (one offset for the window)
                const float wz0 = wz_of(wrec[0], win.x);
                const bool small = fmaf(p.b1 * p.b1, wmax[buf], wz0 * wz0) < 0.0624f;
                if (__all_sync(0xffffffffu, small))
                    sweep(KindTag<3>{});
                else
                    sweep(KindTag<1>{});
            } else if (all_free) {
                sweep(KindTag<2>{});
            } else {
                sweep(KindTag<0>{});
            }
            // segacc complete (SG: and every thread is done reading this window's slots and records). Without
            // per-spin gradients a window whose partials are not summed here (a free window's RF partials are 0)
            // needs no barrier: its buffers alternate with the next window's
            const bool summed = need_seg && !(rf_only && all_free);
            if (SG || summed) __syncthreads();
            if (sacc && !all_free) {  // (!SG: rf_only; a free window's RF partials are 0)
                for (int i = tid; i < 2 * nseg; i += ADJ_THREADS) {
                    const int sgi = i >> 1, comp = (i & 1) ? S_WY : S_WX;
                    float t = 0.0f;
#pragma unroll
                    for (int ww = 0; ww < ADJ_WARPS; ++ww)
                        t += segacc[(ww * BP_ADJ_WIN + sgi) * SGW + (SG ? comp : (i & 1))];
                    float* d = reinterpret_cast<float*>(iacc + (win.x - a.seg0 + sgi)) + (i & 1);
                    *d += t;
                }
            } else if (need_seg && !(rf_only && all_free)) {
                float* dst = a.gseg + ((size_t)blockIdx.x * a.seg_len + (win.x - a.seg0)) * N_SG;
                for (int i = tid; i < nseg * SGW; i += ADJ_THREADS) {
                    float t = 0.0f;
#pragma unroll
                    for (int ww = 0; ww < ADJ_WARPS; ++ww) t += segacc[ww * BP_ADJ_WIN * SGW + i];
                    if (SG)
                        dst[i] += t;
                    else  // (the RF's two components)
                        dst[(i >> 1) * N_SG + ((i & 1) ? S_WY : S_WX)] += t;
                }
            }
            if (SG) __syncthreads();
        }
        if (no_state && lane == 0) atomicOr(a.status, BP_ERR_NO_STATE);
        if (active) {
            a.lam[j] = lx, a.lam[n + j] = ly, a.lam[2 * n + j] = lz;
            if (saved && a.chain) a.chain[j] = cx, a.chain[n + j] = cy, a.chain[2 * n + j] = cz;
            if (SG) {
#pragma unroll
                for (int k = 0; k < N_GS; ++k) a.gs[k * n + j] = g[k];
            }
            if (PH && SG && a.gconc) {
#pragma unroll
                for (int k = 0; k < 7; ++k) a.gconc[k * n + j] = ps.gk[k];
            }
            if (CG) {
#pragma unroll
                for (int c = 0; c < 8 * NCG; ++c) {
                    if (c < a.n_coils) {
                        a.gc[(2 * c) * n + j] = gcr[c];
                        a.gc[(2 * c + 1) * n + j] = gci[c];
                    }
                }
            }
        }
    }
    if (sacc) {  // the interval's RF gradient of this CTA (its rows were cleared at the start)
        __syncthreads();  // every add has ended
        float* dst = a.gseg + (size_t)blockIdx.x * a.seg_len * N_SG;
        for (int i = tid; i < a.seg_len; i += ADJ_THREADS) {
            const float2 v = iacc[i];
            dst[(size_t)i * N_SG + S_WX] = v.x;
            dst[(size_t)i * N_SG + S_WY] = v.y;
        }
    }
}

// SEG[seg0 + s][k] += sum over CTAs (in order) of gseg[cta][s][k], in float64
__global__ void bp_seg_reduce_kernel(const float* __restrict__ gseg, int n_cta, int seg_len, int seg0,
                                     double* __restrict__ seg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= seg_len * N_SG) return;
    double t = 0.0;
    for (int c = 0; c < n_cta; ++c) t += (double)gseg[(size_t)c * seg_len * N_SG + i];
    seg[(size_t)seg0 * N_SG + i] += t;
}

template <int NCG, bool SG>
static size_t adj_smem() {
    const size_t common = (size_t)ADJ_WARPS * BP_ADJ_WIN * N_SG * sizeof(float) + (size_t)BP_ADJ_WIN * sizeof(SegRec);
    if (SG)  // the slots, segacc, the records and the moments
        return (size_t)ADJ_SLOTS * 3 * ADJ_THREADS * sizeof(float) + common + (size_t)BP_ADJ_WIN * sizeof(double4);
    // two of segacc (the RF's two components) and of the records, two staging buffers (raw records, moments,
    // cotangent rows, the state after the window), their two mbarriers, the interval's RF gradient and two of the
    // expanded cotangent rows
    const size_t segacc2 = (size_t)ADJ_WARPS * BP_ADJ_WIN * 2 * sizeof(float) + (size_t)BP_ADJ_WIN * sizeof(SegRec);
    return 2 * segacc2 + 2 * (size_t)BP_ADJ_WIN * (sizeof(SegRec) + sizeof(double4) + 8 * NCG * sizeof(float2)) +
           2 * sizeof(uint64_t) + (size_t)ADJ_SACC_MAX * sizeof(float2) + 2 * 6 * ADJ_THREADS * sizeof(float) +
           2 * (size_t)BP_ADJ_WIN * 8 * NCG * sizeof(float4);
}

// One variant's shared-memory size, set once per device: 0, or -1 on failure.
template <int NCG, bool CG, bool OG, bool SG, bool PH = false>
static int adj_configure() {
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        if (cudaFuncSetAttribute(bp_adjoint_kernel<NCG, CG, OG, SG, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)adj_smem<NCG, SG>()) != cudaSuccess ||
            cudaFuncSetAttribute(bp_adjoint_kernel<NCG, CG, OG, SG, PH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return -1;
        configured[dev] = true;
    }
    return 0;
}

// CTAs per SM of one variant, or -1
template <int NCG, bool CG, bool OG, bool SG, bool PH = false>
static int adj_per_sm() {
    int per_sm = 0;
    if (adj_configure<NCG, CG, OG, SG, PH>() < 0 ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_adjoint_kernel<NCG, CG, OG, SG, PH>, ADJ_THREADS,
                                                      adj_smem<NCG, SG>()) != cudaSuccess)
        return -1;
    return per_sm > 0 ? per_sm : 1;
}

static int adj_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// the rows of gseg: the largest residency of the variants (a variant with fewer resident CTAs launches fewer and
// clears the other rows)
template <int NCG>
static int adj_grid(int n) {
    const int sms = adj_sms();
    const int v[4] = {adj_per_sm<NCG, true, true, true>(), adj_per_sm<NCG, false, true, true>(),
                      adj_per_sm<NCG, false, false, true>(), adj_per_sm<NCG, false, false, false>()};
    int per_sm = v[0];
    for (int k = 0; k < 4; ++k) {
        if (v[k] < 0) return -1;
        per_sm = v[k] > per_sm ? v[k] : per_sm;
    }
    const int n_tiles = (n + ADJ_THREADS - 1) / ADJ_THREADS;
    const int grid = sms * per_sm;
    return grid < n_tiles ? grid : n_tiles;
}

extern "C" int bp_adjoint_grid(int n, int n_coils) {
    if (n < 1 || n_coils < 1 || n_coils > BP_MAX_COILS) return -BP_E_ARG;
    switch ((n_coils + 7) / 8) {
        case 1: return adj_grid<1>(n);
        case 2: return adj_grid<2>(n);
        case 3: return adj_grid<3>(n);
        default: return adj_grid<4>(n);
    }
}

template <int NCG, bool CG, bool OG, bool SG, bool PH = false>
static int launch_variant(const AdjArgs& a, int grid, cudaStream_t st) {
    const int per_sm = adj_per_sm<NCG, CG, OG, SG, PH>();
    if (per_sm < 0) return BP_E_LAUNCH;
    const int own = adj_sms() * per_sm, ctas = grid < own ? grid : own;  // one wave of resident CTAs
    bp_adjoint_kernel<NCG, CG, OG, SG, PH><<<ctas, ADJ_THREADS, adj_smem<NCG, SG>(), st>>>(a);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

template <int NCG, bool PH = false>
static int launch_adj(const AdjArgs& a, int grid, cudaStream_t st) {
    // the offsets' gradients: wanted unless the caller marks the spins' ones unwanted and wants no segment
    // gradient that uses them (with coil gradients, always computed); the per-spin gradients: wanted unless marked
    // unwanted (BP_SPIN_NONE, which implies no offsets' gradients of the spins)
    const bool seg_offsets = (a.seg_mask & (BP_SEG_ALL & ~(BP_SEG_WX | BP_SEG_WY))) != 0;
    const bool og = !(a.seg_mask & (BP_SPIN_NO_OFFSETS | BP_SPIN_NONE)) || seg_offsets;
    const bool sg = !(a.seg_mask & BP_SPIN_NONE) || og;
    if (a.gc) return launch_variant<NCG, true, true, true, PH>(a, grid, st);
    if (og || (PH && a.gconc)) return launch_variant<NCG, false, true, true, PH>(a, grid, st);
    if (sg) return launch_variant<NCG, false, false, true, PH>(a, grid, st);
    return launch_variant<NCG, false, false, false, PH>(a, grid, st);
}

static int adjoint_impl(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                        const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                        const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc,
                        float* gseg, int seg_mask, int grid, int32_t* status, void* stream, const BpPhysics* ph,
                        float* gconc, const int32_t* wslot = nullptr, float* chain = nullptr, int chain_in = 0) {
    if (n < 1 || n_coils < 1 || n_coils > BP_MAX_COILS || wa < 0 || wb < wa || seg0 < 0 || seg_len < 0 || grid < 1 ||
        n_adc < 0)
        return BP_E_ARG;
    if (!spins || !sens || !segs || !seg64 || !windows || !wstates || !lam || (!gs && !wslot) || !status)
        return BP_E_ARG;
    // from saved states: only the sweep without per-spin, coil and offset gradients (the RF's alone)
    if (wslot && (!chain || ph || gc || !(seg_mask & BP_SPIN_NONE) ||
                  (seg_mask & (BP_SEG_ALL & ~(BP_SEG_WX | BP_SEG_WY))) != 0))
        return BP_E_ARG;
    if ((reinterpret_cast<uintptr_t>(h) & 7) != 0) return BP_E_ALIGN;  // read as (re, im) pairs
    // records and moments are staged by TMA bulk copies (16-byte aligned)
    if ((reinterpret_cast<uintptr_t>(segs) & 15) != 0 || (reinterpret_cast<uintptr_t>(seg64) & 15) != 0)
        return BP_E_ALIGN;
    if (ph && (ph->mt || ph->conc_mode < 0 || ph->conc_mode > 2 || (ph->conc_mode && !ph->conc) ||
               (ph->conc_mode == 1 && !ph->segq)))
        return BP_E_ARG;
    if (wb == wa) return BP_OK;
    AdjArgs a{spins, sens, static_cast<const SegRec*>(segs), reinterpret_cast<const double4*>(seg64),
              reinterpret_cast<const int4*>(windows), n, n_coils, wa, wb, seg0, seg_len, wstates, h, n_adc, lam, gs,
              gc, gseg, seg_mask, status, grid};
    a.wslot = wslot;
    a.chain = chain;
    a.chain_in = chain_in;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (ph && ph->conc_mode) {
        a.conc_mode = ph->conc_mode;
        a.conc = ph->conc;
        a.segq = ph->segq;
        a.gconc = gconc;
        switch ((n_coils + 7) / 8) {
            case 1: return launch_adj<1, true>(a, grid, st);
            case 2: return launch_adj<2, true>(a, grid, st);
            case 3: return launch_adj<3, true>(a, grid, st);
            default: return launch_adj<4, true>(a, grid, st);
        }
    }
    switch ((n_coils + 7) / 8) {
        case 1: return launch_adj<1>(a, grid, st);
        case 2: return launch_adj<2>(a, grid, st);
        case 3: return launch_adj<3>(a, grid, st);
        default: return launch_adj<4>(a, grid, st);
    }
}

extern "C" int bp_adjoint(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                          const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                          const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc,
                          float* gseg, int seg_mask, int grid, int32_t* status, void* stream) {
    return adjoint_impl(spins, sens, n, n_coils, segs, seg64, windows, wa, wb, seg0, seg_len, wstates, h, n_adc, lam,
                        gs, gc, gseg, seg_mask, grid, status, stream, nullptr, nullptr);
}

extern "C" int bp_adjoint_saved(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                                const float* wstates, const int32_t* wslot, float* chain, int chain_in,
                                const float* h, int n_adc, float* lam, float* gseg, int seg_mask, int grid,
                                int32_t* status, void* stream) {
    if (!wslot) return BP_E_ARG;
    return adjoint_impl(spins, sens, n, n_coils, segs, seg64, windows, wa, wb, seg0, seg_len, wstates, h, n_adc, lam,
                        nullptr, nullptr, gseg, seg_mask, grid, status, stream, nullptr, nullptr, wslot, chain,
                        chain_in);
}

extern "C" int bp_adjoint_physics(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                  const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                                  const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc,
                                  float* gseg, int seg_mask, int grid, const BpPhysics* ph, float* gconc,
                                  int32_t* status, void* stream) {
    if (!ph) return BP_E_ARG;
    return adjoint_impl(spins, sens, n, n_coils, segs, seg64, windows, wa, wb, seg0, seg_len, wstates, h, n_adc, lam,
                        gs, gc, gseg, seg_mask, grid, status, stream, ph, gconc);
}

extern "C" int bp_seg_reduce(const float* gseg, int n_cta, int seg_len, int seg0, double* seg, void* stream) {
    if (!gseg || !seg || n_cta < 1 || seg_len < 0 || seg0 < 0) return BP_E_ARG;
    if (seg_len == 0) return BP_OK;
    const int total = seg_len * N_SG, threads = 256;
    bp_seg_reduce_kernel<<<(total + threads - 1) / threads, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        gseg, n_cta, seg_len, seg0, seg);
    return cudaGetLastError() == cudaSuccess ? BP_OK : BP_E_LAUNCH;
}

// ---- The adjoint sweep for callers that cannot allocate device memory ----
//
// bp_adjoint needs a scratch buffer for its per-CTA segment gradients (`gseg`), which its callers allocate. Some
// callers of this library cannot: a host runtime that hands the library a fixed set of buffers sized at start-up
// and forbids allocation while it runs, or a foreign-language binding (Go, Java, JavaScript) that passes device
// pointers in but has no way to call cudaMalloc; and cudaFree synchronises the whole device, which such callers
// must not trigger. For them this variant keeps that scratch in a file-scope array in device memory, so the call
// allocates nothing. The array is BP_NOALLOC_SCRATCH_FLOATS floats (8 MiB); every GPU that loads the library
// holds it until the process exits.
#define BP_NOALLOC_SCRATCH_FLOATS (2 * 1024 * 1024)

static __device__ __align__(256) float bp_noalloc_scratch[BP_NOALLOC_SCRATCH_FLOATS];

// Device address of the array per device, looked up once per device with that device current (in host code the
// array's name is only a host-side stand-in, not a device address). std::call_once makes the lookup safe from
// several host threads. A cudaDeviceReset unloads the module, which leaves the stored address stale: callers of
// this entry point must not reset the device between calls.
static std::once_flag g_noalloc_once[64];
static float* g_noalloc_ptr[64];
static int g_noalloc_code[64];

static int noalloc_scratch(float** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BP_E_LAUNCH;
    std::call_once(g_noalloc_once[dev], [dev] {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, bp_noalloc_scratch) != cudaSuccess || p == nullptr) {
            g_noalloc_code[dev] = BP_E_LAUNCH;
            return;
        }
        g_noalloc_ptr[dev] = static_cast<float*>(p);
        g_noalloc_code[dev] = BP_OK;
    });
    if (g_noalloc_code[dev] != BP_OK) return g_noalloc_code[dev];
    *out = g_noalloc_ptr[dev];
    return BP_OK;
}

extern "C" int bp_adjoint_noalloc(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                  const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                                  const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc,
                                  double* seg, int32_t* status, void* stream) {
    if (n < 1 || n_coils < 1 || n_coils > BP_MAX_COILS || wa < 0 || wb < wa || seg_len < 0 || seg0 < 0 || n_adc < 0)
        return BP_E_ARG;
    if (!spins || !sens || !segs || !seg64 || !windows || !wstates || !lam || !gs || !status) return BP_E_ARG;
    // one CTA needs seg_len * N_SG floats of the array; more CTAs share it up to its size
    const long long per_cta = (long long)seg_len * N_SG;
    if (seg && per_cta > BP_NOALLOC_SCRATCH_FLOATS) return BP_E_SIZE;
    if (wb == wa) return BP_OK;
    float* scratch = nullptr;
    int code = noalloc_scratch(&scratch);
    if (code != BP_OK) return code;
    int grid = bp_adjoint_grid(n, n_coils);
    if (grid < 1) return BP_E_LAUNCH;
    if (seg && per_cta > 0 && (long long)grid * per_cta > BP_NOALLOC_SCRATCH_FLOATS)
        grid = (int)(BP_NOALLOC_SCRATCH_FLOATS / per_cta);
    // the kernel clears each CTA's rows of the scratch before accumulating into them
    code = bp_adjoint(spins, sens, n, n_coils, segs, seg64, windows, wa, wb, seg0, seg_len, wstates, h, n_adc, lam, gs,
                      gc, seg ? scratch : nullptr, BP_SEG_ALL, grid, status, stream);
    if (code != BP_OK || !seg) return code;
    return bp_seg_reduce(scratch, grid, seg_len, seg0, seg, stream);
}
