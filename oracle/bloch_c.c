/* CPU float64 oracle of blochparty's plain-Bloch simulation in C, threaded over spins: TEST INFRASTRUCTURE ONLY.
 *
 * The same algorithm as oracle/bloch.py (which restates blochparty's core engine, engines/core.py), for the long
 * sequences of the measured workloads, where the Python restatement's per-segment overhead dominates (a
 * million-segment sequence takes minutes there whatever the spin count). Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU arms may load it, as the checker. It is pinned against blochparty itself through the golden
 * fixtures (tests/golden/*.npz, written by the reference's core) and against oracle/bloch.py on random cases.
 *
 * Per spin, in order (engines/core.py:322-334):
 *  - an RF segment (core.py:124-150, :71-74, :97-108): relax dt/2, rotate about w = -2 pi dt (b1 rf_x, b1 rf_y,
 *    G.r + dB0 + b0_offset) by the Rodrigues formula, relax dt/2; a sample at its end if it has one;
 *  - a run of RF-free segments up to the next RF segment or through a spoiling segment (core.py:268-319): with t,
 *    k and B the run's cumulative time, gradient moment and b0_offset integral (summed segment by segment),
 *    Mxy(t) = Mxy(0) exp(-t/T2) exp(-i 2 pi (k.r + dB0 t + B)) at every sample of the run, and the state at its
 *    end from the same closed form (Mz relaxing exactly);
 *  - a sample (core.py:182-187) adds (Mx + i My) coil to the coil sums, which are demodulated by
 *    exp(-i adc_phase) at the end, taken before the segment's spoil (core.py:391-392), which zeroes Mx and My.
 *
 * Threads: the sequence is cut into chunks at step boundaries, each holding at most CHUNK samples (more when one
 * free run has more); every thread steps its own contiguous block of spins through a chunk, summing its spins'
 * samples into a private float64 buffer; the buffers are then added to the signal in thread order, so the result
 * does not depend on timing.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_PI 6.283185307179586476925286766559
#define CHUNK 16384

typedef struct {
    int64_t n;
    const double *pos, *pd, *t1, *t2, *db0, *b1; /* pos [n][3]; b1 may be NULL */
    const double* coils;                          /* [n][C][2] */
    int n_coils;
    int64_t S;
    const double *dt, *rf, *grad, *b0_offset; /* rf [S][2], grad [S][3]; b0_offset may be NULL */
    const uint8_t *is_rf, *adc, *spoil;
} Case;

/* rotation of m about w by |w| (m cos + (w x m) sin(phi)/phi + w (w.m)(1 - cos phi)/phi^2), phi with the 1e-30
 * floor of the Python restatement under the square root; (1 - cos)/phi^2 as sinc(phi/2)^2 / 2 */
static void rotate(double* mx, double* my, double* mz, double wx, double wy, double wz) {
    const double phi = sqrt(wx * wx + wy * wy + wz * wz + 1e-30);
    const double cs = cos(phi);
    const double s1 = sin(phi) / phi;
    const double h = 0.5 * phi, sh = sin(h) / h;
    const double s2 = 0.5 * sh * sh;
    const double x = *mx, y = *my, z = *mz;
    const double dot = wx * x + wy * y + wz * z;
    *mx = cs * x + s1 * (wy * z - wz * y) + s2 * wx * dot;
    *my = cs * y + s1 * (wz * x - wx * z) + s2 * wy * dot;
    *mz = cs * z + s1 * (wx * y - wy * x) + s2 * wz * dot;
}

static void relax(double* mx, double* my, double* mz, double t, double pd, double t1, double t2) {
    const double e2 = exp(-t / t2), e1 = exp(-t / t1);
    *mx *= e2;
    *my *= e2;
    *mz = pd + (*mz - pd) * e1;
}

/* the steps [start, end) of the sequence: single RF segments, and runs of RF-free segments ending at a spoil or
 * before the next RF segment; returns the step count (steps has room for S + 1 boundaries) */
static int64_t plan_steps(const Case* c, int64_t* bounds) {
    int64_t k = 0, s = 0;
    bounds[k++] = 0;
    while (s < c->S) {
        int64_t e = s + 1;
        if (!c->is_rf[s])
            while (e < c->S && !c->is_rf[e] && !c->spoil[e - 1]) ++e;
        bounds[k++] = e;
        s = e;
    }
    return k - 1;
}

/* one spin through the steps [st0, st1), its samples added to acc[(row - row0)][C][2] */
static void spin_steps(const Case* c, int64_t j, const int64_t* bounds, const int64_t* rows, int64_t st0, int64_t st1,
                       int64_t row0, double* m, double* acc) {
    const int C = c->n_coils;
    const double px = c->pos[3 * j], py = c->pos[3 * j + 1], pz = c->pos[3 * j + 2];
    const double pd = c->pd[j], t1 = c->t1[j], t2 = c->t2[j], db0 = c->db0[j];
    const double b1 = c->b1 ? c->b1[j] : 1.0;
    const double* coil = c->coils + (size_t)j * C * 2;
    double mx = m[0], my = m[1], mz = m[2];
    for (int64_t st = st0; st < st1; ++st) {
        const int64_t a = bounds[st], b = bounds[st + 1];
        int64_t row = rows[st] - row0;
        if (c->is_rf[a]) {
            const double* g = c->grad + 3 * a;
            const double bz = px * g[0] + py * g[1] + pz * g[2] + db0 + (c->b0_offset ? c->b0_offset[a] : 0.0);
            const double half = 0.5 * c->dt[a];
            relax(&mx, &my, &mz, half, pd, t1, t2);
            const double w = -TWO_PI * c->dt[a];
            rotate(&mx, &my, &mz, w * c->rf[2 * a] * b1, w * c->rf[2 * a + 1] * b1, w * bz);
            relax(&mx, &my, &mz, half, pd, t1, t2);
            if (c->adc[a]) {
                double* r = acc + (size_t)row * C * 2;
                for (int q = 0; q < C; ++q) {
                    r[2 * q] += mx * coil[2 * q] - my * coil[2 * q + 1];
                    r[2 * q + 1] += mx * coil[2 * q + 1] + my * coil[2 * q];
                }
            }
        } else {
            double t = 0.0, kx = 0.0, ky = 0.0, kz = 0.0, ex = 0.0;
            for (int64_t s = a; s < b; ++s) {
                const double d = c->dt[s];
                t += d;
                kx += c->grad[3 * s] * d;
                ky += c->grad[3 * s + 1] * d;
                kz += c->grad[3 * s + 2] * d;
                if (c->b0_offset) ex += c->b0_offset[s] * d;
                if (c->adc[s]) {
                    const double cyc = px * kx + py * ky + pz * kz + db0 * t + ex;
                    const double e = exp(-t / t2), ph = -TWO_PI * cyc;
                    const double er = e * cos(ph), ei = e * sin(ph);
                    const double zr = mx * er - my * ei, zi = mx * ei + my * er;
                    double* r = acc + (size_t)row * C * 2;
                    for (int q = 0; q < C; ++q) {
                        r[2 * q] += zr * coil[2 * q] - zi * coil[2 * q + 1];
                        r[2 * q + 1] += zr * coil[2 * q + 1] + zi * coil[2 * q];
                    }
                    ++row;
                }
            }
            const double cyc = px * kx + py * ky + pz * kz + db0 * t + ex;
            const double cs = cos(-TWO_PI * cyc), sn = sin(-TWO_PI * cyc);
            const double x = mx, y = my;
            mx = cs * x - sn * y;
            my = sn * x + cs * y;
            relax(&mx, &my, &mz, t, pd, t1, t2);
        }
        if (c->spoil[b - 1]) mx = my = 0.0;
    }
    m[0] = mx, m[1] = my, m[2] = mz;
}

/* signal [C][n_adc][2] float64 (demodulated), m [n][3] in: the start state, out: the final state; threads (0: all)
 * and chunk (samples per chunk, 0: CHUNK) change nothing but the speed. Returns 0, or -1 when out of memory. */
int bp_oracle_simulate(int64_t n, const double* pos, const double* pd, const double* t1, const double* t2,
                       const double* db0, const double* b1, const double* coils, int n_coils, int64_t S,
                       const double* dt, const double* rf, const double* grad, const double* adc_phase,
                       const double* b0_offset, const uint8_t* is_rf, const uint8_t* adc, const uint8_t* spoil,
                       double* m, double* signal, int threads, int64_t chunk) {
    Case c = {n, pos, pd, t1, t2, db0, b1, coils, n_coils, S, dt, rf, grad, b0_offset, is_rf, adc, spoil};
    const int C = n_coils;
    int64_t n_adc = 0;
    for (int64_t s = 0; s < S; ++s) n_adc += adc[s] ? 1 : 0;
    int64_t* bounds = (int64_t*)malloc((size_t)(S + 2) * sizeof(int64_t));
    int64_t* rows = (int64_t*)malloc((size_t)(S + 2) * sizeof(int64_t));
    double* raw = (double*)calloc((size_t)(n_adc > 0 ? n_adc : 1) * C * 2, sizeof(double));
    if (!bounds || !rows || !raw) {
        free(bounds), free(rows), free(raw);
        return -1;
    }
    const int64_t n_steps = plan_steps(&c, bounds);
    rows[0] = 0;
    for (int64_t st = 0; st < n_steps; ++st) {
        int64_t k = 0;
        for (int64_t s = bounds[st]; s < bounds[st + 1]; ++s) k += adc[s] ? 1 : 0;
        rows[st + 1] = rows[st] + k;
    }
#ifdef _OPENMP
    if (threads < 1) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    if (threads > n) threads = (int)(n > 0 ? n : 1);
    int64_t max_chunk = chunk > 0 ? chunk : CHUNK;
    for (int64_t st = 0; st < n_steps; ++st)
        if (rows[st + 1] - rows[st] > max_chunk) max_chunk = rows[st + 1] - rows[st];
    double* priv = (double*)malloc((size_t)threads * max_chunk * C * 2 * sizeof(double));
    if (!priv) {
        free(bounds), free(rows), free(raw);
        return -1;
    }
    int64_t st0 = 0;
    while (st0 < n_steps) {
        int64_t st1 = st0 + 1;  /* the chunk's steps: as many as fit CHUNK samples (at least one) */
        while (st1 < n_steps && rows[st1 + 1] - rows[st0] <= max_chunk) ++st1;
        const int64_t row0 = rows[st0], nrow = rows[st1] - row0;
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
        {
#ifdef _OPENMP
            const int tid = omp_get_thread_num();
#else
            const int tid = 0;
#endif
            double* acc = priv + (size_t)tid * max_chunk * C * 2;
            memset(acc, 0, (size_t)nrow * C * 2 * sizeof(double));
            const int64_t j0 = n * tid / threads, j1 = n * (tid + 1) / threads;
            for (int64_t j = j0; j < j1; ++j) spin_steps(&c, j, bounds, rows, st0, st1, row0, m + 3 * j, acc);
        }
        for (int tid = 0; tid < threads; ++tid) {
            const double* acc = priv + (size_t)tid * max_chunk * C * 2;
            double* dst = raw + (size_t)row0 * C * 2;
            for (int64_t i = 0; i < nrow * C * 2; ++i) dst[i] += acc[i];
        }
        st0 = st1;
    }
    /* demodulation by exp(-i adc_phase), into [C][n_adc][2] */
    int64_t row = 0;
    for (int64_t s = 0; s < S; ++s) {
        if (!adc[s]) continue;
        const double cs = cos(adc_phase[s]), sn = sin(adc_phase[s]);
        for (int q = 0; q < C; ++q) {
            const double re = raw[((size_t)row * C + q) * 2], im = raw[((size_t)row * C + q) * 2 + 1];
            signal[((size_t)q * n_adc + row) * 2] = re * cs + im * sn;
            signal[((size_t)q * n_adc + row) * 2 + 1] = im * cs - re * sn;
        }
        ++row;
    }
    free(priv), free(bounds), free(rows), free(raw);
    return 0;
}
