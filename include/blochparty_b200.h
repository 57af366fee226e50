/* C ABI of the B200 Bloch-simulation library (libblochparty_b200.so).
 *
 * Every entry point takes plain pointers and sizes: device pointers for all arrays (allocated and owned by the
 * caller), a CUDA stream as `void*` (NULL: the legacy default stream), and returns an int status (BP_OK = 0).
 * Kernels are launched asynchronously on the stream; device-side failures (a bounded wait that gave up) are
 * OR-ed into the caller's `status` word, which the caller reads after synchronising. Nothing here allocates
 * device memory except where a comment says otherwise.
 *
 * These entry points replace the kernel launches of blochparty's GPU driver for static spins:
 * engines/gpu/cuda/rtc.py:116-126 (_Driver.launch of bloch_chunk / bloch_chunk_mma, bloch_replay,
 * bloch_adjoint_c*, seg_reduce), driven by engines/gpu/driver.py:_forward (:197-756) and
 * engines/gpu/adjoint.py:_GPUSimulate (:45-261).
 */
#ifndef BLOCHPARTY_B200_H
#define BLOCHPARTY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BP_OK 0
#define BP_E_ARG 1      /* invalid argument (size, null pointer, coil count) */
#define BP_E_ALIGN 2    /* a buffer that is TMA-copied is not 16-byte aligned */
#define BP_E_LAUNCH 3   /* the CUDA launch failed (cudaGetLastError) */
#define BP_E_SIZE 4     /* a size above a documented maximum */

#define BP_MAX_COILS 32 /* receive coils of the float32 readout */
#define BP_SEG_MAX 160  /* segments per window (one TMA-staged block; five CTAs per SM fit in shared memory) */
#define BP_ADJ_WIN 32   /* segments per adjoint window (recomputed into shared memory) */

/* Window planner (host code, no GPU): cuts `n_segments` segments with per-segment `flags` (bit 1 RF, 2 ADC,
 * 4 spoil) into consecutive windows of at most `seg_max` (<= BP_SEG_MAX) segments and `samp_max` ADC samples;
 * `breaks` (optional, n_segments bytes) forces a window to start at every segment whose byte is nonzero.
 * Writes 4 ints per window (first segment, end segment, first ADC row, samples) into `windows` (room for
 * `max_windows`) and the count into `*n_windows`. A window cut by one of the two limits ends on a multiple of
 * BP_ADJ_WIN segments whenever it still holds one (always for samp_max >= BP_ADJ_WIN), so limit cuts do not depend
 * on the breaks before them. Replaces the dispatch boundaries of engines/gpu/driver.py:617-627. Returns
 * BP_E_SIZE when `max_windows` is too small. */
int bp_plan_windows(const int32_t* flags, int64_t n_segments, int seg_max, int samp_max, const uint8_t* breaks,
                    int32_t* windows, int64_t max_windows, int64_t* n_windows);

/* Device buffer sizes (bytes) of one simulation, host arithmetic only (no GPU): what blochparty's driver sizes in
 * Python (engines/gpu/driver.py:109, engines/gpu/adjoint.py:146), for callers that allocate the buffers
 * themselves. bp_forward_workspace_bytes: the forward's state, raw coil sums, receiver phases, demodulated signal
 * and status word for n spins, n_adc samples and n_coils coils (`raw` and `signal` keep one row when n_adc = 0).
 * bp_adjoint_workspace_bytes: what the checkpointed adjoint adds for a sequence of n_segments segments: the
 * checkpoints (one [6][n] state per interval of checkpoint_every segments, a multiple of BP_ADJ_WIN; with
 * outer_every > 1 intervals per outer block, one state per block start plus one block's interval starts, which
 * the backward rebuilds by one more forward of every block: for sequences whose interval starts alone would not
 * fit the device, e.g. 11.8 M segments x 8.4 M spins), the window
 * states of one replayed interval (max_interval_windows + 1: the most adjoint windows in one interval, from the
 * caller's bp_plan_windows plan, and the state after them), the replayed state, the per-CTA segment gradients (`grid` = bp_adjoint_grid,
 * times the longest interval), the float64 segment gradients, lambda, the per-spin gradients, the coil gradients
 * and the signal's cotangent h. Return BP_OK, or BP_E_ARG. */
typedef struct {
    int64_t state, raw, psi, signal, status, total;
} BpForwardWorkspace;
typedef struct {
    int64_t checkpoints, wstates, replay_state, gseg, seg, lam, gs, gc, h, total;
} BpAdjointWorkspace;
int bp_forward_workspace_bytes(int n, int64_t n_adc, int n_coils, BpForwardWorkspace* out);
int bp_adjoint_workspace_bytes(int n, int64_t n_segments, int64_t n_adc, int n_coils, int checkpoint_every,
                               int max_interval_windows, int grid, int outer_every, BpAdjointWorkspace* out);

/* ADC samples per window that bp_forward's float32 readout accumulates for `n_coils` coils (0 if unsupported). */
int bp_forward_samp_max(int n_coils);

/* Forward propagation of windows [w_begin, w_end) (replaces bloch_chunk_mma, engines/gpu/cuda/kernels.cu.in:2-185,
 * and the dispatch loop engines/gpu/driver.py:658-698).
 *   spins   [8][n] float32: x y z [m], pd, r1 = 1/T1, r2 = 1/T2 [1/s], dB0 [Hz], B1 scale
 *   sens    [16 ceil(C/8)][n] float32: coil c real part at row 2c, imaginary at 2c+1, zero padding rows
 *   segs    [S] 32-byte segment records (dt, -2 pi dt rf_x, -2 pi dt rf_y, g dt (3), b0_offset dt, flags);
 *           flag bits: 1 RF, 2 ADC (sample after the segment), 4 spoil, 8 a free segment equal to the free segment
 *           before it, 16 an RF segment with the dt of the RF segment before it, 32 the same with its moments and
 *           offset too, 64 an RF segment whose rotation angle stays below 1/4 for every spin (optional: it only
 *           spares the kernels' tests of the rotation factors' series; blochparty_b200.engine.mark_small_rf sets
 *           it from a bound on the spins' extents)
 *   seg64   [S][4] float64: g dt (3), b0_offset dt (the free segments' phase, in float64)
 *   windows [n_windows][4] int32 from bp_plan_windows
 *   state   [6][n] float32 in/out: mx my mz and their compensation (low) parts
 *   raw     [n_adc][2C] float64, accumulated (+=) raw coil sums, not demodulated; NULL: no readout
 *   wstates NULL or [ceil((w_end - w_begin) / wstate_stride)][6][n]: the state at every stride-th window start
 *   max_ctas  0: one persistent CTA per resident slot; else at most this many CTAs */
int bp_forward(const float* spins, const float* sens, int n, int n_coils, const void* segs, const double* seg64,
               const int32_t* windows, int w_begin, int w_end, float* state, double* raw, float* wstates,
               int wstate_stride, int max_ctas, int32_t* status, void* stream);

/* bp_forward that saves the state at chosen window starts (the checkpointed forward of a simulation whose backward
 * needs no replay, see bp_adjoint_saved): wslot [n_windows] int32, wslot[w] >= 0 the slot of `wstates` ([slots][6][n]
 * float32) that takes window w's start state, -1 none. Otherwise as bp_forward (no counterpart in the reference,
 * whose checkpointed forward stores every interval start: engines/gpu/driver.py:658-662). */
int bp_forward_saving(const float* spins, const float* sens, int n, int n_coils, const void* segs, const double* seg64,
                      const int32_t* windows, int w_begin, int w_end, float* state, double* raw, const int32_t* wslot,
                      float* wstates, int max_ctas, int32_t* status, void* stream);

/* Readout runs through a nonuniform FFT (simulate(..., readout="nufft"); replaces the NUFFT readouts of
 * engines/gpu/cuda/kernels.cu.in:91-140 with engines/gpu/driver.py:236-266). A run is L consecutive samples with
 * one free segment's factors (dt, moments, offset), so spin j's samples are z1 q^p, p < L, q = e^(-dt r2)
 * e^(-2 pi i x), x the segment's phase in cycles mod 1. With the spins sorted by x (the run's class, host side),
 * bp_forward_nufft steps every window as bp_forward does, except a window that holds one run (run_of[w] = r >= 0):
 * there every spin adds its first sample, times exp(-2 pi i x floor(L/2)) and times exp(-tau_m r2) for each of the
 * M terms of the decay's time segmentation, onto an oversampled grid of G cells with the kernel
 * exp(beta (sqrt(1 - z^2) - 1)) over W cells (z = 2 (cell - x G) / W), coil by coil, and jumps over the run in one
 * free step. bp_nufft_finish then forms every run's samples, raw[rows[r] + p] += sum_m weights[m][p]
 * sum_g grid[r][g][m] exp(-2 pi i (p - floor(L/2)) g / G) in float64 (weights: the time-segmentation coefficient
 * of term m at sample p over G times the kernel's Fourier transform at p - floor(L/2)).
 *   run_of      [n_windows] int32: the run a window holds, or -1 (a run's window holds it alone, and its samples
 *               field is 0: the run's raw rows are filled by bp_nufft_finish)
 *   base        [n] int32: floor(x G) - W/2 + 1, the spin's first cell (taken modulo G)
 *   frac        [n] float32: x G - floor(x G)
 *   shift       [n] (float32, float32): exp(-2 pi i x floor(L/2)) (8-byte aligned)
 *   decay       [M][n] float32: exp(-tau_m r2)
 *   tile_cells  [ceil(n / 128)] (int32, int32): the cells [lo, hi) a tile of 128 spins reaches (at most W + 1 apart
 *               for the sorted spins; 8-byte aligned)
 *   grid        [runs][G][M][2C] float64, accumulated (+=)
 * At most 16 coils and (W + 1) M <= 64 / ceil(C / 8) (BP_E_SIZE otherwise); M <= BP_NUF_MAX_TERMS. */
#define BP_NUF_MAX_TERMS 6
typedef struct {
    const int32_t* run_of;
    const int32_t* base;
    const float* frac;
    const void* shift;
    const float* decay;
    const int32_t* tile_cells;
    double* grid;
    int G, W, M;
    float beta;
} BpNufft;
int bp_forward_nufft(const float* spins, const float* sens, int n, int n_coils, const void* segs, const double* seg64,
                     const int32_t* windows, int w_begin, int w_end, float* state, double* raw, int max_ctas,
                     const BpNufft* nu, int32_t* status, void* stream);
int bp_nufft_finish(const double* grid, const int32_t* run_rows, int n_runs, int G, int M, int L, int n_coils,
                    const double* weights, double* raw, void* stream);

/* The bound pool (magnetization transfer, rate model) and the scanner field model's concomitant fields, forward
 * (replaces the V=1 kernels of engines/gpu/cuda/kernels.cu.in:2-185 with the steps of
 * engines/gpu/shaders/common.metal:40-50 and :145-208, fed by engines/gpu/driver.py:377-440). bp_forward's
 * arguments and layouts, and:
 *   mt         nonzero: a bound pool. Its Mz exchanges with the water's (exact 2x2 step per segment), RF saturates
 *              it at W = w1^2 G(rf_freq - bz - dw); flag bit 128 (BP_BOUND_ONLY) marks an RF segment that only the
 *              pool feels (the water precesses about z alone)
 *   pool       [5][n] float32: f (pool size / free pool), k [1/s] (exchange rate from the bound pool), r1b = 1/T1b
 *              [1/s], T2b [s], dw [Hz] (the pool's resonance shift)
 *   bstate     [2][n] float32 in/out: the bound pool's Mz and its low part
 *   rf_freq    [S] float32: the RF's frequency per segment [Hz]
 *   line       float32: kind (1 Lorentzian, 2 super-Lorentzian), cutoff [Hz], ln x0, step, x_min, size, then `size`
 *              values ln F(x) at ln x = ln x0 + i step (the super-Lorentzian's integral; unused for kind 1)
 *   conc_mode  0 none, 1 leading-order concomitant field, 2 exact |B|
 *   conc       [7][n] float32: mode 1 the quadratic form's coefficients c (6; f_c = c . (gx^2, gy^2, gz^2, gx gy,
 *              gx gz, gy gz)); mode 2 the transverse field's rows ax (3), ay (3) and f0 [Hz]
 *   segq       [S][6] float64, mode 1: dt (gx^2, gy^2, gz^2, gx gy, gx gz, gy gz)
 *   wstates, wstate_stride  as bp_forward's (the replay of the adjoint; without a bound pool), or NULL, 0
 * Positions in `spins` are the encoding positions (gradient nonlinearity applied on the host); the concomitant
 * coefficients come from the true ones. No NUFFT runs. */
#define BP_BOUND_ONLY 128
typedef struct {
    int mt;
    int conc_mode;
    const float* pool;
    float* bstate;
    const float* rf_freq;
    const float* line;
    const float* conc;
    const double* segq;
    float* wstates;
    int wstate_stride;
} BpPhysics;
int bp_forward_physics(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                       const double* seg64, const int32_t* windows, int w_begin, int w_end, float* state, double* raw,
                       int max_ctas, const BpPhysics* ph, int32_t* status, void* stream);

/* Persistent grid (CTAs) that bp_forward launches for n spins and n_coils coils; negative on error. */
int bp_forward_grid(int n, int n_coils);

/* signal[c][t] = raw[t][c] exp(-i psi[t]) in float64, written as complex64 (interleaved float pairs), shape
 * (n_coils, n_adc) (replaces the host-side assembly engines/gpu/driver.py:699-702). */
int bp_signal_finish(const double* raw, const double* psi, int n_adc, int n_coils, void* out, void* stream);

/* Split-bfloat16 tensor-core readout (tcgen05): at most BP_MMA_MAX_COILS coils. The coil sensitivities are
 * first converted into per-128-spin-tile operand blocks ("A tiles", bp_mma_atiles_bytes(n) bytes, 16-byte aligned)
 * by bp_mma_atiles from the same [16][n] `sens` layout as bp_forward. No counterpart in the reference (its CUDA
 * engine's coil sum is float32 on the CUDA cores, engines/gpu/cuda/common.cuh:91-116; its Metal engine uses
 * simdgroup matrices, engines/gpu/shaders/common.metal:653-705). */
#define BP_MMA_MAX_COILS 8
int64_t bp_mma_atiles_bytes(int n);
int bp_mma_atiles(const float* sens, int n, int n_coils, void* atiles, void* stream);

/* bp_forward with the coil contraction on the tensor cores: D += A_hi B_hi + A_hi B_lo + A_lo B_hi in float32
 * (A: coil sensitivities, B: 16 samples' magnetization, both split into bfloat16 high and low parts), summed over
 * the CTA's tiles in tensor memory and added to the float64 `raw` per window. Windows must hold at most 64 samples
 * (bp_plan_windows with samp_max = 64). Same arguments as bp_forward otherwise (no window-state output). */
/* Persistent grid (CTAs) that bp_forward_mma launches for n spins; negative on error. */
int bp_forward_mma_grid(int n);
int bp_forward_mma(const float* spins, const void* atiles, int n, int n_coils, const void* segs, const double* seg64,
                   const int32_t* windows, int w_begin, int w_end, float* state, double* raw, int max_ctas,
                   int32_t* status, void* stream);

/* Grid (persistent CTAs) that bp_adjoint uses for n spins: size the first dimension of its `gseg` scratch with
 * it. Negative on error. */
int bp_adjoint_grid(int n, int n_coils);

/* Reverse sweep of one checkpoint interval (replaces bloch_adjoint_c<NC>, engines/gpu/cuda/adjoint.cu.in:5-121,
 * with the per-segment reverse of shaders/adjoint_common.metal:212-315). `windows` are adjoint windows (at most
 * BP_ADJ_WIN segments, boundaries on multiples of BP_ADJ_WIN), [wa, wb) the interval's, covering segments
 * [seg0, seg0 + seg_len).
 *   wstates [wb - wa + 1][6][n] the state at every window start (bp_forward replay of the interval, stride 1),
 *           then the state after the interval's last window (the replay's final state); the sweep without
 *           per-spin gradients integrates a window of RF segments backward from the state after it
 *   h       [n_adc][2C] float32 dL/d(raw coil sums) = dL/dsignal rotated by exp(+i psi), or NULL (8-byte
 *           aligned: BP_E_ALIGN otherwise); n_adc its rows
 *   lam     [3][n] in: dL/dm after the interval; out: dL/dm before it
 *   gs      [8][n] += dL/d(x, y, z, dB0, pd, r1, r2, b1)
 *   gc      [2C][n] += dL/d(coil c real, imaginary) at rows 2c, 2c+1, or NULL
 *   gseg    [grid][seg_len][8] scratch: per-CTA segment gradients (w.r.t. the record's dt, -2 pi dt rf_x,
 *           -2 pi dt rf_y, g dt (3), b0_offset dt), or NULL when no segment gradient is wanted
 *   seg_mask  the segment gradients wanted (BP_SEG_* bits; the others in gseg are left 0 or unreduced): only
 *           BP_SEG_WX | BP_SEG_WY (the RF alone) takes a cheaper reduction; plus BP_SPIN_NO_OFFSETS when the
 *           rows x, y, z and dB0 of gs are not wanted (left as they were): without coil gradients and without
 *           BP_SEG_DT, KX, KY, KZ, BETA, the sweep then skips the offsets' gradients altogether; or BP_SPIN_NONE
 *           when no row of gs is wanted at all
 *   grid    bp_adjoint_grid(n, n_coils)
 *   status  |= 2 (a malformed window) for every window the sweep skips: more than BP_ADJ_WIN segments, segments
 *           outside [seg0, seg0 + seg_len), or samples outside h's n_adc rows */
#define BP_SEG_DT 1
#define BP_SEG_WX 2
#define BP_SEG_WY 4
#define BP_SEG_KX 8
#define BP_SEG_KY 16
#define BP_SEG_KZ 32
#define BP_SEG_BETA 64
#define BP_SEG_ALL 127
#define BP_SPIN_NO_OFFSETS 128
#define BP_SPIN_NONE 256 /* no per-spin gradient wanted: gs is left as it was (with no coil gradients and no segment
                          * gradient but the RF's, windows of free segments then only carry lambda back) */
int bp_adjoint(const float* spins, const float* sens, int n, int n_coils, const void* segs, const double* seg64,
               const int32_t* windows, int wa, int wb, int seg0, int seg_len, const float* wstates, const float* h,
               int n_adc, float* lam, float* gs, float* gc, float* gseg, int seg_mask, int grid, int32_t* status,
               void* stream);

/* The reverse sweep of bp_adjoint without a replay, for the gradient of the RF waveform alone (seg_mask: BP_SEG_WX,
 * BP_SEG_WY and BP_SPIN_NONE; no coil, per-spin or offset gradient): its windows of free segments carry lambda alone,
 * and its windows of RF segments integrate their states backward from the state after them, so the only states it
 * needs are those after each run of such windows. Replaces the replay (bloch_replay,
 * engines/gpu/cuda/replay.cu.in:3-33) for sequences whose every adjoint window is one of those two kinds (a
 * window of RF segments with one dt and offset, no sample and no spoil, or of free segments with one set of factors
 * spoiling at most in its last segment) and whose spins' relaxation over an RF segment is invertible (T1, T2 above
 * 0.73 dt).
 *   wstates [slots][6][n] the saved states (bp_forward_saving)
 *   wslot   [n_windows + 1] int32: wslot[w] the slot of the state at window w's start (w = n_windows: after the
 *           last window), -1 where none was saved; a window of RF segments whose next window is not one needs it
 *   chain   [3][n] float32 in/out: the start state of the first window of [wa, wb) when it was integrated backward
 *           (read by the next call, for the interval before, as its chain_in state)
 *   chain_in  1 when window wb was integrated backward by the previous call (chain holds its start state)
 * The other arguments are bp_adjoint's (gs and gc are not used). status |= 4 when a window needed a state that was
 * not saved (its results are then invalid). */
int bp_adjoint_saved(const float* spins, const float* sens, int n, int n_coils, const void* segs, const double* seg64,
                     const int32_t* windows, int wa, int wb, int seg0, int seg_len, const float* wstates,
                     const int32_t* wslot, float* chain, int chain_in, const float* h, int n_adc, float* lam,
                     float* gseg, int seg_mask, int grid, int32_t* status, void* stream);

/* bp_adjoint with the scanner field model (gradients through the concomitant field; replaces the V=1 adjoint of
 * engines/gpu/cuda/adjoint.cu.in:5-121): `ph` as bp_forward_physics's (conc_mode 1 or 2, conc, segq; no bound pool:
 * mt must be 0), positions the encoding positions. Besides bp_adjoint's outputs, gconc [7][n] (+=, or NULL) receives
 * dL/d(the concomitant coefficients); the segment gradients include the concomitant field's dependence on the
 * moments and dt. The spins' position gradient is with respect to the encoding positions (the host chains it
 * through the nonlinearity). */
int bp_adjoint_physics(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                       const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                       const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc, float* gseg,
                       int seg_mask, int grid, const BpPhysics* ph, float* gconc, int32_t* status, void* stream);

/* seg[seg0 + s][k] += sum over the `n_cta` CTAs, in CTA order, of gseg[cta][s][k], in float64 (replaces
 * seg_reduce, engines/gpu/cuda/seg_reduce.cu:3-11). `seg` is [S][8] float64. */
int bp_seg_reduce(const float* gseg, int n_cta, int seg_len, int seg0, double* seg, void* stream);

/* bp_adjoint followed by bp_seg_reduce, without the caller's `gseg` scratch: for callers that cannot allocate
 * device memory (a host runtime that hands the library fixed buffers and forbids allocation while it runs, or a
 * foreign-language binding that passes device pointers but cannot call cudaMalloc). No counterpart in the
 * reference. The scratch lives in one file-scope device array of BP_NOALLOC_SCRATCH_BYTES (8 MiB) that every GPU
 * loading the library holds until exit; the call allocates nothing. Returns BP_E_SIZE when one CTA's share,
 * seg_len * 8 floats, exceeds the array; the grid is capped so that all CTAs fit. `seg` ([S][8] float64, +=) may
 * be NULL (no segment gradients). The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current, once per device: make it before any stream capture, and do
 * not reset the device (cudaDeviceReset) between calls. `n_adc` and `status` as in bp_adjoint. Every call uses the same
 * array: calls that overlap on the GPU (other streams, other host threads) race on it. Results equal bp_adjoint's
 * for lam, gs, gc, and seg up to the order of the float64 sum over CTAs. */
#define BP_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
int bp_adjoint_noalloc(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                       const double* seg64, const int32_t* windows, int wa, int wb, int seg0, int seg_len,
                       const float* wstates, const float* h, int n_adc, float* lam, float* gs, float* gc, double* seg,
                       int32_t* status, void* stream);

/* ---- reused pulses (replace the pulse maps of engines/gpu/cuda/pulse.cu.in:3-32 and the reuse branch of
 * engines/gpu/cuda/kernels.cu.in:141-165) ----
 * bp_pulse_maps: per spin, the affine map m -> M m + v of the k_steps RF segments [seg0, seg0 + k_steps) of `segs`
 * (plain RF steps composed in float64), into maps [12][n] float64 (M row-major, then v): BP_PULSE_MAP_BYTES per
 * spin. bp_pulse_apply: one occurrence of that pulse with its RF times exp(i phase) applied to the state [6][n]:
 * m -> Rz(phase) (M Rz(-phase) m + v), in float64 on the compensated state. */
#define BP_PULSE_MAP_BYTES 96
int bp_pulse_maps(const float* spins, int n, const void* segs, const double* seg64, int seg0, int k_steps,
                  double* maps, void* stream);
int bp_pulse_apply(const double* maps, int n, float* state, double phase, void* stream);

/* ---- learned RF surrogate (no counterpart in the reference; its nearest part is the exact per-spin map of a
 * reused pulse, engines/gpu/cuda/pulse.cu.in:3-32) ----
 * A 14 -> 64 -> 64 -> 64 -> 16 GELU network per shaped pulse. The training domain (dom_df, dom_b1, dom_z) bounds
 * |df| [Hz], |b1 - 1| and |z_rel| = |z - z0| / slice thickness (the host side's default: 200 Hz, 0.3, 2). A pulse
 * acts on a spin through f = df + G (z - z0) and b1 alone, so the inputs x are (f^, b^) = (f / F, (b1 - 1) / dom_b1),
 * F = dom_df + |G| dom_z thickness; the 14 features of the first layer are f^, b^, sin(k pi f^), cos(k pi f^) for
 * k = 1..6 (Fourier features). Outputs:
 *   [0, 4)   a unit quaternion (q0, q1, q2, q3), the Cayley-Klein pair alpha = q0 - i q3, beta = -i (q1 + i q2), of
 *            the pulse's rotation reduced by its free precession: R = Rz(wz/2) R~ Rz(wz/2), wz = -2 pi (G z + df) T;
 *   [4, 13)  dA~ / T (row-major), [13, 16) dC~ / T: the pulse's first-order relaxation terms beyond the relax (T/2)
 *            / rotate / relax (T/2) splitting, reduced like R (the pulse maps m to E (R - (r2 - r1) dA)(E m + c) +
 *            c + r1 pd dC, E and c the half-pulse relaxation and recovery).
 * Parameters: BP_MLP_PARAMS floats, W1 (64x14), b1, W2 (64x64), b2, W3 (64x64), b3, W4 (16x64), b4 (16). */
#define BP_MLP_PARAMS 10320
#define BP_MLP_INPUTS 2
#define BP_MLP_OUTPUTS 16

/* Training targets from the plain integrator: samples [n][3] (df [Hz], b1, z_rel) -> targets [n][16] (the outputs
 * above; and the whole rotations qfull [n][4] if not NULL); rf [k_steps][2] float64 [Hz], float64 throughout. */
int bp_pulse_targets(const double* rf, int k_steps, double dt, double gz, double thickness, double z0,
                     const float* samples, int n, float* targets, float* qfull, void* stream);

/* One training step's gradient: x [n][2] inputs (f^, b^), target [n][16]; loss (q0 - t0)^2 + vweight |q_vec -
 * t_vec|^2 + cweight |c - t_c|^2 per sample (q the normalised quaternion, c the 12 correction outputs; vweight > 0
 * weights the vector part: relative precision for small rotations); per-CTA partials gpart
 * [bp_mlp_grad_ctas(n)][BP_MLP_PARAMS] and loss sums lpart [bp_mlp_grad_ctas(n)] (scratch of the caller). */
int bp_mlp_grad_ctas(int n);
int bp_mlp_grad(const float* params, const float* x, const float* target, int n, float vweight, float cweight,
                float* gpart, float* lpart, void* stream);
/* grad = scale * (sum over CTAs in order of gpart), loss = scale * sum of lpart (scale = 1 / batch). */
int bp_mlp_reduce(const float* gpart, const float* lpart, int n_cta, float scale, float* grad, float* loss,
                  void* stream);
/* Adam step number `step` (1-based) on params with moments m, v. */
int bp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2, float eps,
            int step, void* stream);
/* The network's outputs y [n][16] (the quaternion normalised) for inputs x [n][2] (f^, b^). */
int bp_mlp_eval(const float* params, const float* x, int n, float* y, void* stream);

/* One pulse occurrence (segments [seg0, seg0 + k_steps) of `segs`, the trained waveform times exp(i phi0), slice
 * gradient gz along z, uniform offset b0off) applied to every spin's state [6][n]: inside the network's training
 * domain (|df| <= dom_df [Hz], |b1 - 1| <= dom_b1, |z_rel| <= dom_z slice widths) relax T/2, rotate by the
 * network's rotation, relax T/2; outside, the plain sub-stepped segments. counts (NULL or [2]) += spins through the
 * network, through the fallback. */
int bp_surrogate_pulse(const float* spins, float* state, int n, const float* params, const void* segs, int seg0,
                       int k_steps, double T, double gz, double thickness, double z0, double phi0, float b0off,
                       float dom_df, float dom_b1, float dom_z, int32_t* counts, void* stream);

/* The same occurrence with all four layers of the network on the tensor cores (tcgen05, split bfloat16: hi x hi +
 * hi x lo + lo x hi, float32 accumulation in tensor memory; 128 spins per tile, persistent CTAs, at most
 * `max_ctas` when > 0). `params_host` is the network in HOST memory (BP_MLP_PARAMS floats): the biases travel by
 * value in the launch's arguments; `wtiles` (device, 16-byte aligned, bp_mlp_wtiles_bytes() = 40960 bytes) holds
 * every weight split into bfloat16 high / low tiles by bp_mlp_wtiles (W1 zero-padded to 16 columns);
 * `status` |= 1 when a bounded wait on the weights' copy or an MMA ran out (the CTA then stops, its remaining
 * spins not written). Spins outside the domain are queued per CTA and stepped 128 at a time. bp_surrogate_pulse_mma_grid(n) returns the CTA count a launch for n spins uses (< 0: -error). */
int bp_mlp_wtiles_bytes(void);
int bp_mlp_wtiles(const float* params, void* tiles, void* stream);
int bp_surrogate_pulse_mma_grid(int n);
int bp_surrogate_pulse_mma(const float* spins, float* state, int n, const float* params_host, const void* wtiles,
                           const void* segs, int seg0, int k_steps, double T, double gz, double thickness, double z0,
                           double phi0, float b0off, float dom_df, float dom_b1, float dom_z, int32_t* counts,
                           int32_t* status, int max_ctas, void* stream);

/* ---- a forward with pulse occurrences replaced (the launch loop of pulses="reuse" / "surrogate") ----
 * bp_forward_spans steps windows ranges[0] = [w0, w1), then replaces span 0, steps ranges[1], replaces span 1, ...,
 * and steps ranges[n_spans] last: 2 n_spans + 1 launches issued from host code in one call (ranges: host int32
 * [n_spans + 1][2]; spans: host array). Every span replaces the segments [seg0, seg0 + k_steps) it names, which
 * the windows leave out. A span is one of:
 *   BP_SPAN_MAP      bp_pulse_apply(map, n, state, phase)                 (map: device [12][n] float64)
 *   BP_SPAN_NET_MMA  bp_surrogate_pulse_mma(..., params (host), wtiles, ...)
 *   BP_SPAN_NET_F32  bp_surrogate_pulse(..., params (device), ...)
 * with phase = the RF phase (phi0 of a network), and the network fields as in those calls. Returns the first
 * failing call's status (launches before it stay queued). */
#define BP_SPAN_MAP 0
#define BP_SPAN_NET_MMA 1
#define BP_SPAN_NET_F32 2
typedef struct {
    int32_t kind, seg0, k_steps;
    double phase;
    float b0off;
    const double* map;
    const float* params;
    const void* wtiles;
    double T, gz, thickness, z0;
    float dom_df, dom_b1, dom_z;
    int32_t* counts;
} BpSpan;
int bp_forward_spans(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                     const double* seg64, const int32_t* windows, const int32_t* ranges, int n_spans,
                     const BpSpan* spans, float* state, double* raw, int max_ctas, int32_t* status, void* stream);

/* Measurement kernel (the roofline denominator): 4 CTAs x 256 threads per SM, each thread `iters` x 128
 * independent FFMAs; `*flops` receives the flop count of the launch, which the caller divides by the launch's
 * CUDA-event duration. `out` needs 4 * SMs * 256 floats (never written in practice). */
int bp_ffma_peak(float* out, int iters, int64_t* flops, void* stream);
/* The same with paired FMAs (two per instruction on float pairs, 8 independent FMAs per thread per step). */
int bp_ffma2_peak(float* out, int iters, int64_t* flops, void* stream);

#ifdef __cplusplus
}
#endif

#endif
