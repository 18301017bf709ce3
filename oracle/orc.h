/*
 * orc.h -- CPU FP64 restatement of the msosm_gpu coherent-dedispersion path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product
 * path (msosm_gpu_b200, libmsosm_b200.so) never links, loads or calls it.
 *
 * Every function cites the reference file:line whose behaviour it restates.
 * Arithmetic follows the reference's float/double promotion rules exactly
 * where those rules decide an integer (Nd, M, delaycount, delay_points,
 * fold period boundaries); FFTs and filtering run in FP64.
 */
#ifndef MSOSM_ORC_H
#define MSOSM_ORC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- filter design / segmentation (reference L3) ------------ */

/* Nd = floor(kdm*dm*(1/f0^2 - 1/(f0+bw)^2) / (1/fs)), fs = bw.
 * dedispersion/msosm/msosm_prepare.cpp:3-8.  Negative results (dm < 0) are
 * undefined in the reference; here they give 0. */
unsigned long orc_nd(float bw, float dm, float f0);

/* MS-OSM minimum filter order 2^ceil(log2(2*sqrt(Nd))).
 * dedispersion/msosm/msosm_prepare.cpp:17-24.  Nd == 0 gives 0. */
unsigned long orc_msosm_min_order(unsigned long Nd);

/* OSM minimum filter order 2*next_power_of_2((int)Nd).
 * dedispersion/overlap_save/osm_prepare.cpp:17-30,86-99. */
unsigned long orc_osm_min_order(unsigned long Nd);

/* delaycount = (int)ceil(Nd / (float)M).  msosm_prepare.cpp:88. */
int orc_delaycount(unsigned long Nd, unsigned long M);

/* Per-bin integer block delay delay_points[2M] (values 0..delaycount-1).
 * dedispersion/msosm/msosm_prepare.cpp:86-152.  Returns delaycount.
 * delaycount == 0 (Nd == 0, e.g. dm == 0) leaves the reference's array
 * uninitialised; here every bin gets delay 0. */
int orc_segmentation(float bw, float dm, float f0, unsigned long Nd,
                     unsigned long M, int *delay_points);

/* Dedispersion filter H[2M] (interleaved re,im doubles).
 * dedispersion/msosm/msosm_prepare.cpp:37-84 (identical in osm_prepare.cpp:37-84
 * and msosm_prepare_dm_concurrent.cpp:56-103): chirp sampled at M float-rounded
 * offsets, unnormalised inverse M-point DFT (the /M loop is overwritten by the
 * memcpy at :74, so H carries an extra factor M), zero-pad to 2M, forward DFT.
 * sign = -1 gives the dedispersion filter (h = cos - i sin); sign = +1 the
 * dispersion filter of the signal simulator (simulated_complex_signal.cpp:243-244). */
void orc_dedisp_params(float bw, float dm, float f0, unsigned long M,
                       int sign, double *H);

/* The float-rounded chirp phase at offset index i (0..M-1) of msosm_prepare.cpp:50-63. */
double orc_chirp_phase(float bw, float dm, float f0, unsigned long M,
                       unsigned long i);

/* ---------------- FFT (FP64, radix-2, in place) -------------------------- */

/* sign = -1: forward (exp(-2 pi i nk/N)), +1: inverse; unnormalised.
 * N must be a power of two. */
void orc_fft(double *x, unsigned long n, int sign);

/* ---------------- sample codecs (gpu/gpu_kernel.cu) ---------------------- */

/* x == 0 ? 0 : x - 32768  for both halves.  gpu/gpu_kernel.cu:276-299. */
void orc_decode_uint16(const uint16_t *src, size_t n_pairs, double *dst);
/* uint16(v + 32768*(v != 0)), truncating; out-of-range values saturate to
 * [0, 65535] (undefined in the reference).  gpu/gpu_kernel.cu:317-329. */
void orc_encode_uint16(const double *src, size_t n_pairs, uint16_t *dst);

/* ---------------- streaming MS-OSM / OSM (reference L2/L4) --------------- */

/* One object reproduces MSOSM_GPU_DM_concurrent (numDMs >= 1; numDMs == 1 is
 * MSOSM_GPU_BATCH) or, with osm != 0, OSM_GPU_DM_concurrent / OSM_GPU_BATCH.
 *   init:   dedispersion/msosm_dm_concurrent/msosm_gpu_dm_concurrent.cpp:22-108
 *   filter: msosm_gpu_dm_concurrent.cpp:119-151 with the scatter of
 *           gpu/gpu_kernel.cu:128-198 (ring slot (index+c+delay) % S) and the
 *           discard of gpu/gpu_kernel.cu:236-258.
 * The per-DM product ring of the reference is kept literally (FP64). */
typedef struct orc_dedisp orc_dedisp;

orc_dedisp *orc_dedisp_create(const float *bw, const float *dm, const float *f0,
                              int numDMs, unsigned long fftpoint, int count,
                              unsigned long input_size, int osm, int nthreads);
void orc_dedisp_destroy(orc_dedisp *d);
unsigned long orc_dedisp_M(const orc_dedisp *d);
int orc_dedisp_count(const orc_dedisp *d);
int orc_dedisp_ring_slots(const orc_dedisp *d);
int orc_dedisp_delaycount(const orc_dedisp *d, int i);
unsigned long orc_dedisp_Nd(const orc_dedisp *d, int i);
/* in: count*M complex (interleaved doubles).  out: numDMs*count*M complex,
 * layout [dm][c][m] (msosm_gpu_dm_concurrent.cpp:149-150). */
void orc_dedisp_filter(orc_dedisp *d, const double *in, double *out);

/* ---------------- detection + folding (folding/fold_gpu.cpp) ------------- */

/* sqrt(|a|^2 + |b|^2) per sample (b may be NULL).  gpu/gpu_kernel.cu:347-353. */
void orc_intensity(const double *a, const double *b, size_t n, double *out);

/* Fold_GPU state machine.  folding/fold_gpu.cpp:3-194.
 * time_bin == (unsigned long)-1 keeps period_samples bins.
 * accumulate_float != 0 sums in float exactly like the reference (for
 * bit-exact golden checks); 0 sums in double. */
typedef struct orc_fold orc_fold;
orc_fold *orc_fold_create(float period, float fs, unsigned long size,
                          unsigned long time_bin, int accumulate_float);
void orc_fold_destroy(orc_fold *f);
void orc_fold_discard_samples(orc_fold *f, unsigned long Nd);   /* :29-33 */
void orc_fold_data(orc_fold *f, const double *intensity);      /* :48-173, size samples */
unsigned long orc_fold_period_samples(const orc_fold *f);
unsigned long orc_fold_time_bin(const orc_fold *f);
/* folded_data after fold_data_bins (:175-194); time_bin values. */
void orc_fold_data_bins(orc_fold *f, double *out);

/* Period starts of the same state machine in global sample index:
 * start[p] for p = 0..n_periods (start[0] = 0).  Returns how many entries
 * were written (<= cap).  Used to check the device fold's period table. */
size_t orc_fold_period_starts(float period, float fs, unsigned long total,
                              int64_t *start, size_t cap);

/* ---------------- simulated pulsar (simulated_pulsar/) ------------------- */

/* SimulatedComplexSignal::generate_pulsar_signal without noise:
 * simulated_pulsar/simulated_complex_signal.cpp:40-175 (two unit deltas at
 * Np/2 and Np/2+2, dispersed by the +phase chirp, summed over range periods),
 * tiled `repeat` times.  out: repeat*Np complex.  Returns Np. */
unsigned long orc_simulate_two_spike(float bw, float dm, float f0, float period,
                                     unsigned long repeat, double *out,
                                     unsigned long cap);

/* Threads used by the parallel parts (OpenMP); <= 0 means all. */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
