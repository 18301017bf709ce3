/*
 * msosm_b200.h -- C ABI of the B200 (sm_100a) coherent-dedispersion library.
 *
 * Drop-in boundary for the hot path of msosm_gpu: MS-OSM (multi-segment
 * overlap-save) and OSM coherent dedispersion of complex baseband for one or
 * many DM trials, detection and phase folding.  Plain C types only; every
 * entry point returns an msosm_status (0 = OK) and never exits the process.
 * The reference interface each entry point replaces is cited beside it
 * (paths inside the msosm_gpu tree).
 *
 * Memory: a handle owns its device buffers.  Input/output pointers may be
 * host (pageable or pinned) or device pointers; host pointers are copied
 * inside the call.  Calls on one handle are stream-ordered on the handle's
 * stream; a handle is not thread-safe (one host thread per handle).
 */
#ifndef MSOSM_B200_H
#define MSOSM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MSOSM_API __attribute__((visibility("default")))
#else
#define MSOSM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference prints and calls exit(1) instead:
 *      gpu/include/gpu_common.cuh:41-61) ---------------------------------- */
typedef int msosm_status;
#define MSOSM_OK 0
#define MSOSM_ERR_BAD_ARG 1     /* invalid parameter or size */
#define MSOSM_ERR_OOM 2         /* device allocation failed */
#define MSOSM_ERR_CUDA 3        /* CUDA runtime error (message via msosm_last_error) */
#define MSOSM_ERR_TIMEOUT 4     /* a bounded device wait expired */
#define MSOSM_ERR_UNSUPPORTED 5 /* size/mode not built (e.g. FFT size outside 2^5..2^14) */
#define MSOSM_ERR_STATE 6       /* call out of order (e.g. fold not configured) */
#define MSOSM_ERR_NO_DEVICE 7   /* no CUDA device visible */

/* Packed offset-binary sample pair, 0 = blank.
 * Replaces `struct uint16_pair` (utils/include/globals.h:21-25). */
typedef struct msosm_uint16_pair {
    uint16_t first;
    uint16_t second;
} msosm_uint16_pair;

/* Complex sample, layout of cufftComplex (utils/include/globals.h:28). */
typedef struct msosm_complex {
    float x;
    float y;
} msosm_complex;

/* Thread-local message for the last non-OK status of this thread. */
MSOSM_API const char *msosm_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
MSOSM_API int msosm_version(void);
/* Number of CUDA devices (0 on a machine without a GPU; never fails). */
MSOSM_API int msosm_device_count(void);

/* ======================================================================
 * Filter design and segmentation (host math, reference L3)
 * ====================================================================== */

/* Dispersion smear in samples: floor(kdm*dm*(1/f0^2-1/(f0+bw)^2)*fs), fs=bw,
 * kdm=4.15e15, f0 = lower band edge in Hz.  dm <= 0 gives 0.
 * Replaces Prepare_MSOSM::Prepare_MSOSM (dedispersion/msosm/msosm_prepare.cpp:3-15). */
MSOSM_API msosm_status msosm_prepare_nd(float bw, float dm, float f0, unsigned long *Nd);

/* MS-OSM minimum filter order 2^ceil(log2(2*sqrt(Nd))).
 * Replaces Prepare_MSOSM::calculate_min_order (msosm_prepare.cpp:17-30). */
MSOSM_API msosm_status msosm_prepare_min_order_msosm(unsigned long Nd, unsigned long *M_min);

/* OSM minimum filter order 2*next_power_of_2(Nd).
 * Replaces Prepare_OSM::calculate_min_order (dedispersion/overlap_save/osm_prepare.cpp:17-30). */
MSOSM_API msosm_status msosm_prepare_min_order_osm(unsigned long Nd, unsigned long *M_min);

/* Per-bin block delays delay_points[2M] and their count.
 * Replaces Prepare_MSOSM::segmentation (msosm_prepare.cpp:86-152).  Nd == 0
 * (undefined in the reference) gives delaycount 0 and all delays 0. */
MSOSM_API msosm_status msosm_prepare_segmentation(float bw, float dm, float f0, unsigned long M,
                                        int *delaycount, int *delay_points);

/* Dedispersion filter H[2M] exactly as the reference designs it (chirp phase
 * in FP64 on the GPU, unnormalised M-point inverse DFT, zero pad, 2M-point
 * DFT; the extra factor M of the reference is kept).  Needs a GPU.  dm < 0
 * returns MSOSM_ERR_BAD_ARG, as msosm_dedisp_create does.
 * Replaces Prepare_MSOSM::generate_dedisp_params (msosm_prepare.cpp:37-84). */
MSOSM_API msosm_status msosm_prepare_dedisp_params(float bw, float dm, float f0, unsigned long M,
                                         msosm_complex *H);

/* Allocation-free variant of msosm_prepare_dedisp_params.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc: a pipeline that
 * reserves all of its device memory before an observation and may not
 * allocate while samples stream in, a host framework whose allocator owns the
 * device, code that redesigns one trial's filter in the middle of a pass
 * without the device-wide synchronisation cudaMalloc/cudaFree bring.
 * The caller passes H_device, a DEVICE buffer of 2M complex values on the
 * current device (memory of another device returns MSOSM_ERR_BAD_ARG); the
 * design runs asynchronously on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and writes H there, in the reference's scaling.  Its
 * arguments are checked as msosm_prepare_dedisp_params checks them.
 * M: a power of two, 32 <= M <= 8192 (FFT 64..16384 points); anything else
 * returns MSOSM_ERR_BAD_ARG.  Calls no cudaMalloc, cudaFree or allocating
 * library routine.  Scratch (twiddle tables, chirp parameters) lives in one
 * fixed 196,864-byte device array inside the library, which every GPU that
 * loads the library holds until the process exits.  All calls on a device
 * share it: calls whose work overlaps on the GPU (two streams, two host
 * threads) race on it and must be serialised by the caller.  Each call
 * rewrites every scratch byte it reads, so nothing carries over between
 * calls.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture. */
MSOSM_API msosm_status msosm_prepare_dedisp_params_noalloc(float bw, float dm, float f0, unsigned long M,
                                                           msosm_complex *H_device, void *stream);

/* ======================================================================
 * Dedisperser: N DM trials over one input stream
 * ====================================================================== */

typedef struct msosm_dedisp msosm_dedisp;

/* flags for msosm_dedisp_create */
#define MSOSM_FLAG_OSM 0x1u      /* classical overlap-save (OSM_GPU_*) instead of MS-OSM */
#define MSOSM_FLAG_NO_SERIES 0x2u /* do not materialise the dedispersed series (fold only) */
/* Inverse transforms on the tensor cores: f16 operands with a power-of-two
 * scale per work item, f32 accumulation.  No counterpart in the reference
 * (its inverse transform is the FP32 cuFFT).  FFT sizes 4096, 8192 and
 * 16384 (other sizes return MSOSM_ERR_UNSUPPORTED).  Relative RMS error of the series
 * against FP64: about 5e-4; folded profiles much lower. */
#define MSOSM_FLAG_TENSOR_F16 0x4u
/* As MSOSM_FLAG_TENSOR_F16 with bf16 operands (no scaling needed; relative
 * RMS error of the series against FP64 about 4e-3). */
#define MSOSM_FLAG_TENSOR_BF16 0x8u
/* With MSOSM_FLAG_OSM only: the filter designed from the +phase chirp, the
 * dispersion filter of the reference's signal simulator
 * (simulated_pulsar/simulated_complex_signal.cpp:91-107), instead of the
 * dedispersion filter; the output is half the dispersed input, delayed by
 * M - Nd samples at the top of the band. */
#define MSOSM_FLAG_DISPERSE 0x10u

typedef struct msosm_dedisp_info {
    unsigned long M;        /* hop / filter order; FFT size is 2M */
    unsigned long fftpoint; /* 2M */
    unsigned long M_min;    /* largest minimum order over the trials */
    int count;              /* FFT blocks per filter call; a call takes count*M samples */
    int numDMs;
    int ring_slots;         /* spectrum history ring depth */
    int max_delaycount;
    unsigned int flags;
    unsigned long long calls;       /* filter calls done */
    unsigned long long device_bytes; /* device memory held by the handle */
} msosm_dedisp_info;

/* Create and initialise.  bw/dm/f0 are per-trial arrays of numDMs (f0 =
 * lower band edge, Hz).  fftpoint 0 = minimum; a smaller-than-minimum FFT is
 * raised to the minimum (the reference prints a warning and does the same).
 * input_size != 0 sets count = input_size / M.  All trials must share bw and
 * f0 (one input stream).  Replaces MSOSM_GPU_DM_concurrent::
 * MSOSM_GPU_DM_concurrent + initialize_uint16
 * (dedispersion/msosm_dm_concurrent/msosm_gpu_dm_concurrent.cpp:3-108);
 * with numDMs == 1 MSOSM_GPU_BATCH (dedispersion/msosm/msosm_gpu_batch.cpp:10-49);
 * with MSOSM_FLAG_OSM OSM_GPU_BATCH / OSM_GPU_DM_concurrent
 * (dedispersion/overlap_save/osm_gpu_batch.cpp:19-92,
 *  dedispersion/overlap_save_dm_concurrent/osm_gpu_dm_concurrent.cpp:15-75). */
MSOSM_API msosm_status msosm_dedisp_create(const float *bw, const float *dm, const float *f0, int numDMs,
                                 unsigned long fftpoint, int count, unsigned long input_size,
                                 unsigned int flags, msosm_dedisp **out);
MSOSM_API msosm_status msosm_dedisp_destroy(msosm_dedisp *d);
MSOSM_API msosm_status msosm_dedisp_get_info(const msosm_dedisp *d, msosm_dedisp_info *info);

/* Per-trial parameters as computed at create (arrays of numDMs). */
MSOSM_API msosm_status msosm_dedisp_get_nd(const msosm_dedisp *d, unsigned long *Nd);
MSOSM_API msosm_status msosm_dedisp_get_delaycount(const msosm_dedisp *d, int *delaycount);
/* delay_points of trial i, 2M ints (Prepare_*::delay_points). */
MSOSM_API msosm_status msosm_dedisp_get_delay_points(const msosm_dedisp *d, int i, int *delay_points);
/* H of trial i, 2M complex, in the reference's scaling (Prepare_*::dedisp_params). */
MSOSM_API msosm_status msosm_dedisp_get_dedisp_params(const msosm_dedisp *d, int i, msosm_complex *H);

/* Run the CUDA stream of this handle (a cudaStream_t, 0 = the handle's own). */
MSOSM_API msosm_status msosm_dedisp_set_stream(msosm_dedisp *d, void *stream);

/* Dedisperse the next count*M samples (all trials).  Replaces
 * filter_block_uint16 (msosm_gpu_dm_concurrent.cpp:119-151,
 * msosm_gpu_batch.cpp:75-94, osm_gpu_batch.cpp:94-123).  The input is
 * offset-binary (x == 0 is blank, else x - 32768). */
MSOSM_API msosm_status msosm_dedisp_filter_block_uint16(msosm_dedisp *d, const msosm_uint16_pair *input);
/* Same for complex64 input (the reference has no such entry point). */
MSOSM_API msosm_status msosm_dedisp_filter_block_c64(msosm_dedisp *d, const msosm_complex *input);

/* Copy the dedispersed series of the last call: numDMs*count*M + 1 elements,
 * layout [dm][count*M] plus a trailing zero element, as the reference.
 * Scaling is the reference's (half the normalised convolution).  Blocks
 * until the copy is done.  Replaces get_output(Complex*)
 * (msosm_gpu_dm_concurrent.cpp:153-165, msosm_gpu_batch.cpp:96-99). */
MSOSM_API msosm_status msosm_dedisp_get_output_c64(msosm_dedisp *d, msosm_complex *out);
/* Same, requantised to offset-binary (v + 32768 truncated, 0 stays 0,
 * saturating).  Replaces get_output(uint16_pair*) (:167-180) with
 * complexToUint16 (gpu/gpu_kernel.cu:317-329). */
MSOSM_API msosm_status msosm_dedisp_get_output_uint16(msosm_dedisp *d, msosm_uint16_pair *out);
/* Device pointer of the series of the last call ([dm][count*M], complex). */
MSOSM_API msosm_status msosm_dedisp_output_device_ptr(msosm_dedisp *d, msosm_complex **ptr);

/* ---- batches: many observations in one launch ---------------------------
 * One filter call of each of n handles (observations of any length, band
 * and trial grid) with one persistent dedispersion launch per group of up to
 * 128 handles that run the same tensor-core kernel variant (FFT size, operand
 * type, series/fold): the group's work items (handle, trial, block range)
 * are taken by the CTAs from a counter, the largest handle's first, so
 * uneven observations share the GPU without a tail per observation.  Handles of
 * other kernels (FP32, FFT sizes without a tensor-core transform, the
 * four-step sizes) run their calls one after another in the same batch call.
 * The reference has no counterpart (it dedisperses one observation per
 * object); its one-launch pattern for many trials of one observation is
 * MSOSM_GPU_DM_concurrent::filter_block_uint16
 * (dedispersion/msosm_dm_concurrent/msosm_gpu_dm_concurrent.cpp:119-151).
 * msosm_batch_create puts every handle on the batch's stream (until the
 * batch is destroyed); a handle belongs to one batch at a time.  inputs[i]
 * holds count*M samples of handle i (host or device pointers), all of one
 * kind.  Results per handle: msosm_dedisp_get_output_* / get_profiles, as
 * after msosm_dedisp_filter_block_*: each handle keeps its own work items
 * (trial, block range), so its results equal those of its own calls. */
typedef struct msosm_batch msosm_batch;
#define MSOSM_INPUT_UINT16 0
#define MSOSM_INPUT_C64 1
MSOSM_API msosm_status msosm_batch_create(msosm_dedisp *const *handles, int n, msosm_batch **out);
MSOSM_API msosm_status msosm_batch_destroy(msosm_batch *b);
MSOSM_API msosm_status msosm_batch_filter(msosm_batch *b, const void *const *inputs, int input_kind);
/* Run the batch and its handles on a CUDA stream (a cudaStream_t; NULL =
 * the batch's own). */
MSOSM_API msosm_status msosm_batch_set_stream(msosm_batch *b, void *stream);
/* Waits for the batch's work; MSOSM_ERR_TIMEOUT as msosm_dedisp_synchronize. */
MSOSM_API msosm_status msosm_batch_synchronize(msosm_batch *b);
/* Kernel groups, launches per call (groups + handles run alone), work items
 * per call over the groups; any pointer may be NULL. */
MSOSM_API msosm_status msosm_batch_get_info(const msosm_batch *b, int *groups, int *launches_per_call, int *items);

/* ---- fused detection + folding ------------------------------------------
 * Folding follows Fold_GPU (folding/fold_gpu.cpp:3-194): period_samples =
 * (unsigned long)(period*fs), one sample skipped whenever the float drift
 * exceeds 1, the first ceil(discard_Nd/(period*fs)) periods discarded, only
 * complete periods folded, then averaged into time_bin bins of
 * period_samples/time_bin samples (tail dropped).  time_bin 0 keeps
 * period_samples bins (no averaging).  Detection per sample: */
#define MSOSM_DETECT_POWER 0     /* |y|^2 */
#define MSOSM_DETECT_AMPLITUDE 1 /* |y|, the reference's calculateIntensity with one pol */
MSOSM_API msosm_status msosm_dedisp_fold_init(msosm_dedisp *d, float period, float fs, unsigned long time_bin,
                                    unsigned long discard_Nd, int detect);
/* Folded profiles so far, numDMs x time_bin floats (fold_data_bins). */
MSOSM_API msosm_status msosm_dedisp_get_profiles(msosm_dedisp *d, float *out);
/* Number of whole periods folded so far. */
MSOSM_API msosm_status msosm_dedisp_folded_periods(const msosm_dedisp *d, unsigned long long *n);

/* Start a new input stream on the same handle (same band, trials and FFT):
 * the previous stream's history is forgotten, as if the handle had just been
 * created, and folding is unconfigured (call msosm_dedisp_fold_init again,
 * with a new period if wanted).  No counterpart in the reference, whose
 * objects serve one stream.  Waits for the handle's work. */
MSOSM_API msosm_status msosm_dedisp_reset(msosm_dedisp *d);

/* Wait for all work of the handle (MSOSM_GPU_DM_concurrent::synchronize). */
MSOSM_API msosm_status msosm_dedisp_synchronize(msosm_dedisp *d);

/* ======================================================================
 * Fold_GPU: detection and folding of materialised series
 * ====================================================================== */

/* Folds a stream of intensities chunk by chunk with the Fold_GPU state
 * machine (folding/fold_gpu.cpp:48-173) on the device.  size: samples per
 * chunk; time_bin 0 or (unsigned long)-1 keeps period_samples bins.
 * Replaces Fold_GPU::Fold_GPU (fold_gpu.cpp:3-27).  Without a discard (or
 * with Nd = 0) every period is folded; the reference folds nothing then. */
typedef struct msosm_fold msosm_fold;
MSOSM_API msosm_status msosm_fold_create(float period, float fs, unsigned long size, unsigned long time_bin,
                                         msosm_fold **out);
MSOSM_API msosm_status msosm_fold_destroy(msosm_fold *f);
/* Fold_GPU::discard_samples (fold_gpu.cpp:29-33): skip ceil(Nd/(period*fs))
 * periods.  Call before the first msosm_fold_data. */
MSOSM_API msosm_status msosm_fold_discard_samples(msosm_fold *f, unsigned long Nd);
/* Intensity sqrt(|a|^2 + |b|^2) of two DEVICE series of size samples (b may
 * be NULL for one polarisation) into the fold's buffer.  Replaces
 * Fold_GPU::calculate_intensity (fold_gpu.cpp:35-43) and calculateIntensity
 * (gpu/gpu_kernel.cu:347-353); the result stays on the device.  The raw
 * pointers carry no ordering, so this waits for the whole device first; with
 * dedisperser handles use msosm_fold_calculate_intensity_dedisp. */
MSOSM_API msosm_status msosm_fold_calculate_intensity(msosm_fold *f, const msosm_complex *a, const msosm_complex *b);
/* Same from the last series of one or two dedisperser handles (each
 * count*M == size samples, one trial; b may be NULL), ordered after their
 * filter calls by events; their next filter call waits for this read. */
MSOSM_API msosm_status msosm_fold_calculate_intensity_dedisp(msosm_fold *f, msosm_dedisp *a, msosm_dedisp *b);
/* Load size intensities from a host or device float array instead. */
MSOSM_API msosm_status msosm_fold_set_intensity(msosm_fold *f, const float *intensity);
/* Copy the current intensities to host memory (Fold_GPU::total_intensity). */
MSOSM_API msosm_status msosm_fold_get_intensity(msosm_fold *f, float *out);
/* Fold the current chunk (Fold_GPU::fold_data, fold_gpu.cpp:48-173). */
MSOSM_API msosm_status msosm_fold_data(msosm_fold *f);
/* Folded profile, time_bin floats (Fold_GPU::fold_data_bins, fold_gpu.cpp:175-194). */
MSOSM_API msosm_status msosm_fold_data_bins(msosm_fold *f, float *out);
/* period_samples and time_bin as Fold_GPU computes them. */
MSOSM_API msosm_status msosm_fold_get_shape(const msosm_fold *f, unsigned long *period_samples,
                                            unsigned long *time_bin);

/* ---- per-stage device timing -------------------------------------------
 * CUDA events recorded on the handle's stream around each stage of every
 * filter call (no effect on results).  Enabling resets the counters;
 * msosm_dedisp_get_timing waits for the handle's work and sums. */
typedef struct msosm_timing {
    double forward_ms;  /* decode + forward FFT into the spectrum ring */
    double dedisp_ms;   /* fused gather x H, inverse FFT, discard, detect, fold */
    double fold_ms;     /* fold bookkeeping: partial-row clears, ordered reduce, flush */
    double h2d_ms;      /* host-to-device input staging (copy stream) */
    unsigned long long calls;           /* filter calls timed */
    unsigned long long kernel_launches; /* kernels of this library launched by those calls */
} msosm_timing;
MSOSM_API msosm_status msosm_dedisp_enable_timing(msosm_dedisp *d, int on);
MSOSM_API msosm_status msosm_dedisp_get_timing(msosm_dedisp *d, msosm_timing *t);

/* ======================================================================
 * Introspection for tests (host only, no GPU needed)
 * ====================================================================== */

/* Destination of every output sample of one fold chunk under the Fold_GPU
 * state machine (folding/fold_gpu.cpp:48-173), as the device fold uses it:
 * dest[i] = -1 if sample i is not folded (skipped by the drift, discarded, or
 * in a period processed before the fold became ready), else
 * (period_index << 32) | phase, phase in [0, period_samples).  A period only
 * counts once all its period_samples samples have been seen.  The state
 * carries across chunks through the planner handle; *completed returns the
 * number of whole periods folded so far. */
typedef struct msosm_fold_planner msosm_fold_planner;
MSOSM_API msosm_status msosm_fold_planner_create(float period, float fs, unsigned long discard_Nd,
                                       msosm_fold_planner **out);
MSOSM_API msosm_status msosm_fold_planner_destroy(msosm_fold_planner *p);
MSOSM_API msosm_status msosm_fold_planner_chunk(msosm_fold_planner *p, unsigned long size, int64_t *dest,
                                      unsigned long long *completed);

/* ======================================================================
 * PSRDADA baseband files (host I/O)
 * ====================================================================== */

/* A 4096-byte ASCII header of "KEY value" lines, then frames of 2048
 * uint16 pairs of polarisation 1 followed by 2048 of polarisation 2.
 * Replaces the PSRDADA class (psrdada/psrdada.cpp:3-94,
 * psrdada/include/psrdada.h:11-43).  Keys are read as the reference reads
 * them: a line splits at its first space, the value starts at the next
 * non-space character; fields whose key is absent stay 0 (the reference
 * leaves them uninitialised). */
typedef struct msosm_dada msosm_dada;
#define MSOSM_DADA_HAVE_BW 0x1u   /* BW was present */
#define MSOSM_DADA_HAVE_FREQ 0x2u /* FREQ was present */
typedef struct msosm_dada_info {
    float bw;   /* BW, MHz */
    float fc;   /* FREQ (centre), MHz */
    int nbit;
    int nchan;
    int ndim;
    int npol;
    unsigned int have;              /* MSOSM_DADA_HAVE_* */
    unsigned long long filesize;    /* bytes, header included */
} msosm_dada_info;

/* Open and parse the header (PSRDADA::PSRDADA, psrdada.cpp:3-50). */
MSOSM_API msosm_status msosm_dada_open(const char *path, msosm_dada **out);
MSOSM_API msosm_status msosm_dada_close(msosm_dada *d);
MSOSM_API msosm_status msosm_dada_get_info(const msosm_dada *d, msosm_dada_info *info);
/* The raw 4096 header bytes (PSRDADA::headerBuffer). */
MSOSM_API msosm_status msosm_dada_get_header(const msosm_dada *d, char *header4096);
/* Whole reads of n samples per polarisation the file holds:
 * (filesize - 4096) / (2 n 4) (PSRDADA::initBuffer's readCount,
 * psrdada.cpp:57-78).  n: a positive multiple of 2048. */
MSOSM_API msosm_status msosm_dada_read_count(const msosm_dada *d, unsigned long n, unsigned long *count);
/* The next n samples of each polarisation, de-interleaved frame by frame
 * into pol1 and pol2 (host buffers of n pairs each; PSRDADA::readSamples,
 * psrdada.cpp:80-87).  Returns MSOSM_ERR_STATE, reading nothing, when fewer
 * than 2n samples are left (the reference reads past the end silently). */
MSOSM_API msosm_status msosm_dada_read(msosm_dada *d, unsigned long n, msosm_uint16_pair *pol1,
                                       msosm_uint16_pair *pol2);

/* ======================================================================
 * Series files (the reference drivers' output writer threads)
 * ====================================================================== */

/* Appends every call's dedispersed series to a binary file while the device
 * keeps working: the output-file threads of the reference's drivers
 * (multiple_dm_concurrent_msosm.cpp:80-146), which write numDMs * count * M
 * uint16 pairs per call, [dm][count*M], without the trailing element.
 * msosm_writer_push (after a filter call, from the thread that drives the
 * handle) encodes the call's series into one of `depth` device slots on the
 * handle's stream -- the next call may start at once -- copies it to pinned
 * host memory on the writer's own stream and queues it for the writer
 * threads (1 .. depth); it blocks only while all slots are in flight.  No
 * busy-wait.  Each batch lands at its own offset (call index x batch bytes),
 * so several writer threads keep the file in call order.
 * kind: MSOSM_WRITE_UINT16 (the get_output_uint16 codec) or MSOSM_WRITE_C64.
 * msosm_writer_close waits for the queued writes, closes the file and
 * reports the bytes written (and the first error of the writer thread). */
typedef struct msosm_writer msosm_writer;
#define MSOSM_WRITE_UINT16 0
#define MSOSM_WRITE_C64 1
MSOSM_API msosm_status msosm_writer_create(msosm_dedisp *d, const char *path, int kind, int depth, int threads,
                                           msosm_writer **out);
MSOSM_API msosm_status msosm_writer_push(msosm_writer *w);
MSOSM_API msosm_status msosm_writer_close(msosm_writer *w, unsigned long long *bytes_written);

/* ======================================================================
 * Signal simulator (simulated_pulsar/) and host buffers
 * ====================================================================== */

/* Host memory for signals: pinned (cudaMallocHost, as the reference's
 * generate_pulsar_signal(pinned = true) allocates) or plain malloc. */
MSOSM_API msosm_status msosm_host_alloc(size_t bytes, int pinned, void **out);
MSOSM_API msosm_status msosm_host_free(void *p, int pinned);

/* Random numbers of every simulator: Philox4x32-10 (Salmon et al., SC11,
 * 2011) at counter (lo(i), hi(i), tag, 0) under the key (lo(seed), hi(seed))
 * for sample i; Box-Muller in double precision turns the block's four words
 * into two complex unit normals (variance 1 per component) rounded to float.
 * A sample's numbers depend only on (seed, i, tag).  Tags: 0 the pulsar
 * generator (z1: emission, z2: system noise), 1 AWGN. */
#define MSOSM_SIM_TAG_PULSAR 0u
#define MSOSM_SIM_TAG_AWGN 1u
/* z1[j], z2[j] of samples i = start + j, j < n (either may be NULL; host or
 * device pointers).  Needs a GPU. */
MSOSM_API msosm_status msosm_sim_normals(unsigned long long seed, unsigned long long start, unsigned long n,
                                         unsigned int tag, msosm_complex *z1, msosm_complex *z2);

/* AWGN::generateNoiseSamples (simulated_pulsar/AWGN.cpp:29-58) with the
 * tag-1 normals z of `seed`: snr_mode 1 (AWGN(SNR, n)) gives
 * sigma / sqrt(2) * z, sigma = sqrt(10^(-SNR/10)); snr_mode 0 (AWGN(mean,
 * variance, n)) gives z * variance + mean (the reference passes the variance
 * as the standard deviation).  The reference's default-seeded
 * std::default_random_engine sequence is not reproduced. */
MSOSM_API msosm_status msosm_sim_awgn(unsigned long long seed, unsigned long n, int snr_mode, float mean,
                                      float variance, float snr_db, msosm_complex *out);

/* SimulatedComplexSignal's sizes (simulated_complex_signal.cpp:21-25,
 * 52-71): Np = period samples, Nd = dispersion smear, range =
 * ceil(Nd / Np) periods (at least 1), order = 2^ceil(log2(range Np)). */
typedef struct msosm_sim_two_spike_info {
    unsigned long Np, Nd, range, order;
} msosm_sim_two_spike_info;
MSOSM_API msosm_status msosm_sim_two_spike_shape(float bw, float dm, float f0, float period,
                                                msosm_sim_two_spike_info *info);
/* SimulatedComplexSignal(bw, dm, f0, period).generate_pulsar_signal(repeat,
 * add_noise, SNR) (simulated_complex_signal.cpp:40-236) on the device: one
 * period of two unit deltas at Np/2 and Np/2 + 2 dispersed by the +phase
 * chirp filter of `order` points and summed over `range` periods, tiled
 * `repeat` times; with add_noise, AWGN at SNR dB relative to the period's
 * measured power (tag-1 normals of `seed`).  signal: repeat * Np complex;
 * signal_u16: the reference's codec ((v == 0) ? 0 : uint16(v * 32767 +
 * 32768), wrapping); signal_power_db: the measured power.  Outputs may be
 * NULL, host or device.  order 64 .. 2^24. */
MSOSM_API msosm_status msosm_sim_two_spike(float bw, float dm, float f0, float period, unsigned long repeat,
                                           int add_noise, float snr_db, unsigned long long seed,
                                           msosm_complex *signal, msosm_uint16_pair *signal_u16,
                                           float *signal_power_db);

/* Streaming noisy pulsar: x(t) = D[a z1](t) + z2(t) / sqrt(2), t = 0, 1, ...,
 * a(t) = sqrt(snr g(phase)) / sqrt(2), g a Gaussian profile of peak 1 and
 * FWHM `fwhm` (fraction of the period) centred at phase `centre`, phase =
 * frac(t / bw / period), z1 and z2 the tag-0 normals, D the overlap-save
 * dispersion filter (MSOSM_FLAG_OSM | MSOSM_FLAG_DISPERSE, order 2 *
 * nextpow2(Nd); none at Nd = 0).  The pulsar/noise power ratio peaks at snr.
 * The dispersion filter is causal: the emission at t arrives between
 * t + M - Nd (top of the band) and t + M (bottom), M its order. */
typedef struct msosm_sim_pulsar_params {
    float bw;       /* Hz (complex sampling rate) */
    float f0;       /* lower band edge, Hz */
    float dm;       /* pc cm^-3 */
    double period;  /* s */
    double fwhm;    /* pulse FWHM, fraction of the period */
    double centre;  /* pulse centre phase */
    double snr;     /* peak pulsar/noise power ratio per sample */
    unsigned long long seed;
} msosm_sim_pulsar_params;
typedef struct msosm_sim msosm_sim;
typedef struct msosm_sim_pulsar_info {
    unsigned long chunk;            /* samples per msosm_sim_pulsar_next */
    unsigned long M;                /* dispersion filter order (0: none) */
    unsigned long Nd;               /* dispersion smear, samples */
    unsigned long long next_sample; /* index of the next chunk's first sample */
} msosm_sim_pulsar_info;
/* chunk = min_chunk rounded up to a multiple of M (0: 2^22). */
MSOSM_API msosm_status msosm_sim_pulsar_create(const msosm_sim_pulsar_params *p, unsigned long min_chunk,
                                               msosm_sim **out);
MSOSM_API msosm_status msosm_sim_pulsar_destroy(msosm_sim *s);
MSOSM_API msosm_status msosm_sim_pulsar_get_info(const msosm_sim *s, msosm_sim_pulsar_info *info);
/* The next chunk samples: complex (out) and/or offset-binary uint16 pairs of
 * rint(x * u16_scale) + 32768 clipped to 1 .. 65535 (u16); host or device
 * pointers, either may be NULL. */
MSOSM_API msosm_status msosm_sim_pulsar_next(msosm_sim *s, msosm_complex *out, msosm_uint16_pair *u16,
                                             double u16_scale);

/* ======================================================================
 * DM-proposal network (no counterpart in the reference)
 * ====================================================================== */

/* A small 1-D CNN over the folded profiles of in_channels coarse DM trials
 * (length phase bins): `layers` circular convolutions of `channels` outputs
 * and odd `kernel`, each with ReLU, the mean over phase, and two linear
 * heads -- a detection logit and a DM offset.  Weights are kept in FP32 and
 * used rounded to bf16; products accumulate in FP32; every reduction has a
 * fixed order.  Loss: logistic loss of the logit plus dm_weight times the
 * mean over positive samples of the squared offset error.  Parameters, one
 * FP32 vector: per layer weights [C_out][C_in][kernel] then biases [C_out];
 * detection head weights [channels] and bias; offset head weights and bias.
 * in_channels and channels: multiples of 8; length: a multiple of 32. */
typedef struct msosm_cnn msosm_cnn;
typedef struct msosm_cnn_config {
    int in_channels;  /* coarse DM trials per sample */
    int length;       /* phase bins */
    int channels;     /* convolution outputs */
    int kernel;       /* odd kernel width */
    int layers;
    int max_batch;    /* <= 1024 */
    float dm_weight;  /* weight of the offset loss */
} msosm_cnn_config;
/* He-uniform weights from `seed`, zero biases.  Needs a GPU. */
MSOSM_API msosm_status msosm_cnn_create(const msosm_cnn_config *cfg, unsigned long long seed, msosm_cnn **out);
MSOSM_API msosm_status msosm_cnn_destroy(msosm_cnn *n);
MSOSM_API msosm_status msosm_cnn_param_count(const msosm_cnn *n, size_t *count);
MSOSM_API msosm_status msosm_cnn_get_params(msosm_cnn *n, float *params);
/* Also clears the optimiser's state. */
MSOSM_API msosm_status msosm_cnn_set_params(msosm_cnn *n, const float *params);
/* x: [batch][in_channels][length]; logit, offset: [batch]; host or device. */
MSOSM_API msosm_status msosm_cnn_forward(msosm_cnn *n, const float *x, int batch, float *logit, float *offset);
/* Loss and gradient of a batch (label 1 pulsar / 0 noise, target the offset
 * of positive samples); the gradient stays for msosm_cnn_adam_step and is
 * copied to `grad` (param_count floats) when it is not NULL. */
MSOSM_API msosm_status msosm_cnn_gradient(msosm_cnn *n, const float *x, const float *label, const float *target,
                                          int batch, float *loss, float *grad);
/* One Adam step (beta 0.9, 0.999, eps 1e-8) with the last gradient. */
MSOSM_API msosm_status msosm_cnn_adam_step(msosm_cnn *n, float lr);

/* ======================================================================
 * Diagnostics (no counterpart in the reference)
 * ====================================================================== */

/* Limit of each wait of the tensor-core kernel (MSOSM_FLAG_TENSOR_*) on one
 * of its GEMMs, in ns of the global timer; ns < 0 restores the default (1 s),
 * 0 makes every such wait give up at once.  When a wait
 * gives up, the kernel records a nonzero status, waits (1 s at most) for the
 * GEMMs it still has in flight, frees its tensor memory and returns; the
 * next synchronising call (get_output_*, get_profiles, synchronize) returns
 * MSOSM_ERR_TIMEOUT and clears the status, and the handle carries on (the
 * outputs of the calls since the previous check are invalid).  For tests of
 * that path; returns MSOSM_ERR_STATE for a handle without the tensor-core
 * kernel. */
MSOSM_API msosm_status msosm_dedisp_set_tc_wait_limit(msosm_dedisp *d, long long ns);

/* Runs one of the tensor-core GEMMs of MSOSM_FLAG_TENSOR_F16 on given data,
 * with the kernel's own shared-memory layouts, constant operand and
 * tensor-memory read-back: d = a * B_step, a a 128 x K matrix of f16 bit
 * patterns (row-major, host memory), B_step the real form of an inverse DFT
 * with rows [Re | Im] of the input index and columns [Re | Im] of the output
 * frequency.  Step 1: the 64-point DFT of FFT 4096 (K 128, 128 columns);
 * step 2: the 64-point DFT restricted to frequencies 32..63 (K 128, 64
 * columns); step 3: the 128-point DFT of FFT 8192 and 16384 (K 256, 256
 * columns); step 4: the 128-point DFT restricted to frequencies 64..127, the
 * second GEMM of FFT 16384 (K 256, 128 columns).
 * d: host, 128 x columns floats, row-major.  Needs a GPU. */
MSOSM_API msosm_status msosm_tc_gemm_check(int step, const uint16_t *a, float *d);

#ifdef __cplusplus
}
#endif
#endif /* MSOSM_B200_H */
