// kernels.hpp -- host-side launchers of the sm_100a kernels (kernels.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "host_prepare.hpp"
#include "msosm_b200.h"

namespace msosm {

constexpr int kMinLog2N = 6;   // FFT 64 (M = 32) .. 16384 in one thread block
constexpr int kMaxLog2N = 14;

enum InputKind : int { kInputC64 = 0, kInputU16 = 1 };

struct FwdArgs {
    const void *input;      // count*M samples of this call (device)
    const float2 *hist_in;  // previous call's last M samples
    float2 *hist_out;       // this call's last M samples (for the next call)
    float2 *ring;           // [S][N] spectra
    int S;                  // ring depth, a power of two
    long long k0;           // global index of this call's first block
    int count;
    const float2 *tw;       // exp(-2 pi i e/N)
    int tc_order;           // 1: rows in tensor-core order (4096..16384 points)
    float *row_max;         // tc_order: [S] largest |component| of each ring row
};

struct FoldArgs {
    const long long *span_a, *span_b;  // chunk-local [a, b), sorted
    const int *span_phase0, *span_dest; // dest 0 skip / 1 main / 2 pending
    int nspans;
    int bpt;      // samples per output bin
    int nbins;    // output bins
    int detect;   // 0 |y|^2, 1 |y|
    float *part_main, *part_pend;  // [items][nbins]
    int smem_prof;  // 1: the work item's profile rows live in shared memory
    int span_cap;   // spans held in the shared-memory window (>= spans one block can touch)
    float inv_bpt;  // 1/bpt, for the exact-corrected division
    int g_shift;    // log2 of the lanes summing one bin (fold_g_shift)
};

// Lanes per bin in the fold: G ~ bpt/8, a power of two <= 32 (1 below whole warps).
inline int fold_g_shift(int bpt, int threads)
{
    if (threads < 32)
        return 0;
    int g = 0;
    while (g < 5 && (8 << g) < bpt)
        ++g;
    return g;
}

// intensity staging of one block: M samples, one pad slot per 32
__host__ __device__ constexpr int ibuf_floats(int m) { return (m + (m >> 5) + 1) & ~1; }

// Extra dynamic shared memory of the folding dedispersion kernel (threads: its block size).
size_t fold_smem_bytes(int nbins, int span_cap, bool smem_prof, int threads);
constexpr int kMaxSmemBins = 4096;

struct DedispArgs {
    const float2 *ring;
    int S;                    // ring depth, a power of two
    int max_delay;            // largest block delay of any trial
    long long k0;
    int count;
    int D;
    int R;                    // block ranges per trial (work item = (range, trial))
    const float2 *H;          // [D][N], scaled by 1/N^2
    const uint16_t *delays;   // [D][N]
    const float2 *tw;         // exp(+2 pi i e/N)
    float2 *series;           // [D][count*M] or nullptr
    FoldArgs fold;            // fold.nspans < 0: no folding
    // tensor-core kernel only
    int *status;              // nonzero after a timed-out wait
    long long wait_limit_ns;  // limit of each wait on a GEMM (0: give up at the first incomplete probe)
    const float *row_max;     // [S] largest |component| of each ring row
    const float *h_max;       // [D] largest |component| of each trial's H
    const int *delay_max;     // [D] largest block delay of each trial
};

// One launch over the work items of up to kBatchMax handles (observations)
// that run the same kernel variant: handle o's items are [prefix[o],
// prefix[o + 1]), each with args[o]; a CTA takes the next item from *counter
// (zero before the launch), so items of uneven size balance over the grid.
// The table is the kernel's parameter (about 25 KB), so that the kernel reads
// an item's arguments from the constant bank, as the one-handle kernel reads
// its own, not from registers.
constexpr int kBatchMax = 128;
struct BatchArgs {
    int nobs;
    int *counter;
    int prefix[kBatchMax + 1];
    DedispArgs args[kBatchMax];
};
// the one-handle kernel's unused second parameter
struct NoBatch {
    int unused;
};

struct DesignArgs {
    const ChirpParams *chirp;  // [D] device
    int D;
    const float2 *tw_inv_m;    // exp(+2 pi i e/M)
    const float2 *tw_fwd_n;    // exp(-2 pi i e/N)
    float2 *H;                 // [D][N]
    float scale;
    int sign;                  // -1 dedispersion (cos - i sin), +1 dispersion
};

bool log2n_supported(int log2n);

// Sets the message msosm_last_error() returns on this thread.
void set_error_message(const char *msg);

cudaError_t launch_forward(int log2n, InputKind kind, const FwdArgs &a, cudaStream_t st);
// pp: ping-pong shared-memory buffers (one barrier per FFT stage instead of
// two; twice the buffer space); honoured for FFT sizes up to 4096
cudaError_t launch_dedisp(int log2n, bool pp, bool series, bool fold, const DedispArgs &a, int grid,
                          cudaStream_t st);
// CTAs of the dedispersion kernel that fit on one SM (for the persistent grid)
int dedisp_blocks_per_sm(int log2n, bool pp, bool series, bool fold, size_t extra_smem);
cudaError_t launch_design(int log2n, const DesignArgs &a, cudaStream_t st);

cudaError_t launch_fold_reduce(const float *part_main, const float *part_pend, int D, int R, int nbins,
                               double *acc_main, double *acc_pend, cudaStream_t st);
cudaError_t launch_fold_flush(double *acc_main, double *acc_pend, size_t n, cudaStream_t st);
// The n fold spans of a call from their pinned host staging (a, b: long long
// [cap] each, then phase0, dest: int [cap] each), read by a kernel over the
// bus, into the device span arrays
cudaError_t launch_span_upload(const long long *host, int n, int cap, long long *a, long long *b, int *phase0,
                               int *dest, cudaStream_t st);
cudaError_t launch_fold_readout(const double *acc_main, size_t n, double scale, float *out,
                                cudaStream_t st);
cudaError_t launch_encode_u16(const float2 *src, uint32_t *dst, size_t n, cudaStream_t st);
// sqrt(|a|^2 + |b|^2) (b may be null)
cudaError_t launch_intensity(const float2 *a, const float2 *b, float *out, size_t n, cudaStream_t st);
// fold n intensities into R partial rows (fold.part_main/part_pend [R][nbins])
int fold_series_block();
cudaError_t launch_fold_series(const float *I, long long n, int R, const FoldArgs &f, int grid, int trials,
                               cudaStream_t st);

// ---- tensor-core (tcgen05) dedispersion, 4096-, 8192- and 16384-point transforms (tc_dedisp.cu)
bool tc_supported(int log2n);
// threads per CTA of the tensor-core kernel (its fold group size)
int tc_threads(int log2n);
// blocks one step of the kernel transforms: 2 (a pair) at 4096 and 8192, 1 at 16384
int tc_blocks_per_step(int log2n);
// shared memory of the tensor-core kernel before its fold state (tables,
// operand buffers, control), and the device's per-block limit (0 when it
// cannot be read)
size_t tc_smem_base(int log2n);
size_t tc_smem_limit();
int tc_blocks_per_sm(int log2n, bool bf16, bool series, bool fold, size_t extra_smem);
// a.H and a.delays in tensor-core order (tc_layout.hpp), ring written with
// FwdArgs::tc_order; a.R counts ranges of steps (tc_blocks_per_step blocks
// each); bf16: bf16 operands
// (else f16)
cudaError_t launch_tc_dedisp(int log2n, bool bf16, bool series, bool fold, const DedispArgs &a, int grid,
                             cudaStream_t st);
// the same over the items of several handles in one launch (a batch);
// fold_smem: the largest fold shared-memory size over the handles
cudaError_t launch_tc_dedisp_batch(int log2n, bool bf16, bool series, bool fold, const BatchArgs &b,
                                   size_t fold_smem, int grid, cudaStream_t st);
// rows of 2^log2n bins from natural into tensor-core order (out of place)
cudaError_t launch_tc_permute_rows(const float2 *in, float2 *out, int rows, int log2n, cudaStream_t st);
// one GEMM of the kernel on given data: a = 128 x K f16 bit patterns
// (row-major), d = 128 x columns f32 (row-major); steps 1, 2: the
// 4096-point GEMMs (K 128; 128 and 64 columns), 3: the 8192-point GEMM 1
// (K 256, 256 columns)
cudaError_t launch_tc_probe(int step, const uint16_t *a, float *d, int *status, cudaStream_t st);

// ---- FFT sizes above one thread block (largefft.cu) -----------------------
struct LargeColArgs {
    const void *input;        // forward: the call's input (or a vector, kind 2)
    const float2 *in;         // inverse: B[d][w][k1][n2]
    const float2 *hist_in;    // forward windows: previous call's last M samples
    float2 *hist_out;
    float2 *out;              // forward: A[w][k1][n2]
    long long N, N2, len;     // transform size, row length, vector length (kind 2)
    int log2n, count;
    const float2 *tw1;        // exp(sign 2 pi i e / N1) for the pass's sign
    float2 *series;           // inverse: [d][count*M] or null
    float *intensity;         // inverse: [d][count*M] or null
    int detect;
};
struct LargeRowArgs {
    const float2 *in;         // forward: A
    float2 *out;              // inverse: B; design: permuted spectrum
    float2 *ring;
    int S;
    long long k0;
    int count;
    const float2 *H;          // [d][N] permuted, x 1/N^2
    const uint16_t *delays;   // [d][N] permuted
    long long N;
    int log2n;
    const float2 *tw2;        // exp(sign 2 pi i e / N2)
};
void large_split(int log2n, int &log2n1, int &log2n2);
bool large_supported(int log2n);
cudaError_t launch_large_col_fwd(int log2n1, int kind, const LargeColArgs &a, int windows, cudaStream_t st);
cudaError_t launch_large_col_inv(int log2n1, const LargeColArgs &a, int blocks, int trials, cudaStream_t st);
// mode 0: forward row -> ring; 1: gather x H, inverse row -> B; 2: forward row -> out
cudaError_t launch_large_row(int log2n2, int mode, const LargeRowArgs &a, int rows, int windows, int trials,
                             cudaStream_t st);
cudaError_t launch_vec_fft(int log2n, int sign, const float2 *in, float2 *out, const float2 *tw, int count,
                           cudaStream_t st);
cudaError_t launch_chirp_conj(const ChirpParams *cp, float2 *out, long long M, int sign, cudaStream_t st);
cudaError_t launch_unpermute_conj(const float2 *in, float2 *out, long long K, long long K1, long long K2,
                                  long long len_out, cudaStream_t st);
cudaError_t launch_conj_scale(float2 *x, long long n, float scale, int conj, cudaStream_t st);

// Unnormalised inverse M-point DFT (M = 2^log2m, 64 .. 2^24) of the
// reference chirp, sign -1 the dedispersion chirp (msosm_prepare.cpp:40-70)
// and +1 the dispersion chirp of the signal simulator
// (simulated_complex_signal.cpp:91-107), written to P[0, M) with zeros in
// P[M, len_out).  init() allocates the scratch and twiddle tables (status
// codes of msosm_b200.h); run() is ordered on its stream.
// The stream a dedispersion handle's work is ordered on (its own, or the one
// set with msosm_dedisp_set_stream).
cudaStream_t dedisp_stream(const msosm_dedisp *d);

struct ChirpIdft {
    int log2m = 0, m1l = 0, m2l = 0;
    bool large = false;
    ChirpParams *cp_d = nullptr;
    float2 *V = nullptr, *W = nullptr, *A = nullptr, *tw1 = nullptr, *tw2 = nullptr;
    int init(int log2m, cudaStream_t st);
    cudaError_t run(const ChirpParams &cp, int sign, float2 *P, long long len_out, cudaStream_t st);
    void release();
};

}  // namespace msosm
