// kernels.cu -- sm_100a kernels of the MS-OSM / OSM dedispersion path.
//
//   forward_kernel  decode (uint16 offset-binary or complex64) + forward FFT of
//                   the overlapping windows of one call, written into the
//                   spectrum ring shared by all DM trials.  Replaces
//                   uint16ToComplex + the forward cufftExecC2C
//                   (gpu/gpu_kernel.cu:276-299, msosm_gpu_dm_concurrent.cpp:123-129).
//   dedisp_kernel   persistent; per (DM trial, block): gather each bin's
//                   delayed spectrum from the ring, multiply by H, inverse FFT
//                   in shared memory, keep the second half (overlap-save
//                   discard), then write the series and/or detect and fold.
//                   Replaces ComplexMultiplyDelay_concurrent_batch + inverse
//                   cufftExecC2C + DiscardSamples_concurrent_batch
//                   (gpu/gpu_kernel.cu:128-198,236-258) and, fused, the
//                   calculateIntensity kernel + host fold of Fold_GPU
//                   (gpu/gpu_kernel.cu:347-353, folding/fold_gpu.cpp:48-194).
//   design_kernel   dedispersion filter H per trial on the device: FP64 chirp
//                   phase reduced mod 2 pi, M-point inverse FFT, zero pad,
//                   2M-point FFT (msosm_prepare.cpp:37-84 on the host in the
//                   reference).
//
// Ring semantics: the reference scatters X[c][b]*H[b]/N into a per-DM product
// ring at slot (index + c + delay[b]) % S and inverse-transforms slots
// index..index+count-1 (gpu/gpu_kernel.cu:179-184).  A slot therefore holds,
// for bin b, the product of block k - delay[b] (zero before the stream
// start).  Here the ring holds the input spectra once for all trials and
// each trial gathers X[k - delay[b]][b] * H[b] directly.
#include "chirp.cuh"
#include "fft_smem.cuh"
#include "fold_dev.cuh"
#include "kernels.hpp"
#include "tc_layout.hpp"

#include <cuda_runtime.h>

namespace msosm {

// ---------------------------------------------------------------------------
// forward transform of the input windows
// ---------------------------------------------------------------------------

template <int KIND>
__device__ __forceinline__ float2 load_sample(const void *p, long long s)
{
    if constexpr (KIND == kInputC64) {
        return reinterpret_cast<const float2 *>(p)[s];
    } else {
        // offset binary, 0 = blank (gpu/gpu_kernel.cu:291-296)
        const uint32_t u = reinterpret_cast<const uint32_t *>(p)[s];
        const uint32_t x = u & 0xFFFFu, y = u >> 16;
        return make_float2(x ? (float)x - 32768.0f : 0.0f, y ? (float)y - 32768.0f : 0.0f);
    }
}

template <int LOG2N, int KIND, bool PP>
__global__ void __launch_bounds__(FftShape<LOG2N>::T) forward_kernel(FwdArgs a)
{
    using F = FftShape<LOG2N>;
    constexpr int N = F::N, M = N / 2, T = F::T;
    extern __shared__ float2 smem[];
    float2 *buf0 = smem;
    float2 *buf1 = PP ? smem + F::SMEM : smem;
    const int tid = threadIdx.x;
    const int c = blockIdx.x;
    float2 v[16];
    // window c covers input samples [c*M - M, c*M + M); negative indices are
    // the previous call's last M samples (the reference's D2D overlap copy,
    // msosm_gpu_dm_concurrent.cpp:125)
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int n = tid + r * T;
        const long long s = (long long)c * M + n - M;
        const float2 x = (s < 0) ? a.hist_in[M + s] : load_sample<KIND>(a.input, s);
        if (c == a.count - 1 && n >= M)
            a.hist_out[n - M] = x;
        v[r] = x;
    }
    dft16<-1>(v);
    stage_store<LOG2N, 0>(v, buf0, tid);
    run_stages<LOG2N, -1, PP>(v, buf0, buf1, tid, a.tw);
    const int slot_row = (int)((a.k0 + c) & (a.S - 1));
    float2 *row = a.ring + (size_t)slot_row * N;
    if ((LOG2N >= 12 && LOG2N <= 14) && a.tc_order) {
        float mx = 0.f;
#pragma unroll
        for (int slot = 0; slot < 16; ++slot) {
            row[tc::tc_pos(last_out_index<LOG2N>(tid, slot), LOG2N)] = v[slot];
            mx = fmaxf(mx, fmaxf(fabsf(v[slot].x), fabsf(v[slot].y)));
        }
        // the row's largest component (the tensor-core kernel scales by it)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        __syncthreads();  // every thread is done with the FFT buffers
        float *wm = reinterpret_cast<float *>(buf0);
        if ((tid & 31) == 0)
            wm[tid >> 5] = mx;
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < T / 32; ++w)
                mx = fmaxf(mx, wm[w]);
            a.row_max[slot_row] = mx;
        }
    } else {
#pragma unroll
        for (int slot = 0; slot < 16; ++slot)
            row[last_out_index<LOG2N>(tid, slot)] = v[slot];
    }
}

// ---------------------------------------------------------------------------
// fused dedispersion + detection + folding
// ---------------------------------------------------------------------------

template <int LOG2N, bool PP, bool SERIES, bool FOLD>
__global__ void __launch_bounds__(FftShape<LOG2N>::T) dedisp_kernel(DedispArgs a)
{
    using F = FftShape<LOG2N>;
    constexpr int N = F::N, M = N / 2, T = F::T;
    constexpr int RL = F::radix(F::NST - 1);
    extern __shared__ float2 smem[];
    float2 *buf0 = smem;
    float2 *buf1 = PP ? smem + F::SMEM : smem;
    float *ibuf = reinterpret_cast<float *>(smem + (PP ? 2 : 1) * F::SMEM);
    FoldSmem fw;
    if constexpr (FOLD) {
        // after ibuf: [span window a, b, phase0, dest] [partials] [prof_main, prof_pend]
        fold_smem_layout(fw, ibuf + ibuf_floats(M), a.fold);
    }
    const int tid = threadIdx.x;
    const int items = a.D * a.R;
    for (int w = blockIdx.x; w < items; w += gridDim.x) {
        const int dm = w % a.D;
        const int rr = w / a.D;
        const int kb = (int)((long long)a.count * rr / a.R);
        const int ke = (int)((long long)a.count * (rr + 1) / a.R);
        const float2 *__restrict__ Hd = a.H + (size_t)dm * N;
        const uint16_t *__restrict__ dl = a.delays + (size_t)dm * N;
        int sp = 0, sbase = 0, scnt = 0;
        if constexpr (FOLD) {
            if (a.fold.smem_prof) {
                for (int i = tid; i < 2 * a.fold.nbins; i += blockDim.x)
                    fw.prof_main[i] = 0.f;
            } else {
                fw.prof_main = a.fold.part_main + (size_t)w * a.fold.nbins;
                fw.prof_pend = a.fold.part_pend + (size_t)w * a.fold.nbins;
            }
            sp = span_lower_bound(a.fold.span_b, a.fold.nspans, (long long)kb * M);
            span_refill(a.fold, fw, sp, sbase, scnt);
        }
        long long kg = a.k0 + kb;
        const int smask = a.S - 1;  // the ring depth is a power of two
        for (int k = kb; k < ke; ++k, ++kg) {
            float2 v[16];
            const int slot_k = (int)(kg & smask);
            if (kg >= a.max_delay) {
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int b = tid + r * T;
                    const int s = (slot_k - (int)__ldg(&dl[b])) & smask;
                    v[r] = cmul(a.ring[(size_t)s * N + b], __ldg(&Hd[b]));
                }
            } else {
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    const int b = tid + r * T;
                    const int d = (int)__ldg(&dl[b]);
                    float2 x = make_float2(0.f, 0.f);
                    if (kg >= d)  // blocks before the stream start are zero
                        x = a.ring[(size_t)((slot_k - d) & smask) * N + b];
                    v[r] = cmul(x, __ldg(&Hd[b]));
                }
            }
            dft16<+1>(v);
            // the previous block's last-stage loads (and fold reads of ibuf)
            // must be done before buf0 is overwritten; with folding the
            // barrier ahead of the fold already separates them
            if constexpr (!FOLD)
                __syncthreads();
            stage_store<LOG2N, 0>(v, buf0, tid);
            run_stages<LOG2N, +1, PP>(v, buf0, buf1, tid, a.tw);
            // keep outputs n >= M (the last-stage slots with r >= R/2)
#pragma unroll
            for (int slot = 0; slot < 16; ++slot) {
                if ((slot % RL) >= RL / 2) {
                    const int t = last_out_index<LOG2N>(tid, slot) - M;
                    const float2 y = v[slot];
                    if constexpr (SERIES)
                        a.series[(size_t)dm * a.count * M + (size_t)k * M + t] = y;
                    if constexpr (FOLD) {
                        const float p = y.x * y.x + y.y * y.y;
                        ibuf[ipad(t)] = a.fold.detect ? sqrtf(p) : p;
                    }
                }
            }
            if constexpr (FOLD) {
                __syncthreads();
                fold_block<kIbufPadded>(a.fold, fw, ibuf, k * M, M, sp, sbase, scnt);
            }
        }
        if constexpr (FOLD) {
            __syncthreads();
            if (a.fold.smem_prof) {
                float *gm = a.fold.part_main + (size_t)w * a.fold.nbins;
                float *gp = a.fold.part_pend + (size_t)w * a.fold.nbins;
                for (int i = tid; i < a.fold.nbins; i += blockDim.x) {
                    gm[i] = fw.prof_main[i];
                    gp[i] = fw.prof_pend[i];
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// folding of a materialised intensity series (Fold_GPU)
// ---------------------------------------------------------------------------

// sqrt(|a|^2 + |b|^2) per sample (b may be null): gpu/gpu_kernel.cu:347-353.
__global__ void intensity_kernel(const float2 *__restrict__ a, const float2 *__restrict__ b, float *__restrict__ out,
                                 size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float2 x = a[i];
        float p = x.x * x.x + x.y * x.y;
        if (b) {
            const float2 y = b[i];
            p += y.x * y.x + y.y * y.y;
        }
        out[i] = sqrtf(p);
    }
}

// Fold n intensities (one chunk of the stream) into per-work-item partial
// rows with the same span machinery as the fused kernel: work item w covers
// blocks [n_blocks*w/R, n_blocks*(w+1)/R) of kFoldBlock samples.
constexpr int kFoldBlock = 2048;

__global__ void __launch_bounds__(256) fold_series_kernel(const float *__restrict__ I, long long n, int R, FoldArgs f)
{
    // trial blockIdx.y folds I[d*n ...] into partial rows w*gridDim.y + d
    const int d = blockIdx.y, D = gridDim.y;
    I += (size_t)d * n;
    extern __shared__ float2 smem[];
    float *ibuf = reinterpret_cast<float *>(smem);
    FoldSmem fw;
    fold_smem_layout(fw, ibuf + ibuf_floats(kFoldBlock), f);
    const long long nblk = (n + kFoldBlock - 1) / kFoldBlock;
    for (int w = blockIdx.x; w < R; w += gridDim.x) {
        const long long kb = nblk * w / R, ke = nblk * (w + 1) / R;
        if (f.smem_prof) {
            for (int i = threadIdx.x; i < 2 * f.nbins; i += blockDim.x)
                fw.prof_main[i] = 0.f;
        } else {
            fw.prof_main = f.part_main + ((size_t)w * D + d) * f.nbins;
            fw.prof_pend = f.part_pend + ((size_t)w * D + d) * f.nbins;
        }
        int sp = span_lower_bound(f.span_b, f.nspans, kb * kFoldBlock), sbase = 0, scnt = 0;
        span_refill(f, fw, sp, sbase, scnt);
        for (long long k = kb; k < ke; ++k) {
            const int t0 = (int)(k * kFoldBlock);
            for (int t = threadIdx.x; t < kFoldBlock; t += blockDim.x)
                ibuf[ipad(t)] = (long long)t0 + t < n ? I[t0 + t] : 0.f;
            __syncthreads();
            fold_block<kIbufPadded>(f, fw, ibuf, t0, kFoldBlock, sp, sbase, scnt);
            __syncthreads();
        }
        if (f.smem_prof) {
            float *gm = f.part_main + ((size_t)w * D + d) * f.nbins;
            float *gp = f.part_pend + ((size_t)w * D + d) * f.nbins;
            for (int i = threadIdx.x; i < f.nbins; i += blockDim.x) {
                gm[i] = fw.prof_main[i];
                gp[i] = fw.prof_pend[i];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// filter design on the device
// ---------------------------------------------------------------------------

template <int LOG2N, bool PP>
__global__ void __launch_bounds__(FftShape<LOG2N>::T) design_kernel(DesignArgs a)
{
    using F = FftShape<LOG2N>;
    using FM = FftShape<LOG2N - 1>;
    constexpr int N = F::N, M = N / 2, T = F::T, TM = FM::T;
    extern __shared__ float2 smem[];
    float2 *buf0 = smem;
    float2 *buf1 = PP ? smem + F::SMEM : smem;
    const int tid = threadIdx.x;
    const int dm = blockIdx.x;
    const ChirpParams cp = a.chirp[dm];
    const bool act = tid < TM;
    float2 v[16];
    if (act) {
        // h index j holds offset index (j + M/2) mod M (msosm_prepare.cpp:50-63)
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int j = tid + r * TM;
            const unsigned int i = (unsigned int)((j + M / 2) & (M - 1));
            float c, s;
            chirp_cis(chirp_phase(cp, i), c, s);
            v[r] = make_float2(c, a.sign < 0 ? -s : s);
        }
        dft16<+1>(v);
        stage_store<LOG2N - 1, 0>(v, buf0, tid);
    }
    run_stages<LOG2N - 1, +1, PP>(v, buf0, buf1, tid, a.tw_inv_m, act);
    __syncthreads();
    if (act) {
#pragma unroll
        for (int slot = 0; slot < 16; ++slot)
            buf1[smem_pad(last_out_index<LOG2N - 1>(tid, slot))] = v[slot];
    }
    __syncthreads();
    // zero-padded 2M-point forward transform of the M-point result
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const int n = tid + r * T;
        v[r] = n < M ? buf1[smem_pad(n)] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    dft16<-1>(v);
    stage_store<LOG2N, 0>(v, buf0, tid);
    run_stages<LOG2N, -1, PP>(v, buf0, buf1, tid, a.tw_fwd_n);
    float2 *out = a.H + (size_t)dm * N;
#pragma unroll
    for (int slot = 0; slot < 16; ++slot) {
        const float2 y = v[slot];
        out[last_out_index<LOG2N>(tid, slot)] = make_float2(y.x * a.scale, y.y * a.scale);
    }
}

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------

// Sum of the R partial rows of every (trial, bin), in double and in a fixed
// order: G groups of rows (group g: rows g, g + G, ...) are summed by G
// threads, then thread g = 0 adds the G group sums in group order.  A thread
// block covers 32 consecutive (trial, bin) indices x G groups; row r of index
// i sits at r * D * nbins + i, so a warp reads 128 contiguous bytes of a row.
template <int G>
__global__ void __launch_bounds__(32 * G) fold_reduce_kernel(const float *__restrict__ pm,
                                                             const float *__restrict__ pp, int D, int R, int nbins,
                                                             double *am, double *ap)
{
    __shared__ double part[2][G][32];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const long long n = (long long)D * nbins;
    const long long i = (long long)blockIdx.x * 32 + lane;
    double sm = 0.0, sp = 0.0;
    if (i < n) {
        for (int r = g; r < R; r += G) {
            const size_t row = (size_t)r * (size_t)n + (size_t)i;
            sm += (double)pm[row];
            sp += (double)pp[row];
        }
    }
    part[0][g][lane] = sm;
    part[1][g][lane] = sp;
    __syncthreads();
    if (g == 0 && i < n) {
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int k = 0; k < G; ++k) {
            a += part[0][k][lane];
            b += part[1][k][lane];
        }
        am[i] += a;
        ap[i] += b;
    }
}

__global__ void fold_flush_kernel(double *am, double *ap, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        am[i] += ap[i];
        ap[i] = 0.0;
    }
}

__global__ void fold_readout_kernel(const double *am, size_t n, double scale, float *out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = (float)(am[i] * scale);
}

// complexToUint16 (gpu/gpu_kernel.cu:317-329): uint16(v + 32768*(v != 0)),
// truncating; out-of-range values saturate (undefined in the reference).
__device__ __forceinline__ uint32_t encode_u16(float v)
{
    float u = v + (v != 0.0f ? 32768.0f : 0.0f);
    u = fminf(fmaxf(u, 0.0f), 65535.0f);
    return (uint32_t)u;
}

__global__ void encode_u16_kernel(const float2 *__restrict__ src, uint32_t *__restrict__ dst, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float2 v = src[i];
        dst[i] = encode_u16(v.x) | (encode_u16(v.y) << 16);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

bool log2n_supported(int log2n) { return log2n >= kMinLog2N && log2n <= kMaxLog2N; }

template <int LOG2N>
constexpr bool use_pingpong() { return LOG2N <= 12; }

template <int LOG2N>
size_t dedisp_smem_bytes(bool pp)
{
    using F = FftShape<LOG2N>;
    return (pp ? 2 : 1) * F::SMEM * sizeof(float2) + ibuf_floats(F::N / 2) * sizeof(float);
}

template <int LOG2N>
size_t fft_smem_bytes()
{
    using F = FftShape<LOG2N>;
    return (use_pingpong<LOG2N>() ? 2 : 1) * F::SMEM * sizeof(float2);
}

template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes)
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int LOG2N>
static cudaError_t forward_t(InputKind kind, const FwdArgs &a, cudaStream_t st)
{
    constexpr bool PP = use_pingpong<LOG2N>();
    const size_t sm = fft_smem_bytes<LOG2N>();
    cudaError_t e;
    if (kind == kInputU16) {
        auto k = forward_kernel<LOG2N, kInputU16, PP>;
        if ((e = set_smem(k, sm)) != cudaSuccess)
            return e;
        k<<<a.count, FftShape<LOG2N>::T, sm, st>>>(a);
    } else {
        auto k = forward_kernel<LOG2N, kInputC64, PP>;
        if ((e = set_smem(k, sm)) != cudaSuccess)
            return e;
        k<<<a.count, FftShape<LOG2N>::T, sm, st>>>(a);
    }
    return cudaGetLastError();
}

size_t fold_smem_bytes(int nbins, int span_cap, bool smem_prof, int threads)
{
    return (size_t)span_cap * 4 * sizeof(int) + 2 * (size_t)threads * sizeof(float) +
           (smem_prof ? 2 * (size_t)nbins * sizeof(float) : 0);
}

template <int LOG2N, bool PP, bool SERIES, bool FOLD>
static auto dedisp_fn() { return dedisp_kernel<LOG2N, PP && use_pingpong<LOG2N>(), SERIES, FOLD>; }

// Calls go(kernel) with the instantiation for (pp, series, fold).
template <int LOG2N, typename G>
static auto dedisp_select(bool pp, bool series, bool fold, G &&go)
{
    if (pp && use_pingpong<LOG2N>()) {
        if (series && fold)
            return go(dedisp_fn<LOG2N, true, true, true>());
        if (fold)
            return go(dedisp_fn<LOG2N, true, false, true>());
        return go(dedisp_fn<LOG2N, true, true, false>());
    }
    if (series && fold)
        return go(dedisp_fn<LOG2N, false, true, true>());
    if (fold)
        return go(dedisp_fn<LOG2N, false, false, true>());
    return go(dedisp_fn<LOG2N, false, true, false>());
}

template <int LOG2N>
static cudaError_t dedisp_t(bool pp, bool series, bool fold, const DedispArgs &a, int grid, cudaStream_t st)
{
    pp = pp && use_pingpong<LOG2N>();
    const size_t sm = dedisp_smem_bytes<LOG2N>(pp) +
                      (fold ? fold_smem_bytes(a.fold.nbins, a.fold.span_cap, a.fold.smem_prof != 0,
                                              FftShape<LOG2N>::T) : 0);
    return dedisp_select<LOG2N>(pp, series, fold, [&](auto k) -> cudaError_t {
        cudaError_t e = set_smem(k, sm);
        if (e != cudaSuccess)
            return e;
        k<<<grid, FftShape<LOG2N>::T, sm, st>>>(a);
        return cudaGetLastError();
    });
}

template <int LOG2N>
static int dedisp_occ_t(bool pp, bool series, bool fold, size_t extra)
{
    pp = pp && use_pingpong<LOG2N>();
    const size_t sm = dedisp_smem_bytes<LOG2N>(pp) + extra;
    return dedisp_select<LOG2N>(pp, series, fold, [&](auto k) -> int {
        int n = 0;
        if (set_smem(k, sm) != cudaSuccess)
            return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, FftShape<LOG2N>::T, sm) != cudaSuccess)
            return 0;
        return n;
    });
}

template <int LOG2N>
static cudaError_t design_t(const DesignArgs &a, cudaStream_t st)
{
    constexpr bool PP = use_pingpong<LOG2N>();
    const size_t sm = fft_smem_bytes<LOG2N>();
    auto k = design_kernel<LOG2N, PP>;
    cudaError_t e = set_smem(k, sm);
    if (e != cudaSuccess)
        return e;
    k<<<a.D, FftShape<LOG2N>::T, sm, st>>>(a);
    return cudaGetLastError();
}

#define MSOSM_DISPATCH(log2n, CALL)                                                                   \
    switch (log2n) {                                                                                  \
    case 6: return CALL(6);                                                                           \
    case 7: return CALL(7);                                                                           \
    case 8: return CALL(8);                                                                           \
    case 9: return CALL(9);                                                                           \
    case 10: return CALL(10);                                                                         \
    case 11: return CALL(11);                                                                         \
    case 12: return CALL(12);                                                                         \
    case 13: return CALL(13);                                                                         \
    case 14: return CALL(14);                                                                         \
    default: break;                                                                                   \
    }

cudaError_t launch_forward(int log2n, InputKind kind, const FwdArgs &a, cudaStream_t st)
{
#define CALL(L) forward_t<L>(kind, a, st)
    MSOSM_DISPATCH(log2n, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_dedisp(int log2n, bool pp, bool series, bool fold, const DedispArgs &a, int grid,
                          cudaStream_t st)
{
#define CALL(L) dedisp_t<L>(pp, series, fold, a, grid, st)
    MSOSM_DISPATCH(log2n, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

int dedisp_blocks_per_sm(int log2n, bool pp, bool series, bool fold, size_t extra_smem)
{
#define CALL(L) dedisp_occ_t<L>(pp, series, fold, extra_smem)
    MSOSM_DISPATCH(log2n, CALL)
#undef CALL
    return 0;
}

cudaError_t launch_design(int log2n, const DesignArgs &a, cudaStream_t st)
{
#define CALL(L) design_t<L>(a, st)
    MSOSM_DISPATCH(log2n, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

static unsigned int blocks_for(size_t n, unsigned int t) { return (unsigned int)((n + t - 1) / t); }

cudaError_t launch_fold_reduce(const float *pm, const float *pp, int D, int R, int nbins, double *am,
                               double *ap, cudaStream_t st)
{
    const size_t n = (size_t)D * nbins;
    const unsigned int blocks = blocks_for(n, 32);
    // row groups: the largest power of two <= min(R, 32)
    if (R >= 32)
        fold_reduce_kernel<32><<<blocks, 32 * 32, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    else if (R >= 16)
        fold_reduce_kernel<16><<<blocks, 32 * 16, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    else if (R >= 8)
        fold_reduce_kernel<8><<<blocks, 32 * 8, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    else if (R >= 4)
        fold_reduce_kernel<4><<<blocks, 32 * 4, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    else if (R >= 2)
        fold_reduce_kernel<2><<<blocks, 32 * 2, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    else
        fold_reduce_kernel<1><<<blocks, 32, 0, st>>>(pm, pp, D, R, nbins, am, ap);
    return cudaGetLastError();
}

cudaError_t launch_fold_flush(double *am, double *ap, size_t n, cudaStream_t st)
{
    fold_flush_kernel<<<blocks_for(n, 256), 256, 0, st>>>(am, ap, n);
    return cudaGetLastError();
}

// Reads pinned host memory directly (mapped, unified addressing), so the
// upload is ordered on the compute stream alone and never waits behind a
// large input copy on the copy engines
__global__ void span_upload_kernel(const long long *__restrict__ h, int n, int cap, long long *__restrict__ a,
                                   long long *__restrict__ b, int *__restrict__ p, int *__restrict__ dest)
{
    const int *hp = reinterpret_cast<const int *>(h + 2 * (size_t)cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        a[i] = h[i];
        b[i] = h[cap + i];
        p[i] = hp[i];
        dest[i] = hp[cap + i];
    }
}

cudaError_t launch_span_upload(const long long *host, int n, int cap, long long *a, long long *b, int *phase0,
                               int *dest, cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    void *hd = nullptr;
    cudaError_t e = cudaHostGetDevicePointer(&hd, const_cast<long long *>(host), 0);
    if (e != cudaSuccess)
        return e;
    const unsigned int g = blocks_for((size_t)n, 256) < 64 ? blocks_for((size_t)n, 256) : 64;
    span_upload_kernel<<<g, 256, 0, st>>>(static_cast<const long long *>(hd), n, cap, a, b, phase0, dest);
    return cudaGetLastError();
}

cudaError_t launch_fold_readout(const double *am, size_t n, double scale, float *out, cudaStream_t st)
{
    fold_readout_kernel<<<blocks_for(n, 256), 256, 0, st>>>(am, n, scale, out);
    return cudaGetLastError();
}

cudaError_t launch_intensity(const float2 *a, const float2 *b, float *out, size_t n, cudaStream_t st)
{
    intensity_kernel<<<blocks_for(n, 256), 256, 0, st>>>(a, b, out, n);
    return cudaGetLastError();
}

int fold_series_block() { return kFoldBlock; }

cudaError_t launch_fold_series(const float *I, long long n, int R, const FoldArgs &f, int grid, int trials,
                               cudaStream_t st)
{
    const size_t sm =
        ibuf_floats(kFoldBlock) * sizeof(float) + fold_smem_bytes(f.nbins, f.span_cap, f.smem_prof != 0, 256);
    cudaError_t e = set_smem(fold_series_kernel, sm);
    if (e != cudaSuccess)
        return e;
    fold_series_kernel<<<dim3((unsigned)grid, (unsigned)trials), 256, sm, st>>>(I, n, R, f);
    return cudaGetLastError();
}

cudaError_t launch_encode_u16(const float2 *src, uint32_t *dst, size_t n, cudaStream_t st)
{
    encode_u16_kernel<<<blocks_for(n, 256), 256, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}

}  // namespace msosm
