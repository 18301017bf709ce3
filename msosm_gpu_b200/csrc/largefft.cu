// largefft.cu -- MS-OSM / OSM for FFT sizes above one thread block (N > 16384).
//
// Four-step FFT with N = N1 * N2 (N1 <= 1024 columns of a [N1][N2] view, N2
// <= 16384), n = N2*n1 + n2 and k = k1 + N1*k2:
//   forward  A[k1][n2] = W_N^(n2 k1) * FFT_N1 over n1 of x[N2 n1 + n2]   (column pass)
//            X[k1][k2] = FFT_N2 over n2 of A[k1][n2]                     (row pass)
//   inverse  B[k1][n2] = W_N^(-n2 k1) * IFFT_N2 over k2 of Y[k1][k2]     (row pass)
//            y[N2 n1 + n2] = IFFT_N1 over k1 of B[k1][n2]                (column pass)
// Spectra stay in the permuted [k1][k2] order from the forward transform to
// the inverse one: the per-bin operations (multiply by H, per-bin delay) do
// not care about order, so H and the delays are permuted once at set-up and
// no transpose is ever made.  The inverse column pass computes only
// n1 >= N1/2, the overlap-save half that is kept.
//
// Column passes run 16 columns per thread block (16 independent N1-point
// block FFTs whose global reads and writes are 128-byte rows); row passes run
// one N2-point block FFT per thread block.  Twiddles W_N^e come from
// sincospif of the exact float 2e/N.
#include "chirp.cuh"
#include "fft_smem.cuh"
#include "kernels.hpp"

#include <cuda_runtime.h>

namespace msosm {

namespace {

constexpr int kCols = 16;  // columns per thread block in the column passes

template <int LOG2N1>
struct ColShape {
    using F = FftShape<LOG2N1>;
    static constexpr int STR = F::SMEM + 1;  // odd stride: 16 columns hit 16 bank pairs
    static constexpr int THREADS = kCols * F::T;
    static constexpr size_t SMEM_BYTES = (size_t)kCols * STR * sizeof(float2);
};

__device__ __forceinline__ float2 twiddle_n(long long e, int log2n, float sign)
{
    // exp(sign * 2 pi i e / N): 2e/N is exact in float for N <= 2^24
    float s, c;
    sincospif(ldexpf((float)(2 * e), -log2n), &s, &c);
    return make_float2(c, sign * s);
}

template <int KIND>
__device__ __forceinline__ float2 load_in(const void *p, long long s)
{
    if constexpr (KIND == kInputC64) {
        return reinterpret_cast<const float2 *>(p)[s];
    } else {
        const uint32_t u = reinterpret_cast<const uint32_t *>(p)[s];
        const uint32_t x = u & 0xFFFFu, y = u >> 16;
        return make_float2(x ? (float)x - 32768.0f : 0.0f, y ? (float)y - 32768.0f : 0.0f);
    }
}

// Forward column pass.  KIND kInputC64 / kInputU16: the overlapping windows of
// one call (window w covers input samples [w*M - M, w*M + M), negative
// indices from the previous call's history); KIND 2: a plain vector of
// length `len` (zero beyond).  Output A[w][k1][n2] with the twiddle applied.
template <int LOG2N1, int KIND>
__global__ void __launch_bounds__(ColShape<LOG2N1>::THREADS) lcol_fwd_kernel(LargeColArgs a)
{
    using F = FftShape<LOG2N1>;
    using C = ColShape<LOG2N1>;
    constexpr int T1 = F::T;
    extern __shared__ float2 smem[];
    const int c = threadIdx.x % kCols, j = threadIdx.x / kCols;
    const long long n2 = (long long)blockIdx.x * kCols + c;
    const int w = blockIdx.y;
    const long long N = a.N, N2 = a.N2, M = N / 2;
    float2 *buf = smem + c * C::STR;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        const long long pos = N2 * (j + r * T1) + n2;
        float2 x;
        if constexpr (KIND == 2) {
            x = pos < a.len ? reinterpret_cast<const float2 *>(a.input)[pos] : make_float2(0.f, 0.f);
        } else {
            const long long s = (long long)w * M + pos - M;
            x = s < 0 ? a.hist_in[M + s] : load_in<KIND>(a.input, s);
            if (w == a.count - 1 && pos >= M)
                a.hist_out[pos - M] = x;
        }
        v[r] = x;
    }
    dft16<-1>(v);
    stage_store<LOG2N1, 0>(v, buf, j);
    run_stages<LOG2N1, -1, false>(v, buf, buf, j, a.tw1);
    float2 *out = a.out + (size_t)w * N;
#pragma unroll
    for (int slot = 0; slot < 16; ++slot) {
        const int k1 = last_out_index<LOG2N1>(j, slot);
        out[(size_t)k1 * N2 + n2] = cmul(v[slot], twiddle_n(n2 * k1, a.log2n, -1.f));
    }
}

// Row passes (one N2-point FFT per thread block, row k1 = blockIdx.x, window
// or block w = blockIdx.y, trial d = blockIdx.z).
//   MODE 0 forward:  A[w][k1][:] -> spectrum ring row (slot of block k0+w)
//   MODE 1 inverse:  gather X[k - delay][k1][k2] * H[d][k1][k2] from the ring,
//                    inverse FFT, twiddle W_N^(-n2 k1) -> B[d][w][k1][n2]
//   MODE 2 forward:  A[w][k1][:] -> out[w][k1][:] (filter design)
template <int LOG2N2, int MODE>
__global__ void __launch_bounds__(FftShape<LOG2N2>::T) lrow_kernel(LargeRowArgs a)
{
    using F = FftShape<LOG2N2>;
    constexpr int N2 = F::N, T2 = F::T;
    extern __shared__ float2 smem[];
    const int j = threadIdx.x;
    const int k1 = blockIdx.x, w = blockIdx.y, d = blockIdx.z;
    const long long N = a.N;
    const size_t row = (size_t)k1 * N2;
    float2 v[16];
    if constexpr (MODE == 1) {
        const long long kg = a.k0 + w;
        const int smask = a.S - 1;
        const int slot_k = (int)(kg & smask);
        const float2 *__restrict__ Hd = a.H + (size_t)d * N + row;
        const uint16_t *__restrict__ dl = a.delays + (size_t)d * N + row;
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int k2 = j + r * T2;
            const int dly = (int)dl[k2];
            float2 x = make_float2(0.f, 0.f);
            if (kg >= dly)
                x = a.ring[(size_t)((slot_k - dly) & smask) * N + row + k2];
            v[r] = cmul(x, Hd[k2]);
        }
        dft16<+1>(v);
        stage_store<LOG2N2, 0>(v, smem, j);
        run_stages<LOG2N2, +1, false>(v, smem, smem, j, a.tw2);
        float2 *out = a.out + ((size_t)d * a.count + w) * N + row;
#pragma unroll
        for (int slot = 0; slot < 16; ++slot) {
            const int n2 = last_out_index<LOG2N2>(j, slot);
            out[n2] = cmul(v[slot], twiddle_n((long long)n2 * k1, a.log2n, +1.f));
        }
    } else {
        const float2 *in = a.in + (size_t)w * N + row;
#pragma unroll
        for (int r = 0; r < 16; ++r)
            v[r] = in[j + r * T2];
        dft16<-1>(v);
        stage_store<LOG2N2, 0>(v, smem, j);
        run_stages<LOG2N2, -1, false>(v, smem, smem, j, a.tw2);
        float2 *out = MODE == 0 ? a.ring + (size_t)((a.k0 + w) & (a.S - 1)) * N + row
                                : a.out + (size_t)w * N + row;
#pragma unroll
        for (int slot = 0; slot < 16; ++slot)
            out[last_out_index<LOG2N2>(j, slot)] = v[slot];
    }
}

// Inverse column pass of B[d][w][k1][n2], keeping n1 >= N1/2: output sample
// t = N2*(n1 - N1/2) + n2 of block w goes to series[d][w*M + t] and/or, as
// |y|^2 or |y|, to intensity[d][w*M + t].
template <int LOG2N1>
__global__ void __launch_bounds__(ColShape<LOG2N1>::THREADS) lcol_inv_kernel(LargeColArgs a)
{
    using F = FftShape<LOG2N1>;
    using C = ColShape<LOG2N1>;
    constexpr int T1 = F::T, N1 = F::N;
    constexpr int RL = F::radix(F::NST - 1);
    extern __shared__ float2 smem[];
    const int c = threadIdx.x % kCols, j = threadIdx.x / kCols;
    const long long n2 = (long long)blockIdx.x * kCols + c;
    const int w = blockIdx.y, d = blockIdx.z;
    const long long N = a.N, N2 = a.N2, M = N / 2;
    float2 *buf = smem + c * C::STR;
    const float2 *in = a.in + ((size_t)d * a.count + w) * N;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r)
        v[r] = in[(size_t)(j + r * T1) * N2 + n2];
    dft16<+1>(v);
    stage_store<LOG2N1, 0>(v, buf, j);
    run_stages<LOG2N1, +1, false>(v, buf, buf, j, a.tw1);
    const size_t base = ((size_t)d * a.count + w) * M;
#pragma unroll
    for (int slot = 0; slot < 16; ++slot) {
        if ((slot % RL) >= RL / 2) {
            const int n1 = last_out_index<LOG2N1>(j, slot);
            const size_t t = (size_t)N2 * (n1 - N1 / 2) + n2;
            const float2 y = v[slot];
            if (a.series)
                a.series[base + t] = y;
            if (a.intensity) {
                const float p = y.x * y.x + y.y * y.y;
                a.intensity[base + t] = a.detect ? sqrtf(p) : p;
            }
        }
    }
}

// Filter design helpers.
// h (M points, the reference's fftshift: h index j holds offset (j + M/2) mod M)
// written conjugated, so that IFFT_M(h) = conj(FFT_M(conj h)).
__global__ void chirp_conj_kernel(const ChirpParams *cp, float2 *out, long long M, int sign)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M)
        return;
    const unsigned int i = (unsigned int)((j + M / 2) & (M - 1));
    float c, s;
    chirp_cis(chirp_phase(*cp, i), c, s);
    const float im = sign < 0 ? -s : s;
    out[j] = make_float2(c, -im);
}

// out[k] = conj(in[(k mod K1)*K2 + k / K1]) for k < K (un-permute + conj), then
// zero up to len_out
__global__ void unpermute_conj_kernel(const float2 *in, float2 *out, long long K, long long K1, long long K2,
                                      long long len_out)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) {
        const float2 x = in[(k % K1) * K2 + k / K1];
        out[k] = make_float2(x.x, -x.y);
    } else if (k < len_out) {
        out[k] = make_float2(0.f, 0.f);
    }
}

__global__ void conj_scale_kernel(float2 *x, long long n, float scale, int conj)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float2 v = x[i];
        x[i] = make_float2(v.x * scale, (conj ? -v.y : v.y) * scale);
    }
}

// block FFT of `count` vectors of N <= 16384 points (natural order)
template <int LOG2N, int SIGN>
__global__ void __launch_bounds__(FftShape<LOG2N>::T) vec_fft_kernel(const float2 *in, float2 *out, const float2 *tw)
{
    using F = FftShape<LOG2N>;
    extern __shared__ float2 smem[];
    const int j = threadIdx.x;
    const size_t off = (size_t)blockIdx.x * F::N;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r)
        v[r] = in[off + j + r * F::T];
    dft16<SIGN>(v);
    stage_store<LOG2N, 0>(v, smem, j);
    run_stages<LOG2N, SIGN, false>(v, smem, smem, j, tw);
#pragma unroll
    for (int slot = 0; slot < 16; ++slot)
        out[off + last_out_index<LOG2N>(j, slot)] = v[slot];
}

template <typename K>
cudaError_t smem_attr(K k, size_t bytes)
{
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

unsigned int nblk(long long n, unsigned int t) { return (unsigned int)((n + t - 1) / t); }

#define LDISPATCH_COL(log2n, CALL)                                                                     \
    switch (log2n) {                                                                                   \
    case 6: return CALL(6);                                                                            \
    case 7: return CALL(7);                                                                            \
    case 8: return CALL(8);                                                                            \
    case 9: return CALL(9);                                                                            \
    case 10: return CALL(10);                                                                          \
    default: break;                                                                                    \
    }
#define LDISPATCH_ROW(log2n, CALL)                                                                     \
    switch (log2n) {                                                                                   \
    case 6: return CALL(6);                                                                            \
    case 7: return CALL(7);                                                                            \
    case 8: return CALL(8);                                                                            \
    case 9: return CALL(9);                                                                            \
    case 10: return CALL(10);                                                                          \
    case 11: return CALL(11);                                                                          \
    case 12: return CALL(12);                                                                          \
    case 13: return CALL(13);                                                                          \
    case 14: return CALL(14);                                                                          \
    default: break;                                                                                    \
    }

template <int L1>
cudaError_t col_fwd_t(int kind, const LargeColArgs &a, int windows, cudaStream_t st)
{
    using C = ColShape<L1>;
    const dim3 grid((unsigned)(a.N2 / kCols), (unsigned)windows);
    cudaError_t e;
    if (kind == kInputU16) {
        auto k = lcol_fwd_kernel<L1, kInputU16>;
        if ((e = smem_attr(k, C::SMEM_BYTES)) != cudaSuccess)
            return e;
        k<<<grid, C::THREADS, C::SMEM_BYTES, st>>>(a);
    } else if (kind == kInputC64) {
        auto k = lcol_fwd_kernel<L1, kInputC64>;
        if ((e = smem_attr(k, C::SMEM_BYTES)) != cudaSuccess)
            return e;
        k<<<grid, C::THREADS, C::SMEM_BYTES, st>>>(a);
    } else {
        auto k = lcol_fwd_kernel<L1, 2>;
        if ((e = smem_attr(k, C::SMEM_BYTES)) != cudaSuccess)
            return e;
        k<<<grid, C::THREADS, C::SMEM_BYTES, st>>>(a);
    }
    return cudaGetLastError();
}

template <int L1>
cudaError_t col_inv_t(const LargeColArgs &a, int blocks, int trials, cudaStream_t st)
{
    using C = ColShape<L1>;
    auto k = lcol_inv_kernel<L1>;
    cudaError_t e = smem_attr(k, C::SMEM_BYTES);
    if (e != cudaSuccess)
        return e;
    k<<<dim3((unsigned)(a.N2 / kCols), (unsigned)blocks, (unsigned)trials), C::THREADS, C::SMEM_BYTES, st>>>(a);
    return cudaGetLastError();
}

template <int L2>
cudaError_t row_t(int mode, const LargeRowArgs &a, int rows, int windows, int trials, cudaStream_t st)
{
    const size_t sm = FftShape<L2>::SMEM * sizeof(float2);
    const dim3 grid((unsigned)rows, (unsigned)windows, (unsigned)trials);
    cudaError_t e;
    auto go = [&](auto k) -> cudaError_t {
        if ((e = smem_attr(k, sm)) != cudaSuccess)
            return e;
        k<<<grid, FftShape<L2>::T, sm, st>>>(a);
        return cudaGetLastError();
    };
    if (mode == 0)
        return go(lrow_kernel<L2, 0>);
    if (mode == 1)
        return go(lrow_kernel<L2, 1>);
    return go(lrow_kernel<L2, 2>);
}

template <int L, int SIGN>
cudaError_t vec_t(const float2 *in, float2 *out, const float2 *tw, int count, cudaStream_t st)
{
    const size_t sm = FftShape<L>::SMEM * sizeof(float2);
    auto k = vec_fft_kernel<L, SIGN>;
    cudaError_t e = smem_attr(k, sm);
    if (e != cudaSuccess)
        return e;
    k<<<count, FftShape<L>::T, sm, st>>>(in, out, tw);
    return cudaGetLastError();
}

}  // namespace

void large_split(int log2n, int &log2n1, int &log2n2)
{
    // N2 as large as a block FFT allows (16384), N1 >= 64 columns of 16
    log2n2 = log2n - 6 < kMaxLog2N ? log2n - 6 : kMaxLog2N;
    log2n1 = log2n - log2n2;
}

bool large_supported(int log2n)
{
    if (log2n <= kMaxLog2N || log2n > 24)
        return false;
    int l1, l2;
    large_split(log2n, l1, l2);
    return l1 >= 6 && l1 <= 10 && l2 >= 6 && l2 <= kMaxLog2N;
}

cudaError_t launch_large_col_fwd(int log2n1, int kind, const LargeColArgs &a, int windows, cudaStream_t st)
{
#define CALL(L) col_fwd_t<L>(kind, a, windows, st)
    LDISPATCH_COL(log2n1, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_large_col_inv(int log2n1, const LargeColArgs &a, int blocks, int trials, cudaStream_t st)
{
#define CALL(L) col_inv_t<L>(a, blocks, trials, st)
    LDISPATCH_COL(log2n1, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_large_row(int log2n2, int mode, const LargeRowArgs &a, int rows, int windows, int trials,
                             cudaStream_t st)
{
#define CALL(L) row_t<L>(mode, a, rows, windows, trials, st)
    LDISPATCH_ROW(log2n2, CALL)
#undef CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_vec_fft(int log2n, int sign, const float2 *in, float2 *out, const float2 *tw, int count,
                           cudaStream_t st)
{
    if (sign < 0) {
#define CALL(L) vec_t<L, -1>(in, out, tw, count, st)
        LDISPATCH_ROW(log2n, CALL)
#undef CALL
    } else {
#define CALL(L) vec_t<L, +1>(in, out, tw, count, st)
        LDISPATCH_ROW(log2n, CALL)
#undef CALL
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_chirp_conj(const ChirpParams *cp, float2 *out, long long M, int sign, cudaStream_t st)
{
    chirp_conj_kernel<<<nblk(M, 256), 256, 0, st>>>(cp, out, M, sign);
    return cudaGetLastError();
}

cudaError_t launch_unpermute_conj(const float2 *in, float2 *out, long long K, long long K1, long long K2,
                                  long long len_out, cudaStream_t st)
{
    unpermute_conj_kernel<<<nblk(len_out, 256), 256, 0, st>>>(in, out, K, K1, K2, len_out);
    return cudaGetLastError();
}

cudaError_t launch_conj_scale(float2 *x, long long n, float scale, int conj, cudaStream_t st)
{
    conj_scale_kernel<<<nblk(n, 256), 256, 0, st>>>(x, n, scale, conj);
    return cudaGetLastError();
}

}  // namespace msosm
