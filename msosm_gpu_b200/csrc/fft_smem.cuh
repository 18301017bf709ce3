// fft_smem.cuh -- block-wide complex FFT in shared memory for sm_100a.
//
// One thread block transforms N = 2^LOG2N points (32 <= N <= 16384) with
// T = N/16 threads.  Every thread holds 16 complex values in registers.
// Stages are Stockham autosort (natural order in, natural order out): radix
// 16 for floor(LOG2N/4) stages and, when LOG2N is not a multiple of 4, one
// last stage of radix 2, 4 or 8 in which each thread runs 16/R butterflies.
//
//   stage with radix R, sub-transform size Ns (product of earlier radices),
//   butterfly j in [0, N/R):
//     load   v[r] = x[j + r*N/R]                       r = 0..R-1
//     twiddle v[r] *= W^(sign * (j mod Ns) * r), W = exp(2 pi i/(Ns*R))
//     v = DFT_R(v)
//     store  x'[(j / Ns)*Ns*R + (j mod Ns) + r*Ns] = v[r]
//
// Shared memory is float2 with one pad slot every 16 elements (index
// p + p/16): with this layout the 64-bit accesses of every load and store
// pattern above are free of bank conflicts for all N used here.
#pragma once

#include <cuda_runtime.h>

namespace msosm {

__host__ __device__ constexpr int smem_pad(int p) { return p + (p >> 4); }
__host__ __device__ constexpr int smem_elems(int n) { return n + (n >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by SIGN*i  (SIGN = -1: forward transform, +1: inverse)
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 a)
{
    return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// exp(SIGN * 2 pi i * e / 16) for e = 1..15, constants from the mathematics
// (cos(pi/8), sin(pi/8), 1/sqrt(2)).
template <int SIGN, int E>
__device__ __forceinline__ float2 w16(float2 a)
{
    constexpr float C1 = 0.92387953251128675613f;  // cos(pi/8)
    constexpr float S1 = 0.38268343236508977173f;  // sin(pi/8)
    constexpr float R2 = 0.70710678118654752440f;  // 1/sqrt(2)
    constexpr int e = E & 15;
    if constexpr (e == 0) {
        return a;
    } else if constexpr (e == 4) {
        return mul_si<SIGN>(a);
    } else if constexpr (e == 8) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (e == 12) {
        return mul_si<-SIGN>(a);
    } else {
        // general angle theta = 2 pi e / 16
        constexpr float cs[16] = {1.f, C1, R2, S1, 0.f, -S1, -R2, -C1, -1.f, -C1, -R2, -S1, 0.f, S1, R2, C1};
        constexpr float sn[16] = {0.f, S1, R2, C1, 1.f, C1, R2, S1, 0.f, -S1, -R2, -C1, -1.f, -C1, -R2, -S1};
        const float c = cs[e];
        const float s = SIGN * sn[e];
        return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

template <int SIGN>
__device__ __forceinline__ void dft2(float2 *v)
{
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

// natural order in and out
template <int SIGN>
__device__ __forceinline__ void dft4(float2 &x0, float2 &x1, float2 &x2, float2 &x3)
{
    const float2 a = cadd(x0, x2), b = csub(x0, x2);
    const float2 c = cadd(x1, x3), d = mul_si<SIGN>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

template <int SIGN>
__device__ __forceinline__ void dft4(float2 *v) { dft4<SIGN>(v[0], v[1], v[2], v[3]); }

template <int SIGN>
__device__ __forceinline__ void dft8(float2 *v)
{
    // X[k] = E[k] + W8^k O[k], X[k+4] = E[k] - W8^k O[k]
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<SIGN>(e0, e1, e2, e3);
    dft4<SIGN>(o0, o1, o2, o3);
    o1 = w16<SIGN, 2>(o1);
    o2 = w16<SIGN, 4>(o2);
    o3 = w16<SIGN, 6>(o3);
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

template <int SIGN>
__device__ __forceinline__ void dft16(float2 *v)
{
    // n = q + 4m, k = s + 4t:  X[s+4t] = sum_q W4^(qt) W16^(qs) sum_m x[q+4m] W4^(ms)
#pragma unroll
    for (int q = 0; q < 4; ++q)
        dft4<SIGN>(v[q], v[q + 4], v[q + 8], v[q + 12]);
    // now v[q + 4s] holds A[q][s]
    v[5] = w16<SIGN, 1>(v[5]);
    v[9] = w16<SIGN, 2>(v[9]);
    v[13] = w16<SIGN, 3>(v[13]);
    v[6] = w16<SIGN, 2>(v[6]);
    v[10] = w16<SIGN, 4>(v[10]);
    v[14] = w16<SIGN, 6>(v[14]);
    v[7] = w16<SIGN, 3>(v[7]);
    v[11] = w16<SIGN, 6>(v[11]);
    v[15] = w16<SIGN, 9>(v[15]);
    float2 o[16];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        float2 a0 = v[0 + 4 * s], a1 = v[1 + 4 * s], a2 = v[2 + 4 * s], a3 = v[3 + 4 * s];
        dft4<SIGN>(a0, a1, a2, a3);
        o[s] = a0;
        o[s + 4] = a1;
        o[s + 8] = a2;
        o[s + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i)
        v[i] = o[i];
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(float2 *v)
{
    if constexpr (R == 2)
        dft2<SIGN>(v);
    else if constexpr (R == 4)
        dft4<SIGN>(v);
    else if constexpr (R == 8)
        dft8<SIGN>(v);
    else
        dft16<SIGN>(v);
}

template <int LOG2N>
struct FftShape {
    static_assert(LOG2N >= 5 && LOG2N <= 14, "block FFT supports 32..16384 points");
    static constexpr int N = 1 << LOG2N;
    static constexpr int T = N / 16;  // threads per transform
    static constexpr int NS16 = LOG2N / 4;
    static constexpr int RL = 1 << (LOG2N & 3);  // radix of the extra last stage (1: none)
    static constexpr int NST = NS16 + (RL > 1 ? 1 : 0);
    __host__ __device__ static constexpr int radix(int s) { return s < NS16 ? 16 : RL; }
    __host__ __device__ static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
    static constexpr int SMEM = smem_elems(N);  // float2 elements per buffer
};

// Shared-memory addressing.  For stages S >= 1 the load stride N/R and, for
// stores, the sub-transform size NS are multiples of 16, so
// smem_pad(base + r*X) = smem_pad(base) + r*(X + X/16): one padded base per
// butterfly and compile-time offsets per element.  Stage 0 (NS = 1) stores
// element r of butterfly j at 16j + r, padded 17j + r.

// Load of stage S (S >= 1) from shared memory.
template <int LOG2N, int S>
__device__ __forceinline__ void stage_load(float2 (&v)[16], const float2 *__restrict__ buf, int tid)
{
    using F = FftShape<LOG2N>;
    constexpr int R = F::radix(S), B = 16 / R, STRIDE = F::N / R;
    static_assert(S >= 1 && STRIDE % 16 == 0, "stride must be a multiple of 16");
    constexpr int PSTRIDE = STRIDE + STRIDE / 16;
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int j = tid + q * F::T;
        const float2 *p = buf + smem_pad(j);
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[q * R + r] = p[r * PSTRIDE];
    }
}

// Twiddles W^(sign*m*r), r = 1..R-1, from two table reads (W^m and W^(4m))
// and at most three complex products each, tw[e] = exp(sign 2 pi i e / N).
template <int R>
__device__ __forceinline__ void twiddle_powers(float2 (&w)[16], const float2 *__restrict__ tw, int idx1, int idx4)
{
    w[1] = __ldg(&tw[idx1]);
    if constexpr (R > 2) {
        w[2] = cmul(w[1], w[1]);
        w[3] = cmul(w[2], w[1]);
    }
    if constexpr (R > 4) {
        w[4] = __ldg(&tw[idx4]);
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
    }
    if constexpr (R > 8) {
        w[8] = cmul(w[4], w[4]);
        w[9] = cmul(w[8], w[1]);
        w[10] = cmul(w[8], w[2]);
        w[11] = cmul(w[8], w[3]);
        w[12] = cmul(w[8], w[4]);
        w[13] = cmul(w[12], w[1]);
        w[14] = cmul(w[12], w[2]);
        w[15] = cmul(w[12], w[3]);
    }
}

// Twiddle + butterflies of stage S (tw: table exp(SIGN 2 pi i e / N), e < N).
template <int LOG2N, int S, int SIGN>
__device__ __forceinline__ void stage_compute(float2 (&v)[16], int tid, const float2 *__restrict__ tw)
{
    using F = FftShape<LOG2N>;
    constexpr int R = F::radix(S), B = 16 / R, NS = F::ns(S);
#pragma unroll
    for (int q = 0; q < B; ++q) {
        if constexpr (NS > 1) {
            const int j = tid + q * F::T;
            const int m = j & (NS - 1);
            constexpr int STEP = F::N / (NS * R);
            float2 w[16];
            twiddle_powers<R>(w, tw, m * STEP, 4 * m * STEP);
#pragma unroll
            for (int r = 1; r < R; ++r)
                v[q * R + r] = cmul(v[q * R + r], w[r]);
        }
        dft<R, SIGN>(&v[q * R]);
    }
}

template <int LOG2N, int S>
__device__ __forceinline__ void stage_store(const float2 (&v)[16], float2 *__restrict__ buf, int tid)
{
    using F = FftShape<LOG2N>;
    constexpr int R = F::radix(S), B = 16 / R, NS = F::ns(S);
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int j = tid + q * F::T;
        if constexpr (NS == 1) {
            float2 *p = buf + 17 * j;
#pragma unroll
            for (int r = 0; r < R; ++r)
                p[r] = v[q * R + r];
        } else {
            static_assert(NS % 16 == 0, "sub-transform size must be a multiple of 16");
            constexpr int PNS = NS + NS / 16;
            float2 *p = buf + smem_pad((j / NS) * NS * R + (j & (NS - 1)));
#pragma unroll
            for (int r = 0; r < R; ++r)
                p[r * PNS] = v[q * R + r];
        }
    }
}

// Output index of register slot (q, r) of the last stage: n = j + r*N/R.
template <int LOG2N>
__device__ __forceinline__ int last_out_index(int tid, int slot)
{
    using F = FftShape<LOG2N>;
    constexpr int S = F::NST - 1;
    constexpr int R = F::radix(S);
    const int q = slot / R, r = slot % R;
    return tid + q * F::T + r * (F::N / R);
}

// Run stages 1 .. NST-1 after stage 0 has been stored to buf0.  With
// PINGPONG stage s reads buf[(s-1)&1] and writes buf[s&1] (one barrier per
// stage); otherwise a single buffer with a barrier on each side of the
// loads.  On return v holds the outputs of the last stage (see
// last_out_index); the last stage does not write shared memory.  Threads
// with active == false take part in the barriers only.
// Entry: stage-0 results stored, no barrier yet.  Exit: this thread's
// last-stage loads are done (no barrier after them): the caller must
// synchronise before anything overwrites the buffer the last stage read,
// buf[(NST-2)&1] with PINGPONG, buf0 otherwise.
template <int LOG2N, int SIGN, bool PINGPONG, int S = 1>
__device__ __forceinline__ void run_stages(float2 (&v)[16], float2 *buf0, float2 *buf1, int tid,
                                           const float2 *__restrict__ tw, bool active = true)
{
    using F = FftShape<LOG2N>;
    if constexpr (S < F::NST) {
        float2 *src = PINGPONG ? (((S - 1) & 1) ? buf1 : buf0) : buf0;
        float2 *dst = PINGPONG ? ((S & 1) ? buf1 : buf0) : buf0;
        __syncthreads();
        if (active)
            stage_load<LOG2N, S>(v, src, tid);
        if constexpr (S + 1 < F::NST) {
            if constexpr (!PINGPONG)
                __syncthreads();
            if (active) {
                stage_compute<LOG2N, S, SIGN>(v, tid, tw);
                stage_store<LOG2N, S>(v, dst, tid);
            }
            run_stages<LOG2N, SIGN, PINGPONG, S + 1>(v, buf0, buf1, tid, tw, active);
        } else {
            if (active)
                stage_compute<LOG2N, S, SIGN>(v, tid, tw);
        }
    }
}

// Buffer read by the last stage (must not be overwritten before a barrier).
template <int LOG2N, bool PINGPONG>
__device__ __forceinline__ constexpr bool last_reads_buf1()
{
    return PINGPONG && (((FftShape<LOG2N>::NST - 2) & 1) == 1);
}

}  // namespace msosm
