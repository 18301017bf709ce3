// tc_dedisp.cu -- tensor-core (tcgen05) variant of the fused dedispersion
// kernel for 4096-, 8192- and 16384-point transforms.
//
// Same semantics as dedisp_kernel (kernels.cu), which replaces
// ComplexMultiplyDelay_concurrent_batch + inverse cufftExecC2C +
// DiscardSamples_concurrent_batch (gpu/gpu_kernel.cu:128-198,236-258) and the
// host fold of Fold_GPU (folding/fold_gpu.cpp:48-194): per (trial, block)
// gather X[k - delay[b]][b] * H[b] from the spectrum ring, inverse transform,
// keep outputs m >= M, write the series and/or detect and fold.  Here the
// inverse transform of a step (two consecutive blocks of one trial at 4096
// and 8192 points, one block at 16384) runs as two f16 GEMMs with f32
// accumulation in tensor memory (factorisation and layouts in tc_layout.hpp):
// at 4096 GEMM 1 (M 128 = 2 blocks x 64 k1, N 128, K 128), a twiddle pass on
// the CUDA cores, GEMM 2 (M 128 = 2 blocks x 64 m2, N 64, K 128).
//
// Precision: the gathered products of a work item (one trial, a range of
// blocks) are scaled by a power of two chosen so that no component can reach
// 2^8 -- from the largest component of every ring row the item reads
// (recorded by the forward kernel) times the trial's largest filter
// component -- so every GEMM 1 sum stays below 2^15 and every twiddled value
// below 2^15.5, inside f16; f16's 2^-24..2^16 range leaves quiet stretches
// far from underflow unless a burst in the range is ~10^6 times stronger.  The
// twiddle multiply runs in f16 arithmetic on f16-rounded twiddles.  The
// scale is undone exactly on the f32 results.
//
// Waits on the tensor core are bounded (1 s of global timer): on a timeout
// the kernel records a nonzero status, waits once more for its last GEMM,
// frees its tensor memory and returns.
#include <algorithm>
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fold_dev.cuh"
#include "kernels.hpp"
#include "tc_layout.hpp"

namespace msosm {
namespace {

using namespace tc;

constexpr unsigned long long kWaitLimitNs = 1000000000ull;
// Wait limits below this probe without suspending (test_wait); longer ones
// use try_wait, which suspends for the hardware's own time limit per
// attempt (an explicit 100 us suspend hint was 0.4-0.8 % slower)
constexpr unsigned long long kProbeBelowNs = 100000ull;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Probe without suspending: has the phase of the given parity completed?
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity to complete; false after limit_ns.
// A limit below kProbeBelowNs probes without suspending; a limit of 0
// gives up at once, without probing (a diagnostic setting: the kernel then
// takes its timeout exit, whose drain of the GEMMs in flight keeps its own
// limit).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns)
{
    if (limit_ns == 0)
        return false;
    if (limit_ns < kProbeBelowNs) {
        if (mbar_test_wait(bar, parity))
            return true;
        const unsigned long long t0 = global_ns();
        while (!mbar_test_wait(bar, parity))
            if (global_ns() - t0 > limit_ns)
                return false;
        return true;
    }
    if (mbar_try_wait(bar, parity))
        return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns)
            return false;
    return true;
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D (tensor memory) = A * B (+ D when accumulate), one thread issues
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrive on the mbarrier once every GEMM this thread issued has completed
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Two 32-lane x 16-column loads from tensor memory (lane = GEMM row, one
// 32-bit column per register) and the wait for them, in one statement so the
// registers are not read before they arrive.
__device__ __forceinline__ void tmem_ld_2x16(uint32_t ta, uint32_t tb, float (&a)[16], float (&b)[16])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, "
        "[%33];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        a[i] = __uint_as_float(r[i]);
        b[i] = __uint_as_float(r[16 + i]);
    }
}

// 32 words of this thread's TMEM lane, columns ta .. ta + 31 (two x16 stores), then the wait
__device__ __forceinline__ void tmem_st_32(uint32_t ta, const uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17};\n\t"
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%1], {%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33};\n\t"
        "tcgen05.wait::st.sync.aligned;" ::"r"(ta), "r"(ta + 16),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]),
        "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
        "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
}

// D1 re / im (x16 each) and 8 + 8 twiddle words (x8 each), one wait
__device__ __forceinline__ void tmem_ld_twiddle(uint32_t ta, uint32_t tb, uint32_t tc, uint32_t td, float (&a)[16],
                                                float (&b)[16], uint32_t (&c)[8], uint32_t (&d)[8])
{
    uint32_t r[48];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%48];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%49];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%32,%33,%34,%35,%36,%37,%38,%39}, [%50];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%40,%41,%42,%43,%44,%45,%46,%47}, [%51];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47])
        : "r"(ta), "r"(tb), "r"(tc), "r"(td)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        a[i] = __uint_as_float(r[i]);
        b[i] = __uint_as_float(r[16 + i]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        c[i] = r[32 + i];
        d[i] = r[40 + i];
    }
}

// The 16-bit operand type: f16 (scaled into range) or bf16.
struct F16 {
    using h1 = __half;
    using h2 = __half2;
    static constexpr uint32_t fmt = 0;  // instruction-descriptor A/B format
    __device__ static h2 pack(float lo, float hi) { return __floats2half2_rn(lo, hi); }
    __device__ static h1 one(float v) { return __float2half_rn(v); }
};
struct BF16 {
    using h1 = __nv_bfloat16;
    using h2 = __nv_bfloat162;
    static constexpr uint32_t fmt = 1;
    __device__ static h2 pack(float lo, float hi) { return __floats2bfloat162_rn(lo, hi); }
    __device__ static h1 one(float v) { return __float2bfloat16_rn(v); }
};

template <class E>
__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const typename E::h2 h = E::pack(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void st_shared_v4(unsigned char *p, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    *reinterpret_cast<uint4 *>(p) = make_uint4(a, b, c, d);
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The constant operands, K-major: [C | S] of the N2-point inverse DFT for
// GEMM 1 and of the 64-point one (outputs m1 = 32..63) for GEMM 2.
//   GEMM 1, B1[n][k2], k2 < N2: n < N2 -> cos(2 pi k2 n / N2),
//     n >= N2 -> sin(2 pi k2 (n - N2) / N2)           (output frequency m2)
//   GEMM 2, B2[n][k1], k1 < 64: n < 32 -> cos(2 pi k1 (32 + n) / 64),
//     n >= 32 -> sin(2 pi k1 n / 64)                   (output m1 = 32..63)
// At N = 16384 (N1 = N2 = 128) GEMM 2 reads B1's columns 64..127 (C) and
// 192..255 (S) instead of a B2.  At N = 4096 (N1 = N2 = 64) the paired
// tables of TcShape::PAIRED replace B1 and B2 (filled by the first branch).
template <class E, int LOG2N>
__device__ void fill_constants(unsigned char *sm, int tid)
{
    using S = TcShape<LOG2N>;
    constexpr int N2 = S::N2;
    if constexpr (S::PAIRED) {
        // column n: quarter q = n / 32 holds C (q even) or S (q odd) of
        // frequency m = n % 32 (q < 2) or 32 + n % 32 (q >= 2); B1N holds -S
        // where B1 holds C, and C where it holds S
        for (int e = tid; e < 2 * N2 * N2; e += (int)blockDim.x) {
            const int n = e / N2, k = e % N2, q = n >> 5, m = (n & 31) + (q >= 2 ? 32 : 0);
            float s, c;
            sincospif((float)((k * m) & (N2 - 1)) * (2.0f / N2), &s, &c);
            const int off = k_off(n, k, (int)S::SBO_B1);
            *reinterpret_cast<typename E::h1 *>(sm + S::SMEM_B1 + off) = E::one((q & 1) ? s : c);
            *reinterpret_cast<typename E::h1 *>(sm + S::SMEM_B1N + off) = E::one((q & 1) ? c : -s);
        }
        return;
    }
    for (int e = tid; e < 2 * N2 * N2; e += (int)blockDim.x) {
        const int n = e / N2, k = e % N2;
        float s, c;
        sincospif((float)((k * (n & (N2 - 1))) & (N2 - 1)) * (2.0f / N2), &s, &c);
        *reinterpret_cast<typename E::h1 *>(sm + S::SMEM_B1 + k_off(n, k, (int)S::SBO_B1)) = E::one(n < N2 ? c : s);
    }
    for (int e = tid; e < (S::B2_BYTES ? 64 * 64 : 0); e += (int)blockDim.x) {
        const int n = e >> 6, k = e & 63;
        float s, c;
        sincospif((float)((k * (32 + (n & 31))) & 63) * (1.0f / 32.0f), &s, &c);
        *reinterpret_cast<typename E::h1 *>(sm + S::SMEM_B2 + k_off(n, k)) = E::one(n < 32 ? c : s);
        if constexpr (S::B2N_BYTES != 0)
            *reinterpret_cast<typename E::h1 *>(sm + S::SMEM_B2N + k_off(n, k)) = E::one(n < 32 ? -s : c);
    }
}

// mbarriers (GEMM 1, GEMM 2) + tensor memory; every thread returns the TMEM base
template <int LOG2N>
__device__ uint32_t tc_setup(unsigned char *sm, uint32_t s0, int tid, int warp)
{
    using S = TcShape<LOG2N>;
    if (tid == 0) {
        mbar_init(s0 + S::SMEM_CTL, 1);
        mbar_init(s0 + S::SMEM_CTL + 8, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(s0 + S::SMEM_CTL + 16, S::TMEM_COLS);
        tmem_relinquish();
    }
    fence_proxy_async();  // shared-memory operands written so far -> tensor core
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *reinterpret_cast<volatile uint32_t *>(sm + S::SMEM_CTL + 16);
}

template <int LOG2N>
__device__ __forceinline__ void tc_teardown(uint32_t tmem, int warp)
{
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TcShape<LOG2N>::TMEM_COLS);
    }
}

// One complex GEMM: D (2 half columns: [Re | Im]) = data (128 rows x [Re |
// Im], K = 2 x 16 ksteps, MN-major at a) x the DFT whose [C | S] (K = 16
// ksteps, 2 half columns, N-group stride sbo) is at b.  Three passes of
// ksteps K = 16 steps: Re x [C | S], then -Im x S into the Re half, Im x C
// into the Im half.
template <class E>
__device__ __forceinline__ void issue_cgemm(uint32_t tmem_d, uint32_t a, uint32_t b, int half, int ksteps,
                                            uint32_t sbo)
{
    const uint32_t id_full = idesc_f16(128, 2 * half, true, false, E::fmt);
    const uint32_t id_neg = idesc_f16(128, half, true, true, E::fmt);
    const uint32_t id_half = idesc_f16(128, half, true, false, E::fmt);
    // descriptors built once; a K step moves only the 14-bit start field
    // (addresses stay below 256 KB, so the field never carries).  Thread 0
    // issues every MMA while the CTA waits at its next barrier: rebuilding
    // both descriptors per MMA cost 0.6-1.1 % of the kernel
    const uint64_t da = smem_desc(a, 2048, 128), db = smem_desc(b, 128, sbo);
    const uint64_t dbs = smem_desc(b + (uint32_t)(half >> 3) * sbo, 128, sbo);
    const uint64_t sa = kDescStepA >> 4, sb = kDescStepB >> 4;
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + s * sa, db + s * sb, id_full, s > 0 ? 1u : 0u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + (ksteps + s) * sa, dbs + s * sb, id_neg, 1u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d + half, da + (ksteps + s) * sa, db + s * sb, id_half, 1u);
}

// The same complex GEMM with C and S at separate places (bc, bs; N = half
// columns each): Re x C, Re x S, then -Im x S, Im x C.
template <class E>
__device__ __forceinline__ void issue_cgemm_cs(uint32_t tmem_d, uint32_t a, uint32_t bc, uint32_t bs, int half,
                                               int ksteps, uint32_t sbo)
{
    const uint32_t id_neg = idesc_f16(128, half, true, true, E::fmt);
    const uint32_t id_half = idesc_f16(128, half, true, false, E::fmt);
    const uint64_t da = smem_desc(a, 2048, 128), dc = smem_desc(bc, 128, sbo), ds = smem_desc(bs, 128, sbo);
    const uint64_t sa = kDescStepA >> 4, sb = kDescStepB >> 4;
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + s * sa, dc + s * sb, id_half, s > 0 ? 1u : 0u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d + half, da + s * sa, ds + s * sb, id_half, s > 0 ? 1u : 0u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + (ksteps + s) * sa, ds + s * sb, id_neg, 1u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d + half, da + (ksteps + s) * sa, dc + s * sb, id_half, 1u);
}

// GEMM 1 of a step (operand buffer at a), committed to bar
// Re x T + Im x T' into n columns at tmem_d: the data (K = 2 x ksteps of
// 16, Re then Im, MN-major at a) against the paired tables T at b and T' at
// bn (N = n, K-major, N-group stride sbo).  Half the MMAs of issue_cgemm's
// three passes, each of full width.
template <class E>
__device__ __forceinline__ void issue_paired(uint32_t tmem_d, uint32_t a, uint32_t b, uint32_t bn, int n, int ksteps,
                                             uint32_t sbo)
{
    const uint32_t id = idesc_f16(128, n, true, false, E::fmt);
    const uint64_t da = smem_desc(a, 2048, 128), db = smem_desc(b, 128, sbo), dn = smem_desc(bn, 128, sbo);
    const uint64_t sa = kDescStepA >> 4, sb = kDescStepB >> 4;
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + s * sa, db + s * sb, id, s > 0 ? 1u : 0u);
    for (int s = 0; s < ksteps; ++s)
        mma_f16(tmem_d, da + (ksteps + s) * sa, dn + s * sb, id, 1u);
}

template <class E, int LOG2N>
__device__ __forceinline__ void issue_gemm1(uint32_t tmem, uint32_t s0, uint32_t a, uint32_t bar)
{
    using S = TcShape<LOG2N>;
    if constexpr (S::PAIRED)
        issue_paired<E>(tmem, a, s0 + S::SMEM_B1, s0 + S::SMEM_B1N, 2 * S::N2, S::N2 / 16, S::SBO_B1);
    else
        issue_cgemm<E>(tmem, a, s0 + S::SMEM_B1, S::N2, S::N2 / 16, S::SBO_B1);
    mma_commit(bar);
}

// GEMM 2 of a step: one GEMM for both blocks at N = 4096 (rows 64 b + m2),
// one per block at N = 8192 (block b's operand 32 KB on, its result 64
// columns on), one for the block at N = 16384 (K = 128 k1, its C and S
// columns of B1), committed to bar
template <class E, int LOG2N>
__device__ __forceinline__ void issue_gemm2(uint32_t tmem, uint32_t s0, uint32_t a, uint32_t bar)
{
    using S = TcShape<LOG2N>;
    if constexpr (S::N1 == 128) {
        issue_cgemm_cs<E>(tmem + S::D2_COL, a, s0 + S::SMEM_B1 + 8 * S::SBO_B1, s0 + S::SMEM_B1 + 24 * S::SBO_B1,
                          S::D2_HALF, S::N1 / 16, S::SBO_B1);
    } else if constexpr (S::PAIRED) {
        // [C_hi | S_hi] and [-S_hi | C_hi]: the tables' columns 64..127.  The
        // three-pass forms of both GEMMs issued 24 MMAs per pair instead of
        // 16; thread 0's issue is on the CTA's critical path, and the kernel
        // ran 4 % slower (19.05 vs 18.63 ms per 2^24 samples x 256 trials)
        issue_paired<E>(tmem + S::D2_COL, a, s0 + S::SMEM_B1 + 8 * S::SBO_B1, s0 + S::SMEM_B1N + 8 * S::SBO_B1, 64, 4,
                        S::SBO_B1);
    } else if constexpr (S::B2N_BYTES != 0) {
        // N = 8192: each block's GEMM 2 as Re x B2 + Im x B2N (16 MMAs per
        // pair instead of 24: 2 % faster, bit-identical)
        issue_paired<E>(tmem + S::D2_COL, a, s0 + S::SMEM_B2, s0 + S::SMEM_B2N, 64, 4, 1024);
        issue_paired<E>(tmem + S::D2_COL + 64, a + 32768, s0 + S::SMEM_B2, s0 + S::SMEM_B2N, 64, 4, 1024);
    } else {
        issue_cgemm<E>(tmem + S::D2_COL, a, s0 + S::SMEM_B2, 32, 4, 1024);
        if constexpr (S::N2 == 128)
            issue_cgemm<E>(tmem + S::D2_COL + 64, a + 32768, s0 + S::SMEM_B2, 32, 4, 1024);
    }
    mma_commit(bar);
}

// Thread 0 waits for a commit (bounded); every thread learns the outcome.
// Returns false (uniformly) on a timeout; parity then still names the
// phase waited for.
__device__ __forceinline__ bool wait_gemm(int tid, uint32_t bar, uint32_t &parity,
                                          unsigned long long limit_ns = kWaitLimitNs)
{
    bool ok = true;
    if (tid == 0)
        ok = mbar_wait(bar, parity, limit_ns);
    const bool failed = __syncthreads_or(!ok);
    if (!failed)
        parity ^= 1;
    tc_fence_after();
    return !failed;
}

// 2^e with 2^e * mx < 2^X, and its inverse (exponent arithmetic, exact)
template <int X>
__device__ __forceinline__ void pow2_scale_to(float mx, float &s, float &inv)
{
    int e = (__float_as_int(mx) >> 23) & 0xFF;
    e = min(max(e, X), 254);
    s = __int_as_float((X + 253 - e) << 23);
    inv = __int_as_float((e - X + 1) << 23);
}

// The arguments of a work item: the launch's own (one handle), or handle o's
// from the batch's parameter table.
template <bool MULTI, class B>
__device__ __forceinline__ const DedispArgs &item_args(const DedispArgs &a0, const B &bt, int o)
{
    if constexpr (MULTI)
        return bt.args[o];
    else
        return a0;
}

template <int LOG2N, class E, bool SERIES, bool FOLD, bool MULTI>
__global__ void __launch_bounds__(TcShape<LOG2N>::THREADS, TcShape<LOG2N>::CTAS_PER_SM)
    tc_dedisp_kernel(const __grid_constant__ DedispArgs a0,
                     const __grid_constant__ std::conditional_t<MULTI, BatchArgs, NoBatch> bt)
{
    using S = TcShape<LOG2N>;
    constexpr int N = S::N, M = S::M, N1 = S::N1, N2 = S::N2, W = S::WARPS, T = S::THREADS, BPS = S::BPS;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t s0 = smem_addr(sm);
    const uint32_t barA = s0 + S::SMEM_CTL, barB = s0 + S::SMEM_CTL + 8;
    FoldSmem fw;
    if constexpr (FOLD && !MULTI)
        fold_smem_layout(fw, sm + S::SMEM_FOLD, a0.fold);
    fill_constants<E, LOG2N>(sm, tid);
    const uint32_t tmem = tc_setup<LOG2N>(sm, s0, tid, warp);
    // epilogue view: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its GEMM
    // rows) and column group g = w / 4
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t tD1 = tmem + lane_base, tD2 = tmem + lane_base + S::D2_COL;
    const int g = warp >> 2;
    const int row = 32 * (warp & 3) + lane;
    const int rb = N1 == 128 ? 0 : row >> 6, ri = row & (N1 - 1);  // GEMM 1 row: block of the step, k1
    // GEMM 2 rows: N = 4096 -> (block rb, m2 = ri); N = 8192 -> (block g % 2,
    // m2 = row); N = 16384 -> (the step's one block, m2 = row)
    const int ob = N2 == 64 ? rb : (BPS == 2 ? (g & 1) : 0);
    const int om2 = N2 == 64 ? ri : row;
    const int oh = N2 == 64 || BPS == 1 ? g : (g >> 1);  // output columns c = 16 oh .. 16 oh + 15
    const uint32_t tD2b = tD2 + (N2 == 64 ? 0u : 64u * (uint32_t)ob);
    // this thread's twiddles e^{+2 pi i ri m2 / N}, m2 = 32 g + i, as 16-bit
    // pairs (m2, m2 + 1) matching the operand packing
    typename E::h2 twr[16], twi[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        float s0f, c0f, s1f, c1f;
        const int m2 = 32 * g + 2 * i;
        sincospif((float)((ri * m2) & (N - 1)) * (2.0f / N), &s0f, &c0f);
        sincospif((float)((ri * (m2 + 1)) & (N - 1)) * (2.0f / N), &s1f, &c1f);
        twr[i] = E::pack(c0f, c1f);
        twi[i] = E::pack(s0f, s1f);
    }
    // At N = 16384, and in the batch kernel, the twiddles wait in this
    // thread's tensor-memory lane (columns past D2, 32 per column group g)
    // and are read with D1 in each twiddle pass: the 32 registers go to the
    // gather, which at 16384 also holds the filter values it reads each step
    // (29.3 vs 33.4 ms per 2^24 samples x 256 trials), and in the batch
    // kernel to the parameter-table reads (spills 20/20 instead of 152/272
    // bytes; 1-3 % faster).  In the one-handle kernel at 4096 and 8192 the
    // extra tensor-memory read in the twiddle pass cost 8-11 %.
    constexpr bool kTwInTmem = LOG2N == 14 || MULTI;
    const uint32_t tTW = tmem + lane_base + (uint32_t)(S::TW_COL + 32 * g);
    if constexpr (kTwInTmem) {
        uint32_t v[32];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            v[i] = *reinterpret_cast<const uint32_t *>(&twr[i]);
            v[16 + i] = *reinterpret_cast<const uint32_t *>(&twi[i]);
        }
        tmem_st_32(tTW, v);
    }

    uint32_t phA = 0, phB = 0;
    bool pendA = false, pendB = false;  // a commit not yet waited for
    bool failed = false;
    int *status = nullptr;  // batch: the status word of the item that timed out
    // Work item w of one handle: trial w % D, block range w / D.  False
    // after a timed-out wait.
    // Work items: with one handle, trial w % D, block range w / D of a0, w
    // strided over the grid; in a batch, the next item of any handle from the
    // counter, its arguments read from the batch's parameter table.  The
    // item body is written once, inside the loop (as a lambda it cost
    // registers and time).
    __shared__ int swork[2];  // batch only
    const int items0 = MULTI ? 0 : a0.D * a0.R;
    for (int it = 0; !failed; ++it) {
        int w, o = 0;
        if constexpr (!MULTI) {
            w = blockIdx.x + it * gridDim.x;
            if (w >= items0)
                break;
        } else {
            __syncthreads();  // every reader of swork is done
            if (tid == 0) {
                const int gw = atomicAdd(bt.counter, 1);
                int ob_ = -1;
                if (gw < bt.prefix[bt.nobs]) {
                    int lo = 0, hi = bt.nobs - 1;  // last o with prefix[o] <= gw
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (bt.prefix[mid] <= gw)
                            lo = mid;
                        else
                            hi = mid - 1;
                    }
                    ob_ = lo;
                }
                swork[0] = ob_ < 0 ? -1 : gw - bt.prefix[ob_];
                swork[1] = ob_;
            }
            __syncthreads();
            // warp-uniform by construction (lane 0's copy)
            o = __shfl_sync(0xffffffffu, swork[1], 0);
            if (o < 0)
                break;
            w = __shfl_sync(0xffffffffu, swork[0], 0);
        }
        const DedispArgs &a = item_args<MULTI>(a0, bt, o);
        if constexpr (MULTI) {
            status = a.status;
            if constexpr (FOLD)
                fold_smem_layout(fw, sm + S::SMEM_FOLD, a.fold);
        }
        const float4 *__restrict__ ring4 = reinterpret_cast<const float4 *>(a.ring);
        const float2 *__restrict__ ring2 = a.ring;
        const int nunits = (a.count + BPS - 1) >> (BPS - 1);  // steps of the whole call
        const unsigned long long wlim = (unsigned long long)a.wait_limit_ns;
        const int smask = a.S - 1;
        const int dm = w % a.D;
        const int rr = w / a.D;
        const int kb = BPS * (int)((long long)nunits * rr / a.R);
        const int ke = min(a.count, BPS * (int)((long long)nunits * (rr + 1) / a.R));
        const int np = (ke - kb + BPS - 1) >> (BPS - 1);
        // this thread's bin pairs: delays, fixed for the trial (one row half at
        // 4096 and 8192, both at 16384), and at 4096 and 8192 the filter values
        // too (at 16384 they would take 64 registers: read with each step)
        constexpr int NH = 2 / BPS;
        const float4 *__restrict__ H4 = reinterpret_cast<const float4 *>(a.H + (size_t)dm * N);
        float4 hreg[BPS == 2 ? 8 : 1];
        uint32_t dd[8 * NH];
        {
            const uint32_t *__restrict__ dl2 = reinterpret_cast<const uint32_t *>(a.delays + (size_t)dm * N);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
#pragma unroll
                for (int h = 0; h < NH; ++h)
                    dd[NH * j + h] = __ldg(dl2 + h * (N / 4) + (j * W + warp) * 32 + lane);
                if constexpr (BPS == 2)
                    hreg[j] = __ldg(H4 + (j * W + warp) * 32 + lane);
            }
        }
        // power-of-two scale of the work item: |Z| <= 2 max|X| max|H| over
        // every ring row its blocks read (rows k0 + kb - largest delay .. k0 + ke - 1)
        float sc, isc;
        {
            float wm = 0.f;
            const long long r_hi = a.k0 + ke - 1;
            for (long long r = a.k0 + kb - __ldg(a.delay_max + dm) + tid; r <= r_hi; r += T)
                if (r >= 0)
                    wm = fmaxf(wm, a.row_max[r & smask]);
            wm = warp_max(wm);
            float *wmax = reinterpret_cast<float *>(sm + S::SMEM_CTL + 32);
            if (lane == 0)
                wmax[warp] = wm;
            __syncthreads();
#pragma unroll
            for (int i = 0; i < W; ++i)
                wm = fmaxf(wm, wmax[i]);
            pow2_scale_to<S::SCALE_EXP>(2.0f * wm * __ldg(a.h_max + dm), sc, isc);
            if constexpr (BPS == 2) {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    hreg[j] = make_float4(hreg[j].x * sc, hreg[j].y * sc, hreg[j].z * sc, hreg[j].w * sc);
            }
        }
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

        // Gather step i of the item into operand buffer `op`: Z = X[kg + b -
        // delay][bin] * H[bin] * sc, element (row 64 b + k1, k = k2) of the
        // MN-major operand for blocks k, k + 1 (4096, 8192), element (row
        // 64 h + k1 mod 64, k = k2) for row half h of block k (16384); Im
        // parts N2 K-columns on.
        auto gather = [&](int i, unsigned char *op) {
            const int k = kb + BPS * i;
            const bool two = BPS == 2 && k + 1 < ke;
            const long long kg = a.k0 + k;
            const int slot0 = (int)(kg & smask);
            // the scaled product of a bin pair, stored as row-pair words of
            // core-matrix row group 8 b + j
            auto put = [&](int j, int b, const float4 &x, const float4 &hv, float f) {
                const float zr0 = (x.x * hv.x - x.y * hv.y) * f, zi0 = (x.x * hv.y + x.y * hv.x) * f;
                const float zr1 = (x.z * hv.z - x.w * hv.w) * f, zi1 = (x.z * hv.w + x.w * hv.z) * f;
                const int off = (b * 8 + j) * 128 + warp * 2048 + (lane >> 2) * 16 + (lane & 3) * 4;
                *reinterpret_cast<uint32_t *>(op + off) = pack2<E>(zr0, zr1);
                *reinterpret_cast<uint32_t *>(op + off + S::IM_OFF) = pack2<E>(zi0, zi1);
            };
            if constexpr (BPS == 1) {
                if (kg >= a.max_delay) {
                    // as the pair gather below, over the two row halves of
                    // one block in turn, with the filter read alongside the
                    // ring (both halves' loads in flight at once took 7 %
                    // longer, 21 % with the twiddles in registers)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        float4 xa[8], hv[8];
                        float2 xb[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const int q = h * (N / 4) + (j * W + warp) * 32 + lane;
                            const uint32_t d = dd[2 * j + h];
                            const int r0 = (slot0 - (int)(d & 0xFFFFu)) & smask;
                            const int r1 = (slot0 - (int)(d >> 16)) & smask;
                            xa[j] = ring4[(size_t)r0 * (N / 2) + q];
                            xb[j] = r1 != r0 ? ring2[(size_t)r1 * N + 2 * q + 1] : make_float2(0.f, 0.f);
                            hv[j] = __ldg(H4 + q);
                        }
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const uint32_t d = dd[2 * j + h];
                            const bool split = (d & 0xFFFFu) != (d >> 16);
                            const float4 x = split ? make_float4(xa[j].x, xa[j].y, xb[j].x, xb[j].y) : xa[j];
                            put(j, h, x, hv[j], sc);
                        }
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int q = h * (N / 4) + (j * W + warp) * 32 + lane;
                            const uint32_t d = dd[2 * j + h];
                            const int d0 = (int)(d & 0xFFFFu), d1 = (int)(d >> 16);
                            float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                            // blocks before the stream start are zero
                            if (kg >= d0) {
                                const float2 t = ring2[(size_t)((slot0 - d0) & smask) * N + 2 * q];
                                x.x = t.x;
                                x.y = t.y;
                            }
                            if (kg >= d1) {
                                const float2 t = ring2[(size_t)((slot0 - d1) & smask) * N + 2 * q + 1];
                                x.z = t.x;
                                x.w = t.y;
                            }
                            put(j, h, x, __ldg(H4 + q), sc);
                        }
                    }
                }
            } else if (kg >= a.max_delay && two) {
                // every delayed block exists: no zero fill.  No branch on the
                // delays, so all loads of the pair issue before the first use:
                // each bin pair as one float4 from the first bin's row, and,
                // where the second bin's delay differs, that bin again from
                // its own row (a predicated load)
                float4 xa[8][2];
                float2 xb[8][2];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int q = (j * W + warp) * 32 + lane;  // float4 (bin pair) index in a row
                    const int r0 = (slot0 - (int)(dd[j] & 0xFFFFu)) & smask;
                    const int r1 = (slot0 - (int)(dd[j] >> 16)) & smask;
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        xa[j][b] = ring4[(size_t)((r0 + b) & smask) * (N / 2) + q];
                        xb[j][b] = r1 != r0 ? ring2[(size_t)((r1 + b) & smask) * N + 2 * q + 1]
                                            : make_float2(0.f, 0.f);
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 hv = hreg[j];
                    const bool split = (dd[j] & 0xFFFFu) != (dd[j] >> 16);
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const float4 x = split ? make_float4(xa[j][b].x, xa[j][b].y, xb[j][b].x, xb[j][b].y)
                                               : xa[j][b];
                        const float zr0 = x.x * hv.x - x.y * hv.y, zi0 = x.x * hv.y + x.y * hv.x;
                        const float zr1 = x.z * hv.z - x.w * hv.w, zi1 = x.z * hv.w + x.w * hv.z;
                        const int off = (b * 8 + j) * 128 + warp * 2048 + (lane >> 2) * 16 + (lane & 3) * 4;
                        *reinterpret_cast<uint32_t *>(op + off) = pack2<E>(zr0, zr1);
                        *reinterpret_cast<uint32_t *>(op + off + S::IM_OFF) = pack2<E>(zi0, zi1);
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int q = (j * W + warp) * 32 + lane;
                    const float4 hv = hreg[j];
                    const int d0 = (int)(dd[j] & 0xFFFFu), d1 = (int)(dd[j] >> 16);
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (b == 0 || two) {
                            const long long kk = kg + b;
                            // blocks before the stream start are zero
                            if (kk >= d0) {
                                const float2 t = ring2[(size_t)((slot0 + b - d0) & smask) * N + 2 * q];
                                x.x = t.x;
                                x.y = t.y;
                            }
                            if (kk >= d1) {
                                const float2 t = ring2[(size_t)((slot0 + b - d1) & smask) * N + 2 * q + 1];
                                x.z = t.x;
                                x.w = t.y;
                            }
                        }
                        const float zr0 = x.x * hv.x - x.y * hv.y, zi0 = x.x * hv.y + x.y * hv.x;
                        const float zr1 = x.z * hv.z - x.w * hv.w, zi1 = x.z * hv.w + x.w * hv.z;
                        const int off = (b * 8 + j) * 128 + warp * 2048 + (lane >> 2) * 16 + (lane & 3) * 4;
                        *reinterpret_cast<uint32_t *>(op + off) = pack2<E>(zr0, zr1);
                        *reinterpret_cast<uint32_t *>(op + off + S::IM_OFF) = pack2<E>(zi0, zi1);
                    }
                }
            }
        };

        // D1 -> twiddle (16-bit arithmetic) -> 16-bit operand of GEMM 2 in
        // `op`: rows (N = 4096: 64 rb +) m2, m2 = 32 g + 16 p + 8 q + 0..7;
        // k = k1 (Re), N1 + k1 (Im); at N = 8192 block rb's operand 32 KB on
        auto twiddle = [&](unsigned char *op) {
            unsigned char *opb = op + (N2 == 64 ? 0 : 32768 * rb);
            const int rg0 = N2 == 64 ? 8 * rb : 0;  // row group of m2 = 0
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                float re[16], im[16];
                uint32_t w8r[8], w8i[8];
                // D1 columns of m2 = 32 g + 16 p + 0..15: Re and Im N2 apart,
                // or with the paired tables 32 apart within quarters 2 g, 2 g + 1
                const uint32_t cre = S::PAIRED ? 64 * g + 16 * p : 32 * g + 16 * p;
                const uint32_t cim = S::PAIRED ? 64 * g + 32 + 16 * p : N2 + 32 * g + 16 * p;
                if constexpr (kTwInTmem)
                    tmem_ld_twiddle(tD1 + cre, tD1 + cim, tTW + 8 * p, tTW + 16 + 8 * p, re, im, w8r, w8i);
                else
                    tmem_ld_2x16(tD1 + cre, tD1 + cim, re, im);
                uint32_t pr[8], pim[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const typename E::h2 ar = E::pack(re[2 * i], re[2 * i + 1]);
                    const typename E::h2 ai = E::pack(im[2 * i], im[2 * i + 1]);
                    const typename E::h2 wr =
                        kTwInTmem ? *reinterpret_cast<const typename E::h2 *>(&w8r[i]) : twr[8 * p + i];
                    const typename E::h2 wi =
                        kTwInTmem ? *reinterpret_cast<const typename E::h2 *>(&w8i[i]) : twi[8 * p + i];
                    const typename E::h2 orr = __hfma2(ar, wr, __hneg2(__hmul2(ai, wi)));
                    const typename E::h2 oi = __hfma2(ar, wi, __hmul2(ai, wr));
                    pr[i] = *reinterpret_cast<const uint32_t *>(&orr);
                    pim[i] = *reinterpret_cast<const uint32_t *>(&oi);
                }
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int off = (rg0 + 4 * g + 2 * p + q) * 128 + (ri >> 3) * 2048 + (ri & 7) * 16;
                    st_shared_v4(opb + off, pr[4 * q], pr[4 * q + 1], pr[4 * q + 2], pr[4 * q + 3]);
                    st_shared_v4(opb + off + S::IM2_OFF, pim[4 * q], pim[4 * q + 1], pim[4 * q + 2], pim[4 * q + 3]);
                }
            }
        };

        // D2 -> outputs m = M + N2 c + m2 (c = 16 oh + u) of step i: series,
        // detection into the intensity buffers (M floats per block, in `op`)
        auto outputs = [&](int i, unsigned char *op) {
            const int k = kb + BPS * i;
            float yr[16], yi[16];
            tmem_ld_2x16(tD2b + 16 * oh, tD2b + S::D2_HALF + 16 * oh, yr, yi);
            if constexpr (SERIES) {
                if (ob == 0 || k + 1 < ke) {
                    float2 *out = a.series + (size_t)dm * a.count * M + (size_t)(k + ob) * M + 16 * N2 * oh + om2;
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        out[N2 * u] = make_float2(yr[u] * isc, yi[u] * isc);
                }
            }
            if constexpr (FOLD) {
                // detected in the item's scale; its partial profiles are
                // rescaled once at the end of the item (the scale is a power
                // of two, fixed for the item)
                // sample t = t0 + N2 u at iswz(t) (kIbufSwizzled): adding
                // N2 u = 128 u leaves the swizzle bits alone; adding 64 u
                // flips their upper bit with u's parity
                float *ib = reinterpret_cast<float *>(op);
                const int t0 = ob * M + 16 * N2 * oh + om2;
                const int e0 = iswz(t0), e1 = N2 == 64 ? iswz(t0 + 64) - 64 : e0;
                if (a.fold.detect) {
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        ib[((u & 1) ? e1 : e0) + N2 * u] = sqrtf(yr[u] * yr[u] + yi[u] * yi[u]);
                } else {
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        ib[((u & 1) ? e1 : e0) + N2 * u] = yr[u] * yr[u] + yi[u] * yi[u];
                }
            }
        };

        if (np > 0) {
            // prologue: pair 0 through GEMM 2's issue
            unsigned char *opb = sm + S::SMEM_OP0;
            gather(0, opb);
            fence_proxy_async();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                issue_gemm1<E, LOG2N>(tmem, s0, s0 + S::SMEM_OP0, barA);
            }
            pendA = true;
            failed = !wait_gemm(tid, barA, phA, wlim);
            if (!failed) {
                pendA = false;
                twiddle(opb);
                fence_proxy_async();
                tc_fence_before();
                __syncthreads();
                if (tid == 0) {
                    tc_fence_after();
                    issue_gemm2<E, LOG2N>(tmem, s0, s0 + S::SMEM_OP0, barB);
                }
                pendB = true;
            }
            for (int i = 0; i < np && !failed; ++i) {
                const uint32_t cur = (i & 1) ? S::SMEM_OP1 : S::SMEM_OP0, nxt = (i & 1) ? S::SMEM_OP0 : S::SMEM_OP1;
                const bool more = i + 1 < np;
                if (more) {
                    // pair i + 1 into the other buffer; its GEMM 1 overlaps
                    // pair i's outputs and fold
                    gather(i + 1, sm + nxt);
                    fence_proxy_async();
                    __syncthreads();
                    if (tid == 0) {
                        tc_fence_after();
                        issue_gemm1<E, LOG2N>(tmem, s0, s0 + nxt, barA);
                    }
                    pendA = true;
                }
                if (!wait_gemm(tid, barB, phB, wlim)) {
                    failed = true;
                    break;
                }
                pendB = false;
                outputs(i, sm + cur);
                tc_fence_before();
                if constexpr (FOLD) {
                    // the step's intensities are contiguous: one pass when one
                    // period span holds them, else unit by unit (a unit: one
                    // block at 4096 and 8192, half of the block at 16384)
                    constexpr int FU = BPS == 2 ? M : M / 2;
                    const int k = kb + BPS * i;
                    const bool second = BPS == 1 || k + 1 < ke;
                    const float *ib0 = reinterpret_cast<const float *>(sm + cur);
                    __syncthreads();
                    if (!(second && fold_pair<kIbufSwizzled>(a.fold, fw, ib0, k * M, FU, sp, sbase, scnt))) {
                        fold_block<kIbufSwizzled>(a.fold, fw, ib0, k * M, FU, sp, sbase, scnt);
                        if (second) {
                            __syncthreads();
                            fold_block<kIbufSwizzled>(a.fold, fw, ib0 + FU, k * M + FU, FU, sp, sbase, scnt);
                        }
                    }
                }
                if (more) {
                    if (!wait_gemm(tid, barA, phA, wlim)) {
                        failed = true;
                        break;
                    }
                    pendA = false;
                    twiddle(sm + nxt);
                    fence_proxy_async();
                    tc_fence_before();
                    __syncthreads();
                    if (tid == 0) {
                        tc_fence_after();
                        issue_gemm2<E, LOG2N>(tmem, s0, s0 + nxt, barB);
                    }
                    pendB = true;
                }
            }
        }
        if (failed)
            break;
        if constexpr (FOLD) {
            __syncthreads();
            // the item's intensities were folded in its scale: |y|^2 carries
            // sc^2 (|y| carries sc); undo it on the item's partial rows
            const float back = a.fold.detect ? isc : isc * isc;
            float *gm = a.fold.part_main + (size_t)w * a.fold.nbins;
            float *gp = a.fold.part_pend + (size_t)w * a.fold.nbins;
            if (a.fold.smem_prof) {
                for (int i = tid; i < a.fold.nbins; i += blockDim.x) {
                    gm[i] = fw.prof_main[i] * back;
                    gp[i] = fw.prof_pend[i] * back;
                }
            } else {
                for (int i = tid; i < a.fold.nbins; i += blockDim.x) {
                    gm[i] *= back;
                    gp[i] *= back;
                }
            }
            __syncthreads();
        }
    }
    if (failed && tid == 0) {
        atomicExch(MULTI ? status : a0.status, 1);
        // the GEMMs still outstanding get the same time to finish
        if (pendA)
            mbar_wait(barA, phA, kWaitLimitNs);
        if (pendB)
            mbar_wait(barB, phB, kWaitLimitNs);
    }
    tc_teardown<LOG2N>(tmem, warp);
}

// One GEMM of the kernel on given data (layout check): A from a row-major
// 128 x K 16-bit matrix, B the kernel's constant operand, D read back
// through the kernel's tensor-memory view.  Step 1: GEMM 1 (K = 2 N2,
// 2 N2 columns), step 2: GEMM 2 (K = 2 N1, N1 columns).
template <int LOG2N>
__global__ void __launch_bounds__(kThreads, 1) tc_probe_kernel(int step, const uint16_t *A, float *D, int *status)
{
    using S = TcShape<LOG2N>;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t s0 = smem_addr(sm);
    const uint32_t bar = s0 + S::SMEM_CTL;
    const int kdim = step == 1 ? 2 * S::N2 : 2 * S::N1;
    fill_constants<F16, LOG2N>(sm, tid);
    for (int e = tid; e < 128 * kdim; e += blockDim.x) {
        const int r = e & 127, kk = e >> 7;
        *reinterpret_cast<uint16_t *>(sm + S::SMEM_OP0 + mn_off(r, kk)) = A[r * kdim + kk];
    }
    const uint32_t tmem = tc_setup<LOG2N>(sm, s0, tid, warp);
    const uint32_t tcol = step == 1 ? 0u : (uint32_t)S::D2_COL;
    if (tid == 0) {
        tc_fence_after();
        if (step == 1)
            issue_gemm1<F16, LOG2N>(tmem, s0, s0 + S::SMEM_OP0, bar);
        else
            issue_gemm2<F16, LOG2N>(tmem, s0, s0 + S::SMEM_OP0, bar);
    }
    uint32_t parity = 0;
    if (!wait_gemm(tid, bar, parity)) {
        if (tid == 0) {
            atomicExch(status, 1);
            mbar_wait(bar, 0, kWaitLimitNs);
        }
        tc_teardown<LOG2N>(tmem, warp);
        return;
    }
    const int ncol = step == 1 ? 2 * S::N2 : 2 * S::D2_HALF;
    const int row = 32 * (warp & 3) + lane, h = warp >> 2;
    const uint32_t base = tmem + tcol + ((uint32_t)(32 * (warp & 3)) << 16);
    // D column of TMEM column c: [Re | Im] of the output frequency; the paired
    // GEMM 1 leaves [Re_lo | Im_lo | Re_hi | Im_hi] (32 frequencies each)
    auto dcol = [&](int c) {
        if (!(S::PAIRED && step == 1))
            return c;
        return (((c >> 5) & 1) ? 64 : 0) + ((c >> 6) ? 32 : 0) + (c & 31);
    };
    for (int c0 = h * ncol / 2; c0 < (h + 1) * ncol / 2; c0 += 32) {
        float x[16], y[16];
        tmem_ld_2x16(base + c0, base + c0 + 16, x, y);
        for (int i = 0; i < 16; ++i) {
            D[row * ncol + dcol(c0 + i)] = x[i];
            D[row * ncol + dcol(c0 + 16 + i)] = y[i];
        }
    }
    tc_teardown<LOG2N>(tmem, warp);
}

__global__ void tc_permute_kernel(const float2 *__restrict__ in, float2 *__restrict__ out, long long n, int log2n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nmask = (1ll << log2n) - 1;
    if (i < n)
        out[(i & ~nmask) + tc_pos((int)(i & nmask), log2n)] = in[i];
}

template <int LOG2N, class E, bool SERIES, bool FOLD, bool MULTI>
auto tc_fn() { return tc_dedisp_kernel<LOG2N, E, SERIES, FOLD, MULTI>; }

template <int LOG2N, class E, bool MULTI, typename G>
auto tc_select_e(bool series, bool fold, G &&go)
{
    if (series && fold)
        return go(tc_fn<LOG2N, E, true, true, MULTI>());
    if (fold)
        return go(tc_fn<LOG2N, E, false, true, MULTI>());
    return go(tc_fn<LOG2N, E, true, false, MULTI>());
}

template <int LOG2N, bool MULTI = false, typename G>
auto tc_select_n(bool bf16, bool series, bool fold, G &&go)
{
    if (bf16)
        return tc_select_e<LOG2N, BF16, MULTI>(series, fold, go);
    return tc_select_e<LOG2N, F16, MULTI>(series, fold, go);
}

template <int LOG2N>
int tc_blocks_per_sm_t(bool bf16, bool series, bool fold, size_t extra_smem)
{
    using S = TcShape<LOG2N>;
    const size_t sm = (size_t)S::SMEM_FOLD + extra_smem;
    int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0, smem_block = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess)
        return 0;
    if (sm > (size_t)smem_block)
        return 0;
    return tc_select_n<LOG2N>(bf16, series, fold, [&](auto k) -> int {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k) != cudaSuccess)
            return 0;
        const int by_smem = smem_sm / (int)(sm + (size_t)reserved);
        const int regs_cta = ((fa.numRegs + 7) / 8) * 8 * S::THREADS;
        const int by_regs = regs_cta > 0 ? regs_sm / regs_cta : 0;
        return std::min(S::CTAS_PER_SM, std::min(by_smem, by_regs));
    });
}

template <int LOG2N, bool MULTI, class B>
cudaError_t launch_tc_t(bool bf16, bool series, bool fold, const DedispArgs &a, const B &b,
                        size_t fold_smem, int grid, cudaStream_t st)
{
    using S = TcShape<LOG2N>;
    const size_t sm = (size_t)S::SMEM_FOLD + (fold ? fold_smem : 0);
    // no more CTAs per SM than the tensor memory holds (shared memory decides)
    if (S::CTAS_PER_SM == 2 && sm * 3 <= 228u * 1024u)
        return cudaErrorInvalidConfiguration;
    if (S::CTAS_PER_SM == 1 && sm * 2 <= 228u * 1024u)
        return cudaErrorInvalidConfiguration;
    return tc_select_n<LOG2N, MULTI>(bf16, series, fold, [&](auto k) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess)
            return e;
        k<<<grid, S::THREADS, sm, st>>>(a, b);
        return cudaGetLastError();
    });
}

}  // namespace

bool tc_supported(int log2n) { return log2n >= kLog2NMin && log2n <= kLog2NMax; }

int tc_threads(int log2n) { return log2n == 12 ? TcShape<12>::THREADS : TcShape<13>::THREADS; }

int tc_blocks_per_step(int log2n) { return log2n == 14 ? TcShape<14>::BPS : TcShape<12>::BPS; }

size_t tc_smem_base(int log2n)
{
    return log2n == 14 ? TcShape<14>::SMEM_FOLD : (log2n == 13 ? TcShape<13>::SMEM_FOLD : TcShape<12>::SMEM_FOLD);
}

size_t tc_smem_limit()
{
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    return (size_t)v;
}

// Resident CTAs per SM from the shared-memory and register limits (the
// tensor memory allows two at N = 4096, one at N = 8192 and 16384); 0 when it
// does not fit.  The occupancy API is not used: it reports one CTA per SM for the
// 4096-point kernel where the hardware runs two.
int tc_blocks_per_sm(int log2n, bool bf16, bool series, bool fold, size_t extra_smem)
{
    if (log2n == 14)
        return tc_blocks_per_sm_t<14>(bf16, series, fold, extra_smem);
    if (log2n == 13)
        return tc_blocks_per_sm_t<13>(bf16, series, fold, extra_smem);
    return tc_blocks_per_sm_t<12>(bf16, series, fold, extra_smem);
}

cudaError_t launch_tc_dedisp(int log2n, bool bf16, bool series, bool fold, const DedispArgs &a, int grid,
                             cudaStream_t st)
{
    if (!a.status || !tc_supported(log2n))
        return cudaErrorInvalidValue;
    const NoBatch none{};
    const size_t fs = fold ? fold_smem_bytes(a.fold.nbins, a.fold.span_cap, a.fold.smem_prof != 0, tc_threads(log2n))
                           : 0;
    if (log2n == 14)
        return launch_tc_t<14, false>(bf16, series, fold, a, none, fs, grid, st);
    if (log2n == 13)
        return launch_tc_t<13, false>(bf16, series, fold, a, none, fs, grid, st);
    return launch_tc_t<12, false>(bf16, series, fold, a, none, fs, grid, st);
}

cudaError_t launch_tc_dedisp_batch(int log2n, bool bf16, bool series, bool fold, const BatchArgs &b,
                                   size_t fold_smem, int grid, cudaStream_t st)
{
    if (!b.counter || b.nobs < 1 || b.nobs > kBatchMax || !tc_supported(log2n))
        return cudaErrorInvalidValue;
    DedispArgs none{};
    if (log2n == 14)
        return launch_tc_t<14, true>(bf16, series, fold, none, b, fold_smem, grid, st);
    if (log2n == 13)
        return launch_tc_t<13, true>(bf16, series, fold, none, b, fold_smem, grid, st);
    return launch_tc_t<12, true>(bf16, series, fold, none, b, fold_smem, grid, st);
}

cudaError_t launch_tc_permute_rows(const float2 *in, float2 *out, int rows, int log2n, cudaStream_t st)
{
    const long long n = (long long)rows << log2n;
    tc_permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, out, n, log2n);
    return cudaGetLastError();
}

cudaError_t launch_tc_probe(int step, const uint16_t *a, float *d, int *status, cudaStream_t st)
{
    // steps 1, 2: the 4096-point GEMMs; step 3: the 8192-point GEMM 1 (also
    // the 16384-point GEMM 1); step 4: the 16384-point GEMM 2
    if (step < 1 || step > 4)
        return cudaErrorInvalidValue;
    auto run = [&](auto k, size_t sm, int st_) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess)
            return e;
        k<<<1, kThreads, sm, st>>>(st_, a, d, status);
        return cudaGetLastError();
    };
    if (step == 4)
        return run(tc_probe_kernel<14>, (size_t)TcShape<14>::SMEM_FOLD, 2);
    if (step == 3)
        return run(tc_probe_kernel<13>, (size_t)TcShape<13>::SMEM_FOLD, 1);
    return run(tc_probe_kernel<12>, (size_t)TcShape<12>::SMEM_FOLD, step);
}

}  // namespace msosm
