// tc_dedisp.cu -- tensor-core (tcgen05) variant of the fused dedispersion
// kernel for 4096-point transforms.
//
// Same semantics as dedisp_kernel (kernels.cu), which replaces
// ComplexMultiplyDelay_concurrent_batch + inverse cufftExecC2C +
// DiscardSamples_concurrent_batch (gpu/gpu_kernel.cu:128-198,236-258) and the
// host fold of Fold_GPU (folding/fold_gpu.cpp:48-194): per (trial, block)
// gather X[k - delay[b]][b] * H[b] from the spectrum ring, inverse transform,
// keep outputs m >= M, write the series and/or detect and fold.  Here the
// inverse transform of two consecutive blocks of one trial runs as two f16
// GEMMs with f32 accumulation in tensor memory (factorisation and layouts in
// tc_layout.hpp): GEMM 1 (M 128 = 2 blocks x 64 k1, N 128, K 128), a twiddle
// pass on the CUDA cores, GEMM 2 (M 128 = 2 blocks x 64 m2, N 64, K 128).
//
// Precision: the gathered products of a block pair are scaled by a power of
// two chosen so that no component can reach 2^8 -- from the largest
// component of every ring row the pair reads (recorded by the forward
// kernel) times the trial's largest filter component -- so every GEMM 1 sum
// stays below 2^15 and every twiddled value below 2^15.5, inside f16.  The
// twiddle multiply runs in f16 arithmetic on f16-rounded twiddles.  The
// scale is undone exactly on the f32 results.
//
// Waits on the tensor core are bounded (1 s of global timer): on a timeout
// the kernel records a nonzero status, waits once more for its last GEMM,
// frees its tensor memory and returns.
#include <algorithm>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "fold_dev.cuh"
#include "kernels.hpp"
#include "tc_layout.hpp"

namespace msosm {
namespace {

using namespace tc;

constexpr unsigned long long kWaitLimitNs = 1000000000ull;

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

// Waits for the phase of the given parity to complete; false after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns)
{
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

__device__ __forceinline__ uint32_t pack_half2(float lo, float hi)
{
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ void st_shared_v4(unsigned char *p, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    *reinterpret_cast<uint4 *>(p) = make_uint4(a, b, c, d);
}

// 2^e with 2^e * mx < 2^8, and its inverse (exponent arithmetic, exact)
__device__ __forceinline__ void pow2_scale(float mx, float &s, float &inv)
{
    int e = (__float_as_int(mx) >> 23) & 0xFF;
    e = min(max(e, 8), 254);
    s = __int_as_float((261 - e) << 23);
    inv = __int_as_float((e - 7) << 23);
}

__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The constant operands: the 64-point inverse DFT in real form.
//   GEMM 1, B1[n][kk]: n < 64 -> Re A[m2 = n], n >= 64 -> Im A[m2 = n - 64];
//     kk < 64 -> Re Z[k2 = kk], kk >= 64 -> Im Z[k2 = kk - 64]
//   GEMM 2, B2[n][kk]: n < 32 -> Re y[m1 = 32 + n], n >= 32 -> Im y[m1 = n];
//     kk < 64 -> Re A'[k1 = kk], kk >= 64 -> Im A'[k1 = kk - 64]
__device__ void fill_constants(unsigned char *sm, int tid)
{
    for (int e = tid; e < 128 * 128; e += kThreads) {
        const int n = e >> 7, kk = e & 127;
        const int k2 = kk & 63, m2 = n & 63;
        float s, c;
        sincospif((float)((k2 * m2) & 63) * (1.0f / 32.0f), &s, &c);
        const float v = kk < 64 ? (n < 64 ? c : s) : (n < 64 ? -s : c);
        *reinterpret_cast<__half *>(sm + kSmemBA + k_off(n, kk)) = __float2half_rn(v);
    }
    for (int e = tid; e < 64 * 128; e += kThreads) {
        const int n = e >> 7, kk = e & 127;
        const int k1 = kk & 63, m1 = 32 + (n & 31);
        float s, c;
        sincospif((float)((k1 * m1) & 63) * (1.0f / 32.0f), &s, &c);
        const float v = kk < 64 ? (n < 32 ? c : s) : (n < 32 ? -s : c);
        *reinterpret_cast<__half *>(sm + kSmemBC + k_off(n, kk)) = __float2half_rn(v);
    }
}

// mbarrier + tensor memory; every thread returns the TMEM base address
__device__ uint32_t tc_setup(unsigned char *sm, uint32_t s0, int tid, int warp)
{
    if (tid == 0) {
        mbar_init(s0 + kSmemCtl, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(s0 + kSmemCtl + 8, kTmemCols);
        tmem_relinquish();
    }
    fence_proxy_async();  // shared-memory operands written so far -> tensor core
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *reinterpret_cast<volatile uint32_t *>(sm + kSmemCtl + 8);
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem, int warp)
{
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// eight K = 16 steps of one GEMM, then the commit to the mbarrier
__device__ __forceinline__ void issue_gemm(uint32_t tmem_d, uint32_t a_addr, uint32_t b_addr, uint32_t idesc,
                                           uint32_t bar)
{
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const uint64_t da = smem_desc(a_addr + s * kDescStepA, 2048, 128);
        const uint64_t db = smem_desc(b_addr + s * kDescStepB, 128, 2048);
        mma_f16(tmem_d, da, db, idesc, s > 0 ? 1u : 0u);
    }
    mma_commit(bar);
}

template <bool SERIES, bool FOLD>
__global__ void __launch_bounds__(kThreads, 2) tc_dedisp_kernel(DedispArgs a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t s0 = smem_addr(sm);
    const uint32_t bar = s0 + kSmemCtl;
    unsigned char *op = sm + kSmemOp;
    float *ibuf0 = reinterpret_cast<float *>(sm + kSmemOp);
    float *ibuf1 = ibuf0 + ibuf_floats(kM);
    FoldSmem fw;
    if constexpr (FOLD) {
        fw.wa = reinterpret_cast<int *>(sm + kSmemFold);
        fw.wb = fw.wa + a.fold.span_cap;
        fw.wp = fw.wb + a.fold.span_cap;
        fw.wd = fw.wp + a.fold.span_cap;
        fw.prof_main = reinterpret_cast<float *>(fw.wd + a.fold.span_cap);
        fw.prof_pend = fw.prof_main + a.fold.nbins;
    }
    fill_constants(sm, tid);
    const uint32_t tmem = tc_setup(sm, s0, tid, warp);
    // epilogue view: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its GEMM
    // rows) and half h = w / 4 of the columns
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t tD1 = tmem + lane_base, tD2 = tmem + lane_base + 128;
    const int h = warp >> 2;
    const int row = 32 * (warp & 3) + lane;
    const int rb = row >> 6, ri = row & 63;  // block of the pair; k1 (GEMM 1) / m2 (GEMM 2)
    // this thread's twiddles e^{+2 pi i ri m2 / 4096}, m2 = 32 h + i, as f16
    // pairs (m2, m2 + 1) matching the operand packing
    __half2 twr[16], twi[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        float s0f, c0f, s1f, c1f;
        const int m2 = 32 * h + 2 * i;
        sincospif((float)((ri * m2) & 4095) * (1.0f / 2048.0f), &s0f, &c0f);
        sincospif((float)((ri * (m2 + 1)) & 4095) * (1.0f / 2048.0f), &s1f, &c1f);
        twr[i] = __floats2half2_rn(c0f, c1f);
        twi[i] = __floats2half2_rn(s0f, s1f);
    }

    const float4 *__restrict__ ring4 = reinterpret_cast<const float4 *>(a.ring);
    const float2 *__restrict__ ring2 = a.ring;
    const int items = a.D * a.R;
    const int npairs = (a.count + 1) >> 1;
    const int smask = a.S - 1;
    uint32_t phase = 0;
    bool failed = false;
    for (int w = blockIdx.x; w < items; w += gridDim.x) {
        const int dm = w % a.D;
        const int rr = w / a.D;
        const int kb = 2 * (int)((long long)npairs * rr / a.R);
        const int ke = min(a.count, 2 * (int)((long long)npairs * (rr + 1) / a.R));
        const float4 *__restrict__ H4 = reinterpret_cast<const float4 *>(a.H + (size_t)dm * kN);
        // this thread's bin-pair delays are fixed for the trial
        uint32_t dd[8];
        {
            const uint32_t *__restrict__ dl2 = reinterpret_cast<const uint32_t *>(a.delays + (size_t)dm * kN);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                dd[j] = __ldg(dl2 + (j * 8 + warp) * 32 + lane);
        }
        const float hmx = __ldg(a.h_max + dm);
        const int nrow = __ldg(a.delay_max + dm) + 2;
        int sp = 0, sbase = 0, scnt = 0;
        if constexpr (FOLD) {
            if (a.fold.smem_prof) {
                for (int i = tid; i < 2 * a.fold.nbins; i += blockDim.x)
                    fw.prof_main[i] = 0.f;
            } else {
                fw.prof_main = a.fold.part_main + (size_t)w * a.fold.nbins;
                fw.prof_pend = a.fold.part_pend + (size_t)w * a.fold.nbins;
            }
            sp = span_lower_bound(a.fold.span_b, a.fold.nspans, (long long)kb * kM);
            span_refill(a.fold, fw, sp, sbase, scnt);
        }
        for (int k = kb; k < ke; k += 2) {
            const bool two = k + 1 < ke;
            const long long kg = a.k0 + k;
            const bool warm = kg >= a.max_delay;
            const int slot0 = (int)(kg & smask);
            // ---- power-of-two scale of the pair: |Z| <= 2 max|X| max|H| over
            // the ring rows kg + 1 - j (j <= largest delay + 1) it reads
            float wm = 0.f;
            for (int j = lane; j < nrow; j += 32) {
                const long long r = kg + 1 - j;
                if (r >= 0 && (j > 0 || two))
                    wm = fmaxf(wm, a.row_max[r & smask]);
            }
            wm = warp_max(wm);
            float sc, isc;
            pow2_scale(2.0f * wm * hmx, sc, isc);
            // ---- gather Z = X[kg + b - delay][bin] * H[bin] * sc of both
            // blocks into the f16 operand of GEMM 1
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int q = (j * 8 + warp) * 32 + lane;  // float4 (bin pair) index in a row
                float4 hv = __ldg(H4 + q);
                hv.x *= sc;
                hv.y *= sc;
                hv.z *= sc;
                hv.w *= sc;
                const int d0 = (int)(dd[j] & 0xFFFFu), d1 = (int)(dd[j] >> 16);
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (b == 0 || two) {
                        const long long kk = kg + b;
                        if (d0 == d1) {
                            if (warm || kk >= d0)  // blocks before the stream start are zero
                                x = ring4[(size_t)((slot0 + b - d0) & smask) * (kN / 2) + q];
                        } else {
                            if (warm || kk >= d0) {
                                const float2 t = ring2[(size_t)((slot0 + b - d0) & smask) * kN + 2 * q];
                                x.x = t.x;
                                x.y = t.y;
                            }
                            if (warm || kk >= d1) {
                                const float2 t = ring2[(size_t)((slot0 + b - d1) & smask) * kN + 2 * q + 1];
                                x.z = t.x;
                                x.w = t.y;
                            }
                        }
                    }
                    const float zr0 = x.x * hv.x - x.y * hv.y, zi0 = x.x * hv.y + x.y * hv.x;
                    const float zr1 = x.z * hv.z - x.w * hv.w, zi1 = x.z * hv.w + x.w * hv.z;
                    // element (row 64 b + k1, k = k2) of the MN-major operand
                    const int off = (b * 8 + j) * 128 + warp * 2048 + (lane >> 2) * 16 + (lane & 3) * 4;
                    *reinterpret_cast<uint32_t *>(op + off) = pack_half2(zr0, zr1);
                    *reinterpret_cast<uint32_t *>(op + off + 8 * 2048) = pack_half2(zi0, zi1);
                }
            }
            fence_proxy_async();
            __syncthreads();
            bool ok = true;
            if (tid == 0) {
                tc_fence_after();
                issue_gemm(tmem, s0 + kSmemOp, s0 + kSmemBA, kIdesc1, bar);
                ok = mbar_wait(bar, phase, kWaitLimitNs);
            }
            phase ^= 1;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            tc_fence_after();
            // ---- twiddle D1 (f16 arithmetic) into the f16 operand of GEMM 2
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                float re[16], im[16];
                tmem_ld_2x16(tD1 + 32 * h + 16 * p, tD1 + 64 + 32 * h + 16 * p, re, im);
                uint32_t pr[8], pim[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const __half2 ar = __floats2half2_rn(re[2 * i], re[2 * i + 1]);
                    const __half2 ai = __floats2half2_rn(im[2 * i], im[2 * i + 1]);
                    const __half2 wr = twr[8 * p + i], wi = twi[8 * p + i];
                    const __half2 orr = __hfma2(ar, wr, __hneg2(__hmul2(ai, wi)));
                    const __half2 oi = __hfma2(ar, wi, __hmul2(ai, wr));
                    pr[i] = *reinterpret_cast<const uint32_t *>(&orr);
                    pim[i] = *reinterpret_cast<const uint32_t *>(&oi);
                }
#pragma unroll
                for (int g = 0; g < 2; ++g) {
                    // rows 64 rb + m2 (m2 = 32 h + 16 p + 8 g + 0..7), k = k1 (Re), 64 + k1 (Im)
                    const int off = (rb * 8 + 4 * h + 2 * p + g) * 128 + (ri >> 3) * 2048 + (ri & 7) * 16;
                    st_shared_v4(op + off, pr[4 * g], pr[4 * g + 1], pr[4 * g + 2], pr[4 * g + 3]);
                    st_shared_v4(op + off + 8 * 2048, pim[4 * g], pim[4 * g + 1], pim[4 * g + 2], pim[4 * g + 3]);
                }
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            ok = true;
            if (tid == 0) {
                tc_fence_after();
                issue_gemm(tmem + 128, s0 + kSmemOp, s0 + kSmemBC, kIdesc2, bar);
                ok = mbar_wait(bar, phase, kWaitLimitNs);
            }
            phase ^= 1;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            tc_fence_after();
            // ---- outputs m = M + 64 c + m2 (c = 16 h + i): series, detection
            {
                float yr[16], yi[16];
                tmem_ld_2x16(tD2 + 16 * h, tD2 + 32 + 16 * h, yr, yi);
                float *ib = rb ? ibuf1 : ibuf0;
                const bool valid = rb == 0 || two;
                const float is2 = isc * isc;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int t = 64 * (16 * h + i) + ri;
                    if constexpr (SERIES) {
                        if (valid)
                            a.series[(size_t)dm * a.count * kM + (size_t)(k + rb) * kM + t] =
                                make_float2(yr[i] * isc, yi[i] * isc);
                    }
                    if constexpr (FOLD) {
                        const float pw = (yr[i] * yr[i] + yi[i] * yi[i]) * is2;
                        ib[ipad(t)] = a.fold.detect ? sqrtf(pw) : pw;
                    }
                }
            }
            tc_fence_before();
            if constexpr (FOLD) {
                __syncthreads();
                fold_block(a.fold, fw, ibuf0, k * kM, kM, sp, sbase, scnt);
                if (two) {
                    __syncthreads();
                    fold_block(a.fold, fw, ibuf1, (k + 1) * kM, kM, sp, sbase, scnt);
                }
                __syncthreads();  // fold reads done before the next gather overwrites them
            }
        }
        if (failed)
            break;
        if constexpr (FOLD) {
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
    if (failed && tid == 0) {
        atomicExch(a.status, 1);
        mbar_wait(bar, phase ^ 1, kWaitLimitNs);  // the GEMM the timed-out wait was for
    }
    tc_teardown(tmem, warp);
}

// One GEMM of the kernel on given data (layout check): A from a row-major
// 128 x 128 f16 matrix, B the kernel's constant operand, D read back through
// the kernel's tensor-memory view.
__global__ void __launch_bounds__(kThreads, 1) tc_probe_kernel(int step, const uint16_t *A, float *D, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t s0 = smem_addr(sm);
    const uint32_t bar = s0 + kSmemCtl;
    fill_constants(sm, tid);
    for (int e = tid; e < 128 * 128; e += kThreads) {
        const int r = e & 127, kk = e >> 7;
        *reinterpret_cast<uint16_t *>(sm + kSmemOp + mn_off(r, kk)) = A[r * 128 + kk];
    }
    const uint32_t tmem = tc_setup(sm, s0, tid, warp);
    const uint32_t tcol = step == 1 ? 0u : 128u;
    if (tid == 0) {
        tc_fence_after();
        issue_gemm(tmem + tcol, s0 + kSmemOp, s0 + (step == 1 ? kSmemBA : kSmemBC), step == 1 ? kIdesc1 : kIdesc2,
                   bar);
    }
    bool ok = mbar_wait(bar, 0, kWaitLimitNs);
    if (!ok && tid == 0)
        atomicExch(status, 1);
    if (__syncthreads_or(!ok)) {
        if (tid == 0)
            mbar_wait(bar, 0, kWaitLimitNs);
        tc_teardown(tmem, warp);
        return;
    }
    tc_fence_after();
    const int ncol = step == 1 ? 128 : 64;
    const int row = 32 * (warp & 3) + lane, h = warp >> 2;
    const uint32_t base = tmem + tcol + ((uint32_t)(32 * (warp & 3)) << 16);
    for (int c0 = h * ncol / 2; c0 < (h + 1) * ncol / 2; c0 += 32) {
        float x[16], y[16];
        tmem_ld_2x16(base + c0, base + c0 + 16, x, y);
        for (int i = 0; i < 16; ++i) {
            D[row * ncol + c0 + i] = x[i];
            D[row * ncol + c0 + 16 + i] = y[i];
        }
    }
    tc_teardown(tmem, warp);
}

__global__ void tc_permute_kernel(const float2 *__restrict__ in, float2 *__restrict__ out, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[(i & ~(long long)(kN - 1)) + tc_pos((int)(i & (kN - 1)))] = in[i];
}

template <bool SERIES, bool FOLD>
auto tc_fn() { return tc_dedisp_kernel<SERIES, FOLD>; }

template <typename G>
auto tc_select(bool series, bool fold, G &&go)
{
    if (series && fold)
        return go(tc_fn<true, true>());
    if (fold)
        return go(tc_fn<false, true>());
    return go(tc_fn<true, false>());
}

}  // namespace

bool tc_supported(int log2n) { return log2n == kLog2N; }

size_t tc_smem_bytes(size_t extra) { return (size_t)kSmemFold + extra; }

// Resident CTAs per SM from the shared-memory and register limits (at most
// two: each CTA holds 256 of the SM's 512 tensor-memory columns).  The
// occupancy API is not used here: it reports one CTA per SM for this kernel
// where the hardware runs two.
int tc_blocks_per_sm(bool series, bool fold, size_t extra_smem)
{
    const size_t sm = tc_smem_bytes(extra_smem);
    int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess)
        return 0;
    return tc_select(series, fold, [&](auto k) -> int {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k) != cudaSuccess)
            return 0;
        const int by_smem = smem_sm / (int)(sm + (size_t)reserved);
        const int regs_cta = ((fa.numRegs + 7) / 8) * 8 * kThreads;
        const int by_regs = regs_cta > 0 ? regs_sm / regs_cta : 0;
        return std::min(2, std::min(by_smem, by_regs));
    });
}

cudaError_t launch_tc_dedisp(bool series, bool fold, const DedispArgs &a, int grid, cudaStream_t st)
{
    if (!a.status)
        return cudaErrorInvalidValue;
    const size_t sm = tc_smem_bytes(fold ? fold_smem_bytes(a.fold.nbins, a.fold.span_cap, a.fold.smem_prof != 0) : 0);
    // at most two CTAs per SM (tensor memory: 256 of 512 columns each)
    if (sm * 3 <= 228u * 1024u)
        return cudaErrorInvalidConfiguration;
    return tc_select(series, fold, [&](auto k) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess)
            return e;
        k<<<grid, kThreads, sm, st>>>(a);
        return cudaGetLastError();
    });
}

cudaError_t launch_tc_permute_rows(const float2 *in, float2 *out, int rows, cudaStream_t st)
{
    const long long n = (long long)rows * kN;
    tc_permute_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_tc_probe(int step, const uint16_t *a, float *d, int *status, cudaStream_t st)
{
    if (step != 1 && step != 2)
        return cudaErrorInvalidValue;
    const size_t sm = kSmemFold;
    cudaError_t e = cudaFuncSetAttribute(tc_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess)
        return e;
    tc_probe_kernel<<<1, kThreads, sm, st>>>(step, a, d, status);
    return cudaGetLastError();
}

}  // namespace msosm
