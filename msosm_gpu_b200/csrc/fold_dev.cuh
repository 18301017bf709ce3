// fold_dev.cuh -- device side of the deterministic fold shared by the fused
// dedispersion kernels (CUDA-core and tensor-core) and the series fold.
#pragma once

#include "kernels.hpp"

namespace msosm {

// Folding inside the dedispersion kernel.  The host fold planner cuts each
// call's output samples into spans (one period each, sorted); a work item
// keeps a window of them in shared memory and its two partial profiles
// (complete periods, pending period) in shared memory too.  A block of 8
// samples per thread that lies inside one span, with at least 8 samples per
// output bin, takes the fast path: each thread sums its 8 consecutive
// samples into at most two bin partials, and a group of lanes per bin adds
// that bin's partials in thread order.  Other blocks go span piece by span
// piece: every bin is summed by a group of lanes strided over its samples.
// Either way the summation order is fixed, so the result does not depend on
// scheduling.
struct FoldSmem {
    float *prof_main, *prof_pend;  // [nbins] each (or the global rows)
    int *wa, *wb, *wp, *wd;        // span window (chunk-local sample indices < 2^31)
    float *pa;                     // [2][threads] per-thread bin partials of the fast path
};

// Shared-memory layout of the fold state at `base` (sized by fold_smem_bytes).
__device__ __forceinline__ void fold_smem_layout(FoldSmem &w, void *base, const FoldArgs &f)
{
    w.wa = reinterpret_cast<int *>(base);
    w.wb = w.wa + f.span_cap;
    w.wp = w.wb + f.span_cap;
    w.wd = w.wp + f.span_cap;
    w.pa = reinterpret_cast<float *>(w.wd + f.span_cap);
    w.prof_main = w.pa + 2 * blockDim.x;
    w.prof_pend = w.prof_main + f.nbins;
}

__device__ __forceinline__ int span_lower_bound(const long long *b, int n, long long t)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (b[mid] <= t)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Load spans [at, at + cap) into the window (all threads; barriers inside).
__device__ __forceinline__ void span_refill(const FoldArgs &f, FoldSmem &w, int at, int &base, int &cnt)
{
    __syncthreads();
    const int n = min(f.span_cap, f.nspans - at);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        w.wa[i] = (int)f.span_a[at + i];
        w.wb[i] = (int)f.span_b[at + i];
        w.wp[i] = f.span_phase0[at + i];
        w.wd[i] = f.span_dest[at + i];
    }
    base = at;
    cnt = n;
    __syncthreads();
}

// floor(x / bpt) for x >= 0 with x / bpt < 2^22 (at most nbins + 1; the host
// bounds nbins) from a float reciprocal, corrected to exact
__device__ __forceinline__ int div_bpt(int x, int bpt, float inv_bpt)
{
    if (bpt == 1)
        return x;
    int q = __float2int_rz((float)x * inv_bpt);
    if (q * bpt > x)
        --q;
    else if ((q + 1) * bpt <= x)
        ++q;
    return q;
}

// Layouts of the intensity buffer (sample t of the buffer at index ...):
//  kIbufPadded: t + t/32, one pad slot per 32 samples, so that threads
//    reading bins of any length one sample at a time hit different banks;
//  kIbufSwizzled: t with its 16-byte chunk index c = t/4 XORed with
//    (c/8) % 4: eight threads reading 16 (or 8) consecutive samples each as
//    128-bit loads touch eight different 16-byte bank groups (plain, every
//    second thread would meet the same group), and a warp storing 32
//    consecutive samples still fills one 128-byte row.  The swizzle moves
//    chunks only inside aligned 32-sample groups.
constexpr int kIbufPadded = 1, kIbufSwizzled = 2;
__device__ __forceinline__ int ipad(int t) { return t + (t >> 5); }
__device__ __forceinline__ int iswz(int t) { return t ^ (((t >> 5) & 3) << 2); }
template <int L>
__device__ __forceinline__ int iidx(int t) { return L == kIbufPadded ? ipad(t) : iswz(t); }

template <int L>
__device__ __forceinline__ void fold_piece(const FoldArgs &f, float *prof, const float *ibuf, int off,
                                           int ph_lo, int ph_hi)
{
    // sample of phase p sits at chunk-local block offset off + p.  Each bin is
    // summed by a group of G = 2^g_shift lanes (G ~ bpt/8, a power of two <= 32,
    // chosen on the host), lane l taking samples l, l+G, ...; the group then
    // reduces with a fixed xor butterfly.  G*bins ~ M/8 keeps every warp of
    // the block busy for any bin length, and the loop trip count is uniform
    // so whole warps shuffle.
    const int b_lo = div_bpt(ph_lo, f.bpt, f.inv_bpt);
    int b_hi = div_bpt(ph_hi - 1, f.bpt, f.inv_bpt);
    if (b_hi > f.nbins - 1)
        b_hi = f.nbins - 1;
    if (b_hi < b_lo)
        return;
    const int G = 1 << f.g_shift;
    const int g = (int)threadIdx.x >> f.g_shift, l = (int)threadIdx.x & (G - 1);
    const int ngroups = (int)blockDim.x >> f.g_shift;
    for (int first = b_lo; first <= b_hi; first += ngroups) {
        const int bin = first + g;
        float a0 = 0.f, a1 = 0.f;
        if (bin <= b_hi) {
            const int s0 = bin * f.bpt;
            const int s_lo = max(ph_lo, s0);
            const int s_hi = min(ph_hi, s0 + f.bpt);
            int p = s_lo + l;
            for (; p + G < s_hi; p += 2 * G) {
                a0 += ibuf[iidx<L>(off + p)];
                a1 += ibuf[iidx<L>(off + p + G)];
            }
            if (p < s_hi)
                a0 += ibuf[iidx<L>(off + p)];
        }
        float sum = a0 + a1;
        for (int o = G >> 1; o > 0; o >>= 1)
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (bin <= b_hi && l == 0)
            prof[bin] += sum;
    }
}

// Fast path of fold_block: the SPT * blockDim.x samples all lie in one span
// (phases ph_lo ..), bpt >= SPT, so a thread's SPT consecutive samples (8,
// or 16 for a pair of blocks) touch at most two bins.  Samples whose bin is
// past the last output bin are not folded (n_valid of them are).  Each
// thread sums its samples of its first bin (and of the next one); every bin
// is then completed by the thread holding its first sample (thread 0 for the
// bin running into the range), adding the following threads' first-bin sums
// in thread order.
template <int L, int SPT = 8>
__device__ __forceinline__ void fold_block_fast(const FoldArgs &f, FoldSmem &w, float *prof, const float *ibuf,
                                                int ph_lo, int n_valid)
{
    static_assert(SPT == 8 || (SPT == 16 && L == kIbufSwizzled), "8 samples per thread, or 16 from a swizzled buffer");
    const int tid = threadIdx.x, T = blockDim.x;
    const int bpt = f.bpt;
    const int j0 = SPT * tid;
    const int ph = ph_lo + j0;
    const int b0 = div_bpt(ph, bpt, f.inv_bpt);
    const int r0 = ph - b0 * bpt;  // place of the first sample in its bin
    const int n0 = bpt - r0;       // samples left in bin b0 (>= 1)
    const int nv = min(SPT, n_valid - j0);
    float x[SPT];
    if constexpr (L == kIbufPadded) {
#pragma unroll
        for (int u = 0; u < SPT; ++u)
            x[u] = ibuf[ipad(j0 + u)];
    } else {
        // chunks c = (SPT/4) tid + v, stored at c ^ ((c / 8) % 4)
        const int sw = ((SPT / 4) * tid >> 3) & 3;
#pragma unroll
        for (int v = 0; v < SPT / 4; ++v) {
            const float4 q = reinterpret_cast<const float4 *>(ibuf)[((SPT / 4) * tid + v) ^ sw];
            x[4 * v] = q.x;
            x[4 * v + 1] = q.y;
            x[4 * v + 2] = q.z;
            x[4 * v + 3] = q.w;
        }
    }
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int u = 0; u < SPT; ++u) {
        const float v = u < nv ? x[u] : 0.f;
        if (u < n0)
            s0 += v;
        else
            s1 += v;
    }
    w.pa[tid] = s0;
    w.pa[T + tid] = s1;
    __syncthreads();
    if (bpt <= 256) {
        // bin B starting at this thread, first sums acc: add the first-bin sums
        // of the threads up to the bin's end
        auto finish = [&](int B, float acc) {
            const int e = min((B + 1) * bpt - ph_lo, n_valid);
            for (int t = tid + 1; SPT * t < e; ++t)
                acc += w.pa[t];
            prof[B] += acc;
        };
        if (nv > 0) {
            if (tid == 0 && r0 != 0)
                finish(b0, s0);
            if (r0 == 0)
                finish(b0, s0);
            else if (n0 < nv)
                finish(b0 + 1, s1);
        }
        return;
    }
    // long bins: G lanes per bin over the threads ta..tb that hold its samples
    // (first bin B when the thread's first phase is >= B*bpt, else its second)
    int g2 = 0;
    while (g2 < 5 && (4 << g2) < bpt / SPT + 2)
        ++g2;
    const int G = 1 << g2, g = tid >> g2, l = tid & (G - 1), ngroups = T >> g2;
    const int b_first = div_bpt(ph_lo, bpt, f.inv_bpt);
    const int b_last = div_bpt(ph_lo + n_valid - 1, bpt, f.inv_bpt);
    for (int first = b_first; first <= b_last; first += ngroups) {
        const int B = first + g;
        float sum = 0.f;
        if (B <= b_last) {
            const int lo = B * bpt - ph_lo;
            const int ta = lo > 0 ? lo / SPT : 0;
            const int tb = min((B + 1) * bpt - 1 - ph_lo, n_valid - 1) / SPT;
            for (int t = ta + l; t <= tb; t += G)
                sum += (SPT * t >= lo) ? w.pa[t] : w.pa[T + t];
        }
        for (int o = G >> 1; o > 0; o >>= 1)
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (B <= b_last && l == 0)
            prof[B] += sum;
    }
}

// Both blocks of a pair (2M contiguous intensities from chunk-local t0, M =
// 8 * blockDim.x) in one pass of 16 samples per thread, when one span covers
// them and bins hold >= 16 samples; false (nothing folded) when the caller
// has to fold them block by block.
template <int L>
__device__ __forceinline__ bool fold_pair(const FoldArgs &f, FoldSmem &w, const float *ibuf, int t0, int M, int &sp,
                                          int &base, int &cnt)
{
    if (f.bpt < 16 || M != 8 * (int)blockDim.x)
        return false;
    while (sp < f.nspans) {
        if (sp < base || sp >= base + cnt)
            span_refill(f, w, sp, base, cnt);
        if (w.wb[sp - base] <= t0)
            ++sp;
        else
            break;
    }
    if (sp >= f.nspans)
        return false;
    const int i = sp - base;
    const int sa = w.wa[i];
    if (!(sa <= t0 && w.wb[i] >= t0 + 2 * M))
        return false;
    const int dest = w.wd[i];
    if (dest != 0) {
        const int ph_lo = w.wp[i] + (t0 - sa);
        const int n_valid = min(2 * M, f.nbins * f.bpt - ph_lo);
        if (n_valid > 0)
            fold_block_fast<L, 16>(f, w, dest == 1 ? w.prof_main : w.prof_pend, ibuf, ph_lo, n_valid);
    }
    return true;
}

// Fold the M intensities of one block (ibuf: chunk-local samples t0..t0+M-1).
// sp/base/cnt: the work item's running span cursor and window (uniform).
template <int L>
__device__ __forceinline__ void fold_block(const FoldArgs &f, FoldSmem &w, const float *ibuf, int t0, int M,
                                           int &sp, int &base, int &cnt)
{
    // advance to the first span ending after t0
    while (sp < f.nspans) {
        if (sp < base || sp >= base + cnt)
            span_refill(f, w, sp, base, cnt);
        if (w.wb[sp - base] <= t0)
            ++sp;
        else
            break;
    }
    if (sp < f.nspans && f.bpt >= 8 && M == 8 * (int)blockDim.x) {
        const int i = sp - base;
        const int sa = w.wa[i];
        if (sa <= t0 && w.wb[i] >= t0 + M) {
            const int dest = w.wd[i];
            if (dest != 0) {
                const int ph_lo = w.wp[i] + (t0 - sa);
                const int n_valid = min(M, f.nbins * f.bpt - ph_lo);
                if (n_valid > 0)
                    fold_block_fast<L>(f, w, dest == 1 ? w.prof_main : w.prof_pend, ibuf, ph_lo, n_valid);
            }
            return;
        }
    }
    const int t1 = t0 + M;
    for (int s = sp; s < f.nspans; ++s) {
        if (s >= base + cnt)
            span_refill(f, w, s, base, cnt);
        const int i = s - base;
        const int sa = w.wa[i];
        if (sa >= t1)
            break;
        const int dest = w.wd[i];
        if (dest != 0) {
            const int sb = w.wb[i];
            const int a = max(sa, t0), b = min(sb, t1);
            if (a < b) {
                const int ph_lo = w.wp[i] + (a - sa);
                fold_piece<L>(f, dest == 1 ? w.prof_main : w.prof_pend, ibuf, a - t0 - ph_lo, ph_lo, ph_lo + (b - a));
            }
            // a later span of this block may fold into the same bins
            if (sb < t1)
                __syncthreads();
        }
    }
}

}  // namespace msosm
