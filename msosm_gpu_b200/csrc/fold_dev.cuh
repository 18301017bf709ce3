// fold_dev.cuh -- device side of the deterministic fold shared by the fused
// dedispersion kernels (CUDA-core and tensor-core) and the series fold.
#pragma once

#include "kernels.hpp"

namespace msosm {

// Folding inside the dedispersion kernel.  The host fold planner cuts each
// call's output samples into spans (one period each, sorted); a work item
// keeps a window of them in shared memory and its two partial profiles
// (complete periods, pending period) in shared memory too.  Every bin of a
// span piece is summed by one warp (lanes strided over its samples, then a
// fixed xor-butterfly) or, for bins of fewer than 16 samples, by one thread
// in sample order; span pieces are separated by barriers.  The result does
// not depend on scheduling.
struct FoldSmem {
    float *prof_main, *prof_pend;  // [nbins] each (or the global rows)
    int *wa, *wb, *wp, *wd;        // span window (chunk-local sample indices < 2^31)
};

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

// ibuf holds intensities at index t + t/32 (one pad slot per 32 samples), so
// that threads reading bins of any length hit different banks
__device__ __forceinline__ int ipad(int t) { return t + (t >> 5); }

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
                a0 += ibuf[ipad(off + p)];
                a1 += ibuf[ipad(off + p + G)];
            }
            if (p < s_hi)
                a0 += ibuf[ipad(off + p)];
        }
        float sum = a0 + a1;
        for (int o = G >> 1; o > 0; o >>= 1)
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (bin <= b_hi && l == 0)
            prof[bin] += sum;
    }
}

// Fold the M intensities of one block (ibuf: chunk-local samples t0..t0+M-1).
// sp/base/cnt: the work item's running span cursor and window (uniform).
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
                fold_piece(f, dest == 1 ? w.prof_main : w.prof_pend, ibuf, a - t0 - ph_lo, ph_lo, ph_lo + (b - a));
            }
            // a later span of this block may fold into the same bins
            if (sb < t1)
                __syncthreads();
        }
    }
}

}  // namespace msosm
