// Host check of the tensor-core row order (tc_layout.hpp): for FFT 4096,
// 8192 and 16384, tc_pos is a permutation of the N positions, and each bin
// pair a gather thread reads (warp w, lane l, pass j, row part b) is the pair
// of bins whose GEMM 1 operand element the thread writes: rows
// 64 b + 8 j + 2 (l & 3) + {0, 1} and K index k2 = 8 w + (l >> 2).  At 4096
// and 8192 row part b is block b of a pair (the same bins, read from two ring
// rows); at 16384 it is half b of one block's row (k1 = 64 b + ...).
// Prints "ok" and exits 0, else names the first mismatch and exits 1.
#include <cstdio>
#include <vector>

#include "tc_layout.hpp"

using namespace msosm::tc;

template <int LOG2N>
static bool check()
{
    using S = TcShape<LOG2N>;
    constexpr int N = S::N;
    std::vector<int> inv(N, -1);
    for (int b = 0; b < N; ++b) {
        const int p = tc_pos(b, LOG2N);
        if (p < 0 || p >= N || inv[p] >= 0) {
            std::printf("N=%d: bin %d -> position %d is not a permutation\n", N, b, p);
            return false;
        }
        inv[p] = b;
    }
    const int parts = S::BPS == 2 ? 1 : 2;  // row halves read per step
    for (int w = 0; w < S::WARPS; ++w)
        for (int l = 0; l < 32; ++l)
            for (int j = 0; j < 8; ++j)
                for (int h = 0; h < parts; ++h)
                    for (int e = 0; e < 2; ++e) {
                        const int q = h * (N / 4) + (j * S::WARPS + w) * 32 + l;  // float4 index
                        const int bin = inv[2 * q + e];
                        const int k1 = bin % S::N1, k2 = bin / S::N1;
                        const int row = 64 * h + 8 * j + 2 * (l & 3) + e;  // row within the step's operand
                        const int kk = 8 * w + (l >> 2);
                        if (k1 != row || k2 != kk) {
                            std::printf("N=%d: w %d l %d j %d h %d e %d reads bin %d (k1 %d k2 %d), writes row %d k %d\n",
                                        N, w, l, j, h, e, bin, k1, k2, row, kk);
                            return false;
                        }
                    }
    return true;
}

int main()
{
    if (!check<12>() || !check<13>() || !check<14>())
        return 1;
    std::printf("ok\n");
    return 0;
}
