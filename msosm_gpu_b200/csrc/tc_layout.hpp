// tc_layout.hpp -- data layout of the tensor-core (tcgen05) dedispersion path
// for 4096-, 8192- and 16384-point transforms, shared by the host (set-up
// permutations) and the device (kernels).
//
// The inverse N-point DFT is split as N1 x N2 (four-step; N1 = 64 at 4096
// and 8192, 128 at 16384; N2 = N / N1): bin k = k1 + N1 k2, output
// m = N2 m1 + m2,
//   A[k1][m2]  = sum_k2 Z[k1 + N1 k2] e^{+2 pi i k2 m2 / N2}          (GEMM 1)
//   A'[k1][m2] = A[k1][m2] e^{+2 pi i k1 m2 / N}                      (twiddle)
//   y[N2 m1 + m2] = sum_k1 A'[k1][m2] e^{+2 pi i k1 m1 / N1}, m1 >= N1/2 (GEMM 2)
// Only m1 >= N1 / 2 (outputs m >= M = N / 2) survive the overlap-save
// discard, so GEMM 2 computes half of its outputs.  Complex GEMMs run as real
// GEMMs: with the data [Re | Im] and the DFT C + iS, the constant operand
// holds only [C | S] and
//   [Re | Im] of the product = Re x [C | S]  +  [-Im x S | Im x C],
// the negation coming from the instruction's negate-A bit.
//
// Shared-memory operands use the canonical no-swizzle UMMA layouts of 8 x 8
// f16 core matrices (8 rows of 16 contiguous bytes):
//   data operand A (M = 128 rows x K), MN-major: 8 consecutive rows of one K
//     column are contiguous; row groups 128 B apart, K groups 2048 B
//   constant operand B (N x K), K-major: 8 consecutive K of one column
//     contiguous; K groups 128 B apart, N groups K / 8 x 128 B apart
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msosm {
namespace tc {

// Shape of the tensor-core path for an N-point transform, N = 4096, 8192 or
// 16384: bin k = k1 + N1 k2 (k1 < N1, k2 < N2), output m = N2 m1 + m2; GEMM 1
// sums over k2 (an N2-point DFT), GEMM 2 over k1 (N1 points, m1 >= N1 / 2
// kept).  GEMM 1 has 128 rows: two blocks x 64 k1 at N = 4096 and 8192 (a
// step handles a pair of blocks), one block x 128 k1 at N = 16384 (a step
// handles one block).  At N = 4096 one GEMM 2 covers both blocks of a pair
// (rows 64 b + m2); at N = 8192 each block has its own (rows m2 < 128); at
// N = 16384 the single block's GEMM 2 has rows m2 < 128 and takes its
// constant from GEMM 1's (the 128-point [C | S], columns m1 = 64 .. 127 of
// each half), so it needs no table of its own.
template <int LOG2N>
struct TcShape {
    static constexpr int N = 1 << LOG2N, M = N / 2;
    static constexpr int N1 = LOG2N == 14 ? 128 : 64;  // GEMM 2 length (k1)
    static constexpr int N2 = N / N1;                  // GEMM 1 length (k2): 64 or 128
    static constexpr int BPS = 128 / N1;               // blocks per step: 2 or 1
    static constexpr int WARPS = N2 / 8;               // 8 or 16
    static constexpr int THREADS = 32 * WARPS;         // 256 or 512
    static constexpr int CTAS_PER_SM = LOG2N == 12 ? 2 : 1;
    static constexpr int B1_BYTES = 2 * N2 * N2 * 2;                  // [C | S]: 2 N2 columns x N2 K, 16-bit
    // At N = 4096 (N1 = N2 = 64) both GEMMs are 64-point DFTs: B1 holds
    // [C_lo | S_lo | C_hi | S_hi] (32 frequencies each, lo = 0..31, hi =
    // 32..63) and B1N the companion [-S_lo | C_lo | -S_hi | C_hi], so each
    // GEMM is Re x B1 + Im x B1N (GEMM 2 on columns 64..127): 8 MMAs each
    // instead of 12, no B2 table, the same shared memory.  GEMM 1 then
    // leaves D1 as [Re_lo | Im_lo | Re_hi | Im_hi].
    static constexpr bool PAIRED = LOG2N == 12;
    static constexpr int B2_BYTES = LOG2N == 13 ? 64 * 64 * 2 : 0;    // [C | S]: 64 columns x 64 K
    static constexpr int B1N_BYTES = PAIRED ? 2 * N2 * N2 * 2 : 0;
    // at N = 8192 (GEMM 1 128-point, GEMM 2 64-point) [-S | C] beside B2, so
    // that each block's GEMM 2 is Re x B2 + Im x B2N: 8 MMAs instead of 12
    static constexpr int B2N_BYTES = LOG2N == 13 ? 64 * 64 * 2 : 0;
    static constexpr int OP_BYTES = 128 * 2 * N2 * 2;    // GEMM 1 data operand (128 rows x 2 N2 K)
    static constexpr int SMEM_B1 = 0;
    static constexpr int SMEM_B2 = B1_BYTES;
    static constexpr int SMEM_B1N = B1_BYTES + B2_BYTES;
    static constexpr int SMEM_B2N = B1_BYTES + B2_BYTES + B1N_BYTES;
    static constexpr int SMEM_OP0 = B1_BYTES + B2_BYTES + B1N_BYTES + B2N_BYTES;  // two operand buffers; a buffer then
    static constexpr int SMEM_OP1 = SMEM_OP0 + OP_BYTES;  // holds its step's intensities
    static constexpr int SMEM_CTL = SMEM_OP1 + OP_BYTES;  // mbarriers, TMEM address, per-warp maxima
    static constexpr int SMEM_FOLD = SMEM_CTL + 256;      // fold span window, partials, profiles
    static constexpr uint32_t SBO_B1 = (uint32_t)N2 * 16;  // B1 N-group stride (N2 / 8 K-groups x 128 B)
    static constexpr int IM_OFF = (N2 / 8) * 2048;         // GEMM 1 operand: Im part, K = N2 on
    static constexpr int IM2_OFF = (N1 / 8) * 2048;        // GEMM 2 operand: Im part, K = N1 on
    static constexpr int D2_COL = 2 * N2;                  // TMEM: D1 at 0 .. 2 N2 - 1, D2 after it
    static constexpr int D2_HALF = N1 / 2;                 // D2 columns per part (Re, Im) of one block
    static constexpr int TW_COL = D2_COL + (N2 == 64 ? 64 : 128);  // past D2: 32 spare columns per column group
    static constexpr int TMEM_COLS = LOG2N == 12 ? 256 : 512;
    static constexpr int SCALE_EXP = LOG2N == 12 ? 8 : 7;  // |Z| < 2^SCALE_EXP: GEMM 1 sums < 2^15
};

constexpr int kLog2NMin = 12, kLog2NMax = 14;
// threads of the GEMM layout check (tc_probe_kernel)
constexpr int kThreads = 256;

// MN-major data operand (K groups 2048 B apart, row groups 128 B): element
// (row r, k) -> byte offset
__host__ __device__ constexpr int mn_off(int r, int k)
{
    return (r >> 3) * 128 + (k >> 3) * 2048 + (k & 7) * 16 + (r & 7) * 2;
}
// K-major constant operand with N-group stride sbo: element (column n, k) -> byte offset
__host__ __device__ constexpr int k_off(int n, int k, int sbo = 1024)
{
    return (n >> 3) * sbo + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

// Position of bin b in a tensor-core-ordered spectrum row (ring, H, delays)
// of N = 2^log2n points.  Thread (warp w, lane l) of the gather reads, in pass
// j, the bin pair at positions 64 (W j + w) + 2 l + {0, 1} (W warps): bins
// k1 = 8 j + 2 (l & 3) + {0, 1}, k2 = 8 w + (l >> 2), which it stores as one
// 32-bit word of one core-matrix row -- a warp fills a whole 128-byte core
// matrix per store.  At N = 16384 (k1 < 128) the row holds two halves of
// 8192 positions, k1 < 64 then k1 >= 64, each in the 8192-point order of
// (k1 mod 64, k2): the gather reads both halves of one block where the
// smaller sizes read two blocks.
__host__ __device__ constexpr int tc_pos(int b, int log2n)
{
    if (log2n == 14)
        return ((b >> 6) & 1) * 8192 + tc_pos((b & 63) | ((b >> 7) << 6), 13);
    const int k1 = b & 63, k2 = b >> 6;
    const int warps = (1 << (log2n - 6)) / 8;
    const int u = (k1 >> 3) * warps + (k2 >> 3);
    const int l = (k2 & 7) * 4 + ((k1 & 7) >> 1);
    return u * 64 + l * 2 + (k1 & 1);
}

// Shared-memory matrix descriptor, no swizzle (tcgen05 descriptor format:
// start >> 4 in bits 0-13, leading byte offset >> 4 in 16-29, stride byte
// offset >> 4 in 32-45, version 1 in 46-47, layout 0 in 61-63).  For the
// no-swizzle layouts the leading offset is the K-direction step between core
// matrices and the stride offset the M/N-direction step.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// descriptor steps: K step of 16 elements (two core-matrix columns)
constexpr uint32_t kDescStepA = 2 * 2048;  // MN-major data operand (LBO 2048, SBO 128)
constexpr uint32_t kDescStepB = 2 * 128;   // K-major constant operand (LBO 128)

// Instruction descriptor, kind::f16: f32 accumulator (bits 4-5 = 1), A and
// B of one type (bits 7-9 and 10-12: 0 f16, 1 bf16), negate A (bit 13), A
// MN-major (bit 15), B K-major (bit 16 = 0), N >> 3 in bits 17-22, M >> 4 in
// bits 24-28.
__host__ __device__ constexpr uint32_t idesc_f16(int m, int n, bool a_mn_major, bool neg_a = false,
                                                 uint32_t fmt = 0)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((neg_a ? 1u : 0u) << 13) | ((a_mn_major ? 1u : 0u) << 15) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

}  // namespace tc
}  // namespace msosm
