// tc_layout.hpp -- data layout of the tensor-core (tcgen05) dedispersion path
// for 4096-point transforms, shared by the host (set-up permutations) and the
// device (kernels).
//
// The inverse 4096-point DFT is split as 64 x 64 (four-step): bin
// k = k1 + 64 k2, output m = 64 m1 + m2,
//   A[k1][m2]  = sum_k2 Z[k1 + 64 k2] e^{+2 pi i k2 m2 / 64}        (GEMM 1)
//   A'[k1][m2] = A[k1][m2] e^{+2 pi i k1 m2 / 4096}                   (twiddle)
//   y[64 m1 + m2] = sum_k1 A'[k1][m2] e^{+2 pi i k1 m1 / 64}, m1 >= 32 (GEMM 2)
// Only m1 >= 32 (outputs m >= M = 2048) survive the overlap-save discard, so
// GEMM 2 computes half of its outputs.  Complex GEMMs run as real GEMMs:
// with the data [Re | Im] (K = 128) and the DFT C + iS, the constant operand
// holds only [C | S] (K = 64) and
//   [Re | Im] of the product = Re x [C | S]  +  [-Im x S | Im x C],
// the negation coming from the instruction's negate-A bit.
//
// Shared-memory operands use the canonical no-swizzle UMMA layouts of 8 x 8
// f16 core matrices (8 rows of 16 contiguous bytes):
//   data operand A (M = 128 rows x K = 128), MN-major: 8 consecutive rows of
//     one K column are contiguous; row groups 128 B apart, K groups 2048 B
//   constant operand B (N x K = 64), K-major: 8 consecutive K of one column
//     contiguous; K groups 128 B apart, N groups 1024 B
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msosm {
namespace tc {

constexpr int kLog2N = 12;
constexpr int kN = 1 << kLog2N, kM = kN / 2;
constexpr int kThreads = 256;

// byte offsets in dynamic shared memory
constexpr int kSmemB1 = 0;        // GEMM 1 constant [C | S]: 128 (N) x 64 (K) f16
constexpr int kSmemB2 = 16384;    // GEMM 2 constant [C | S]:  64 (N) x 64 (K) f16
constexpr int kSmemOp0 = 24576;   // two data-operand buffers (128 x 128 f16 each); a
constexpr int kSmemOp1 = 57344;   //   buffer then holds its pair's intensities
constexpr int kSmemCtl = 90112;   // mbarriers, TMEM address
constexpr int kSmemFold = 90368;  // fold span window, partials and profiles
constexpr int kTmemCols = 256;    // D1 at columns 0..127, D2 at 128..191

// MN-major data operand: element (row r, k) -> byte offset
__host__ __device__ constexpr int mn_off(int r, int k)
{
    return (r >> 3) * 128 + (k >> 3) * 2048 + (k & 7) * 16 + (r & 7) * 2;
}
// K-major constant operand (K = 64): element (column n, k) -> byte offset
__host__ __device__ constexpr int k_off(int n, int k)
{
    return (n >> 3) * 1024 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
}

// Position of bin b in a tensor-core-ordered spectrum row (ring, H, delays).
// Thread (warp w, lane l) of the gather reads, in pass j, the bin pair at
// positions 64 (8 j + w) + 2 l + {0, 1}: bins k1 = 8 j + 2 (l & 3) + {0, 1},
// k2 = 8 w + (l >> 2), which it stores as one 32-bit word of one core matrix
// row -- a warp fills a whole 128-byte core matrix per store.
__host__ __device__ constexpr int tc_pos(int b)
{
    const int k1 = b & 63, k2 = b >> 6;
    const int u = (k1 >> 3) * 8 + (k2 >> 3);
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
// descriptor steps: K step of 16 f16 (two core-matrix columns) and the
// constant operand's column offset
constexpr uint32_t kDescStepA = 2 * 2048;  // MN-major data operand (LBO 2048, SBO 128)
constexpr uint32_t kDescStepB = 2 * 128;   // K-major constant operand (LBO 128, SBO 1024)
__host__ __device__ constexpr uint32_t b_col(int n) { return (uint32_t)(n >> 3) * 1024; }

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
