// Float64 tensor-core GEMM on shared-memory tiles for sm_100a: mma.sync
// m8n8k4 f64 (DMMA) fragments and a block-wide C = A B with a per-element
// epilogue.  Shared by the float64 right-hand side and its derivatives.
#pragma once

#include <cuda_runtime.h>

namespace apollo {

// Float64 tensor-core fragments: mma.sync m8n8k4 f64 (DMMA).  Fragment layout
// (PTX ISA, mma.m8n8k4 .f64): A 8x4, lane holds A[lane/4][lane%4]; B 4x8, lane
// holds B[lane%4][lane/4]; C 8x8, lane holds C[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }
// leading dimension (in doubles) of a shared-memory tile read by fragments:
// rows 4 apart must land 8 banks apart, i.e. ld = 4 (mod 16)
constexpr int pad_ld(int x) { return x + ((4 - x % 16) + 16) % 16; }

constexpr int tile_n(int cblocks, int rblocks, int warps) {
  // widest column tile (4, 2, 1 blocks of 8) that still gives every warp work
  return (cblocks % 4 == 0 && rblocks * (cblocks / 4) >= warps) ? 4
         : (cblocks % 2 == 0 && rblocks * (cblocks / 2) >= warps) ? 2 : 1;
}

// C[ROWS x COLS] = A[ROWS x K] B[K x COLS] over the block's warps; A, B in
// shared memory; the epilogue gets (row, col, value) per output.  KSPLIT > 1
// accumulates the k-steps round robin into that many partial sums (summed at
// the end), so a long K is not one chain of dependent DMMAs.
template <int ROWS, int COLS, int K, int LDA, int LDB, int NWARPS, int KSPLIT = 1, class Epi>
__device__ __forceinline__ void block_dgemm(const double* A, const double* B, Epi epi) {
  constexpr int RB = ROWS / 8, CB = COLS / 8, KS = K / 4;
  constexpr int TN = tile_n(CB, RB, NWARPS);
  constexpr int NT = RB * (CB / TN);
  constexpr int SP = KSPLIT < KS ? KSPLIT : (KS > 0 ? KS : 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lr = lane >> 2, lc = lane & 3;
  for (int t = warp; t < NT; t += NWARPS) {
    const int rb = t % RB, cg = t / RB;
    double c[SP][TN][2];
#pragma unroll
    for (int p = 0; p < SP; ++p)
#pragma unroll
      for (int n = 0; n < TN; ++n) c[p][n][0] = c[p][n][1] = 0.0;
    const double* ap = A + (rb * 8 + lr) * LDA + lc;
    const double* bp = B + lc * LDB + cg * TN * 8 + lr;
    if constexpr (SP == 1) {
#pragma unroll 4
      for (int k = 0; k < KS; ++k) {
        const double a = ap[k * 4];
#pragma unroll
        for (int n = 0; n < TN; ++n) dmma_8x8x4(c[0][n], a, bp[k * 4 * LDB + n * 8]);
      }
    } else {
      constexpr int KF = KS / SP * SP;
      for (int k0 = 0; k0 < KF; k0 += SP) {
#pragma unroll
        for (int p = 0; p < SP; ++p) {
          const double a = ap[(k0 + p) * 4];
#pragma unroll
          for (int n = 0; n < TN; ++n) dmma_8x8x4(c[p][n], a, bp[(k0 + p) * 4 * LDB + n * 8]);
        }
      }
#pragma unroll
      for (int k = KF; k < KS; ++k) {
        const double a = ap[k * 4];
#pragma unroll
        for (int n = 0; n < TN; ++n) dmma_8x8x4(c[k - KF][n], a, bp[k * 4 * LDB + n * 8]);
      }
#pragma unroll
      for (int p = 1; p < SP; ++p)
#pragma unroll
        for (int n = 0; n < TN; ++n) {
          c[0][n][0] += c[p][n][0];
          c[0][n][1] += c[p][n][1];
        }
    }
#pragma unroll
    for (int n = 0; n < TN; ++n) {
      const int col = (cg * TN + n) * 8 + 2 * lc;
      epi(rb * 8 + lr, col, c[0][n][0]);
      epi(rb * 8 + lr, col + 1, c[0][n][1]);
    }
  }
}

}  // namespace apollo
