// Split-precision FP64 contraction on the 5th-generation tensor cores (tcgen05).
//
// C = alpha * A B + beta * C with FP64 operands, computed from FP16 slices
// (Ozaki-style): every row of A (and every column of B) is scaled by a power
// of two so that its largest element is below 1 and cut into three integer
// slices of 6, 11 and 11 bits,
//     a = 2^e (S1 2^-6 + S2 2^-17 + S3 2^-28),
// each slice an integer stored exactly in FP16.  The six slice products with
// p + q <= 4 are summed by tcgen05.mma (kind::f16, FP32 accumulation in
// TMEM) into three groups of equal weight 2^-12, 2^-23 and 2^-34.  The
// leading group (|S1 S1| <= 2^12) is exact in FP32 over K chunks of 4096;
// after each chunk the groups are combined in FP64 and added to C.
// Precision: 28 bits of each operand relative to its row / column maximum.
#pragma once

#include "gemm_f64.cuh"

namespace cc4s_b200 {

struct SplitScratch {
  void* p = nullptr;     // device scratch for the packed slices
  size_t bytes = 0;
  int* error = nullptr;  // device flag: non-zero if a bounded wait gave up
};

// Same contraction semantics as gemm() (two-level index maps, optional C2).
// The batch dimension must be 1.  Falls back to nothing: throws if the
// contraction cannot be expressed (the caller then uses gemm()).
void gemm_split(const Contraction& g, cudaStream_t s, SplitScratch& ws);

// Bytes of scratch gemm_split needs for this contraction.
size_t gemm_split_scratch_bytes(const Contraction& g);

// Operand B of a one-panel split contraction, sliced once and reused by several
// contractions that share B (same N, K and B view), e.g. the ladder's X panel
// for every block pair of one c range.
struct SplitPackedB {
  void* slices = nullptr;  // [3][Np][Kp] FP16
  int* exps = nullptr;     // [Np] power-of-two column scales
  int64_t N = 0, K = 0, Np = 0, Kp = 0;
};
// Bytes split_pack_b writes (slices, row maxima, exponents).
size_t split_packed_b_bytes(const Contraction& g);
// Scratch bytes of gemm_split_packed_b for this contraction (packed A and metadata).
size_t split_scratch_bytes_packed_b(const Contraction& g);
// True if g runs as one K panel (the condition for a pre-packed B).
bool split_single_panel(const Contraction& g);
// Slices B of g into dst (device memory of split_packed_b_bytes(g) bytes, 1 KiB aligned).
SplitPackedB split_pack_b(const Contraction& g, void* dst, cudaStream_t s);
// gemm_split with B taken from split_pack_b (A is sliced into ws as usual; ws must
// not overlap b).
void gemm_split_packed_b(const Contraction& g, const SplitPackedB& b, cudaStream_t s,
                         SplitScratch& ws);

// An operand sliced once for many contractions: R rows of K elements as three FP16
// planes [3][Rp][Kp] with one power-of-two exponent per row (the scaling of every
// row over its whole K, as gemm_split slices its operands).
struct SplitOperand {
  void* slices = nullptr;
  int* exps = nullptr;   // [Rp]
  int64_t R = 0, K = 0, Rp = 0, Kp = 0;
};
// Device bytes of a sliced operand of R rows and K columns.
size_t split_operand_bytes(int64_t R, int64_t K);
// Slices the rows of src into dst (device memory of split_operand_bytes bytes):
// element (r, k) at src[(r / Ri) * s_ro + (r % Ri) * s_ri + k * s_k] (Ri = 0: one level).
SplitOperand split_pack_operand(const double* src, int64_t R, int64_t Ri, int64_t s_ro,
                                int64_t s_ri, int64_t K, int64_t s_k, void* dst, cudaStream_t s);
// The rows of a contraction inside a sliced operand: logical index x is packed row
//   base + (x / run) * stride + x % run.
struct SplitRuns {
  int64_t base = 0, run = 0, stride = 0;
};
// C = alpha A B + beta C (g gives M, N, K, the output views, alpha, beta) with the rows
// m of A and the columns n of B taken from sliced operands (B sliced by its columns,
// i.e. its rows are n).  Tiles never straddle a run, so a run shorter than a tile
// costs a partial tile.  Persistent kernel only.
void gemm_split_prepacked(const Contraction& g, const SplitOperand& A, const SplitRuns& ar,
                          const SplitOperand& B, const SplitRuns& br, cudaStream_t s,
                          SplitScratch& ws);

uint64_t split_launch_count();
// Number of operand-slicing kernel launches issued so far (two per sliced operand).
uint64_t split_pack_launch_count();

}  // namespace cc4s_b200
