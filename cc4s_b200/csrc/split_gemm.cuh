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

uint64_t split_launch_count();

}  // namespace cc4s_b200
