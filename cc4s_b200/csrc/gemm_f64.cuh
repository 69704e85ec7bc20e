// Strided FP64 tensor contraction on the B200 FP64 tensor pipe (mma.sync DMMA).
//
// Every contraction of the CCSD residual is expressed as
//     C[b](m, n) = alpha * sum_k A[b](m, k) * B[b](k, n) + beta * C[b](m, n)
// where each of the indices m, n, k and the batch index b may be split into
// two levels (outer, inner) with independent strides in every operand.  This
// lets permuted tensor layouts (e.g. T_abij read as a (ai) x (bj) matrix, or
// the exchange pairing (aj) x (bi)) feed the tensor cores without explicit
// transpose passes, and lets the epilogue scatter into any pairing of R_abij.
#pragma once

#include "common.cuh"

namespace cc4s_b200 {

// Element (r, c, b) of an operand lives at
//   p + (r / Ri) * s_ro + (r % Ri) * s_ri + (c / Ci) * s_co + (c % Ci) * s_ci
//     + (b / Bi) * s_bo + (b % Bi) * s_bi
// with the inner extents (Ri, Ci, Bi) supplied by the contraction.
struct View {
  double* p = nullptr;
  int64_t s_ro = 0, s_ri = 0, s_co = 0, s_ci = 0, s_bo = 0, s_bi = 0;
};

// Row-major matrix view with leading dimension ld (rows stride ld, cols stride 1).
inline View rm(double* p, int64_t ld) {
  View v; v.p = p; v.s_ri = ld; v.s_ci = 1; return v;
}
// Transposed view of a row-major matrix with leading dimension ld:
// element (r, c) is p[c * ld + r].
inline View tr(double* p, int64_t ld) {
  View v; v.p = p; v.s_ri = 1; v.s_ci = ld; return v;
}
inline View with_batch(View v, int64_t s_bi, int64_t s_bo = 0) {
  v.s_bi = s_bi; v.s_bo = s_bo; return v;
}

struct Contraction {
  int64_t M = 0, N = 0, K = 0, batch = 1;
  // Inner extents of the two-level splits; 0 means "one level" (= full extent).
  int64_t Mi = 0, Ni = 0, Ki = 0, Bi = 0;
  View A;   // rows m, cols k
  View B;   // rows k, cols n
  View C;   // rows m, cols n
  View C2;  // optional second output (C2.p == nullptr: none): C2 = alpha*AB + beta*C2
  double alpha = 1.0, beta = 0.0;
};

// Scratch memory used by split-K partial sums.
struct GemmScratch {
  double* p = nullptr;
  size_t elems = 0;
};

void gemm(const Contraction& g, cudaStream_t s, const GemmScratch& ws);

// Number of FP64 GEMM kernel launches issued so far (for launch accounting).
uint64_t gemm_launch_count();

}  // namespace cc4s_b200
