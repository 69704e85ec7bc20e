// Kernel-level check and timing of the split-precision contraction (gemm_split)
// against the FP64 DMMA contraction (gemm) on plain row-major operands.
// Usage: split_check [shape index]; prints one line per shape and exits non-zero
// on a CUDA error, a bounded-wait error flag or a relative difference above 1e-5.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cmath>
#include "../../cc4s_b200/csrc/split_gemm.cuh"
using namespace cc4s_b200;

int main(int argc, char** argv) {
  // view 0: row-major C; views 1 and 2: the block array S[224][224][224] of the
  // perturbative triples written through a permuted two-level view (1: columns
  // contiguous, 2: rows contiguous), accumulating (beta = 1) as there.
  struct S { int64_t M, N, K; int tA, tB; double beta; int view; };
  S shapes[] = {{128, 128, 64, 0, 0, 0.0, 0}, {200, 136, 100, 0, 1, 0.0, 0},
                {1000, 700, 5000, 1, 0, 0.0, 0}, {4096, 4096, 4096, 0, 0, 0.0, 0},
                {8192, 8192, 8192, 0, 0, 0.0, 0}, {4096, 4096, 40960, 0, 0, 0.0, 0},
                {16384, 16384, 2560, 0, 0, 0.0, 0}, {8192, 8192, 65536, 0, 0, 0.0, 0},
                {1000, 700, 5000, 1, 0, 1.0, 0}, {7168, 1568, 256, 0, 0, 1.0, 1},
                {7168, 1568, 256, 0, 0, 1.0, 2}};
  const int64_t L = 224, o = 32;
  int* err; cudaMalloc(&err, 4); cudaMemset(err, 0, 4);
  SplitScratch ws; ws.bytes = size_t(4) << 30; cudaMalloc(&ws.p, ws.bytes); ws.error = err;  // >= any panel
  GemmScratch gs; gs.elems = 1 << 24; cudaMalloc(&gs.p, gs.elems * 8);
  const int only = argc > 1 ? atoi(argv[1]) : -1;
  int idx = -1;
  for (auto& s : shapes) {
    ++idx;
    if (only >= 0 && idx != only) continue;
    double *A, *B, *C1, *C2;
    const int64_t nc = s.view ? L * L * L : s.M * s.N;
    cudaMalloc(&A, s.M * s.K * 8); cudaMalloc(&B, s.K * s.N * 8);
    cudaMalloc(&C1, nc * 8); cudaMalloc(&C2, nc * 8);
    std::vector<double> h(std::max(std::max(s.M * s.K, s.K * s.N), nc));
    srand(7);
    for (auto& x : h) x = ((rand() / (double)RAND_MAX) - 0.5) * std::pow(2.0, (rand() % 9) - 4);
    cudaMemcpy(A, h.data(), s.M * s.K * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(B, h.data(), s.K * s.N * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(C1, h.data(), nc * 8, cudaMemcpyHostToDevice);  // the same start for beta = 1
    cudaMemcpy(C2, h.data(), nc * 8, cudaMemcpyHostToDevice);
    Contraction c; c.M = s.M; c.N = s.N; c.K = s.K; c.beta = s.beta;
    c.A = s.tA ? tr(A, s.M) : rm(A, s.K);
    c.B = s.tB ? tr(B, s.K) : rm(B, s.N);
    auto cview = [&](double* p) {
      View v;
      v.p = p;
      if (s.view == 1) {         // rows (pair p, hole q), columns (virtual q, pair r)
        v.s_ro = L * L; v.s_ri = L; v.s_co = o * L; v.s_ci = 1;
      } else if (s.view == 2) {  // rows (hole q, pair p) with pair p contiguous
        v.s_ro = L; v.s_ri = 1; v.s_co = o * L; v.s_ci = L * L;
      } else {
        v = rm(p, s.N);
      }
      return v;
    };
    if (s.view) { c.Mi = s.view == 1 ? o : L; c.Ni = L; }
    c.C = cview(C1);
    cudaEvent_t e0, e1, e2; cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
    gemm(c, 0, gs);
    cudaEventRecord(e0);
    gemm(c, 0, gs);
    cudaEventRecord(e1);
    c.C = cview(C2);
    gemm_split(c, 0, ws);
    cudaEventRecord(e2);
    gemm_split(c, 0, ws);
    cudaEvent_t e3; cudaEventCreate(&e3); cudaEventRecord(e3);
    cudaError_t ce = cudaDeviceSynchronize();
    float ms64 = 0, ms = 0; cudaEventElapsedTime(&ms64, e0, e1); cudaEventElapsedTime(&ms, e2, e3);
    int herr = 0; cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    std::vector<double> r1(nc), r2(nc);
    cudaMemcpy(r1.data(), C1, nc * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(r2.data(), C2, nc * 8, cudaMemcpyDeviceToHost);
    double md = 0, mx = 0;
    for (size_t i = 0; i < r1.size(); ++i) {
      // beta = 1: both paths ran twice onto the same start; compare the added products
      const double a = r1[i] - (s.beta != 0.0 ? h[i] : 0.0);
      md = std::fmax(md, std::fabs(r1[i] - r2[i]));
      mx = std::fmax(mx, std::fabs(a));
    }
    const double f = 2.0 * s.M * s.N * s.K;
    printf("M=%ld N=%ld K=%ld tA=%d tB=%d beta=%g view=%d: cuda=%s errflag=%d max|diff|/max=%.3e fp64 %.3f ms = %.1f TF; split %.3f ms = %.1f TF(fp64-equiv)\n",
           (long)s.M, (long)s.N, (long)s.K, s.tA, s.tB, s.beta, s.view, cudaGetErrorString(ce), herr, md / mx,
           ms64, f / (ms64 * 1e-3) / 1e12, ms, f / (ms * 1e-3) / 1e12);
    if (ce != cudaSuccess || herr || !(md / mx < 1e-5)) return 1;
    cudaFree(A); cudaFree(B); cudaFree(C1); cudaFree(C2);
  }
  return 0;
}
