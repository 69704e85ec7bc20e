// TEST INFRASTRUCTURE ONLY: plain-loop CPU emulation of the device operations
// declared in cc4s_b200/csrc/ops.h and gemm_f64.cuh.
//
// It is linked with the product's schedule and driver sources into a separate
// test library (tests/emu/_build/libcc4s_emu.so) so that the index and stride
// bookkeeping of every contraction can be checked against the oracle on a
// machine without a GPU.  The product library never contains this file.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../cc4s_b200/csrc/ops.h"
#include "../../cc4s_b200/csrc/split_gemm.cuh"

namespace cc4s_b200 {

namespace {
struct Ax {
  int64_t inner, so, si;
  int64_t off(int64_t x) const { return (x / inner) * so + (x % inner) * si; }
};
Ax ax(int64_t inner, int64_t so, int64_t si) { return Ax{inner > 0 ? inner : 1, so, si}; }
uint64_t g_gemm = 0, g_ops = 0;
}  // namespace

uint64_t gemm_launch_count() { return g_gemm; }

void gemm(const Contraction& g, cudaStream_t, const GemmScratch&) {
  ++g_gemm;
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  const int64_t Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1), Bi = g.Bi > 0 ? g.Bi : g.batch;
  Ax Am = ax(Mi, g.A.s_ro, g.A.s_ri), Ak = ax(Ki, g.A.s_co, g.A.s_ci);
  Ax Bk = ax(Ki, g.B.s_ro, g.B.s_ri), Bn = ax(Ni, g.B.s_co, g.B.s_ci);
  Ax Cm = ax(Mi, g.C.s_ro, g.C.s_ri), Cn = ax(Ni, g.C.s_co, g.C.s_ci);
  Ax C2m = ax(Mi, g.C2.s_ro, g.C2.s_ri), C2n = ax(Ni, g.C2.s_co, g.C2.s_ci);
  Ax Ab = ax(Bi, g.A.s_bo, g.A.s_bi), Bb = ax(Bi, g.B.s_bo, g.B.s_bi);
  Ax Cb = ax(Bi, g.C.s_bo, g.C.s_bi), C2b = ax(Bi, g.C2.s_bo, g.C2.s_bi);
  std::vector<int64_t> ak(g.K), bk(g.K);
  for (int64_t k = 0; k < g.K; ++k) { ak[k] = Ak.off(k); bk[k] = Bk.off(k); }
  for (int64_t b = 0; b < g.batch; ++b) {
    const double* A = g.A.p ? g.A.p + Ab.off(b) : nullptr;
    const double* B = g.B.p ? g.B.p + Bb.off(b) : nullptr;
    for (int64_t m = 0; m < g.M; ++m) {
      const int64_t am = Am.off(m);
      for (int64_t n = 0; n < g.N; ++n) {
        const int64_t bn = Bn.off(n);
        double s = 0.0;
        for (int64_t k = 0; k < g.K; ++k) s += A[am + ak[k]] * B[bk[k] + bn];
        const double v = g.alpha * s;
        double* c = g.C.p + Cb.off(b) + Cm.off(m) + Cn.off(n);
        *c = g.beta != 0.0 ? v + g.beta * *c : v;
        if (g.C2.p) {
          double* c2 = g.C2.p + C2b.off(b) + C2m.off(m) + C2n.off(n);
          *c2 = g.beta != 0.0 ? v + g.beta * *c2 : v;
        }
      }
    }
  }
}

// Emulation of the split-precision contraction: the same row/column scaling,
// integer slices (6, 11, 11 bits) and the six slice products p + q <= 2
// (0-based), summed exactly in FP64 (the device sums the leading group exactly
// in FP32 per 4096-wide chunk; the lower groups differ only below 2^-50 relative).
static uint64_t g_split = 0, g_pack = 0;
uint64_t split_launch_count() { return g_split; }
uint64_t split_pack_launch_count() { return g_pack; }
size_t gemm_split_scratch_bytes(const Contraction&) { return 64; }

void gemm_split(const Contraction& g, cudaStream_t, SplitScratch&) {
  ++g_split;
  g_pack += 4;  // the device slices both operands (two launches each)
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  const int64_t Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1);
  Ax Am = ax(Mi, g.A.s_ro, g.A.s_ri), Ak = ax(Ki, g.A.s_co, g.A.s_ci);
  Ax Bk = ax(Ki, g.B.s_ro, g.B.s_ri), Bn = ax(Ni, g.B.s_co, g.B.s_ci);
  Ax Cm = ax(Mi, g.C.s_ro, g.C.s_ri), Cn = ax(Ni, g.C.s_co, g.C.s_ci);
  Ax C2m = ax(Mi, g.C2.s_ro, g.C2.s_ri), C2n = ax(Ni, g.C2.s_co, g.C2.s_ci);
  auto split = [](const std::vector<double>& x, std::vector<double> (&s)[3], int& e) {
    double m = 0.0;
    for (double v : x) m = std::max(m, std::fabs(v));
    e = 0;
    if (m > 0.0) std::frexp(m, &e);
    for (auto& v : s) v.assign(x.size(), 0.0);
    for (size_t k = 0; k < x.size(); ++k) {
      double y = std::ldexp(x[k], -e) * 64.0;
      const double s1 = std::nearbyint(y);
      double t = (y - s1) * 2048.0;
      const double s2 = std::nearbyint(t);
      t = (t - s2) * 2048.0;
      s[0][k] = s1; s[1][k] = s2; s[2][k] = std::nearbyint(t);
    }
  };
  std::vector<std::vector<double>> as[3], bs[3];
  std::vector<int> ea(g.M), eb(g.N);
  for (auto& v : as) v.resize(g.M);
  for (auto& v : bs) v.resize(g.N);
  std::vector<double> row(g.K);
  for (int64_t m = 0; m < g.M; ++m) {
    for (int64_t k = 0; k < g.K; ++k) row[k] = g.A.p[Am.off(m) + Ak.off(k)];
    std::vector<double> s[3];
    split(row, s, ea[m]);
    for (int q = 0; q < 3; ++q) as[q][m] = s[q];
  }
  for (int64_t n = 0; n < g.N; ++n) {
    for (int64_t k = 0; k < g.K; ++k) row[k] = g.B.p[Bk.off(k) + Bn.off(n)];
    std::vector<double> s[3];
    split(row, s, eb[n]);
    for (int q = 0; q < 3; ++q) bs[q][n] = s[q];
  }
  const double w[3] = {0x1p-12, 0x1p-23, 0x1p-34};
  for (int64_t m = 0; m < g.M; ++m)
    for (int64_t n = 0; n < g.N; ++n) {
      double acc[3] = {0, 0, 0};
      for (int pa = 0; pa < 3; ++pa)
        for (int pb = 0; pb + pa < 3; ++pb) {
          double s = 0.0;
          const auto& x = as[pa][m];
          const auto& y = bs[pb][n];
          for (int64_t k = 0; k < g.K; ++k) s += x[k] * y[k];
          acc[pa + pb] += s;
        }
      const double v = g.alpha * std::ldexp(acc[0] * w[0] + acc[1] * w[1] + acc[2] * w[2], ea[m] + eb[n]);
      double* c = g.C.p + Cm.off(m) + Cn.off(n);
      *c = g.beta != 0.0 ? v + g.beta * *c : v;
      if (g.C2.p) {
        double* c2 = g.C2.p + C2m.off(m) + C2n.off(n);
        *c2 = g.beta != 0.0 ? v + g.beta * *c2 : v;
      }
    }
}

// Pre-packed B: the emulation keeps a dense copy B[n][k] of the operand's values
// and slices it again in gemm_split (same values, same slices).
size_t split_packed_b_bytes(const Contraction& g) { return size_t(g.N) * g.K * 8 + 64; }
size_t split_scratch_bytes_packed_b(const Contraction&) { return 64; }
bool split_single_panel(const Contraction& g) { return g.batch == 1; }

SplitPackedB split_pack_b(const Contraction& g, void* dst, cudaStream_t) {
  const int64_t Ni = g.Ni > 0 ? g.Ni : g.N, Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1);
  Ax Bk = ax(Ki, g.B.s_ro, g.B.s_ri), Bn = ax(Ni, g.B.s_co, g.B.s_ci);
  double* d = static_cast<double*>(dst);
  for (int64_t n = 0; n < g.N; ++n)
    for (int64_t k = 0; k < g.K; ++k) d[n * g.K + k] = g.B.p[Bk.off(k) + Bn.off(n)];
  SplitPackedB b;
  b.slices = dst; b.N = g.N; b.K = g.K; b.Np = g.N; b.Kp = g.K;
  g_pack += 2;
  return b;
}

void gemm_split_packed_b(const Contraction& g, const SplitPackedB& b, cudaStream_t s,
                         SplitScratch& ws) {
  if (b.N != g.N || b.K != g.K) throw Error(ERR_INVALID_ARGUMENT, "pre-packed B of another shape");
  const int64_t Ni = g.Ni > 0 ? g.Ni : g.N, Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1);
  Contraction h = g;   // B(k, n) = copy[n * K + k] in the contraction's two-level k and n
  h.B.p = static_cast<double*>(b.slices);
  h.B.s_ro = Ki; h.B.s_ri = 1; h.B.s_co = Ni * g.K; h.B.s_ci = g.K;
  gemm_split(h, s, ws);
  g_pack -= 2;  // B was sliced before
}

// Sliced operands: the emulation keeps the rows as a dense copy [R][K] and slices the
// rows a contraction reads again in gemm_split (same rows, same slices).
size_t split_operand_bytes(int64_t R, int64_t K) { return size_t(R) * K * 8 + 64; }

SplitOperand split_pack_operand(const double* src, int64_t R, int64_t Ri, int64_t s_ro,
                                int64_t s_ri, int64_t K, int64_t s_k, void* dst, cudaStream_t) {
  if (R <= 0 || K <= 0) throw Error(ERR_BAD_SHAPE, "split_pack_operand: empty operand");
  Ax r = ax(Ri > 0 ? Ri : R, s_ro, s_ri);
  double* d = static_cast<double*>(dst);
  for (int64_t i = 0; i < R; ++i)
    for (int64_t k = 0; k < K; ++k) d[i * K + k] = src[r.off(i) + k * s_k];
  SplitOperand o;
  o.slices = dst; o.R = R; o.K = K; o.Rp = R; o.Kp = K;
  g_pack += 2;
  return o;
}

void gemm_split_prepacked(const Contraction& g, const SplitOperand& A, const SplitRuns& ar,
                          const SplitOperand& B, const SplitRuns& br, cudaStream_t s,
                          SplitScratch& ws) {
  if (g.M <= 0 || g.N <= 0) return;
  if (A.K != g.K || B.K != g.K)
    throw Error(ERR_INVALID_ARGUMENT, "gemm_split_prepacked: operands of another K");
  const int64_t K = g.K;
  auto rows = [&](const SplitOperand& o, const SplitRuns& r, int64_t X) {
    if (r.run <= 0) throw Error(ERR_INVALID_ARGUMENT, "gemm_split_prepacked: bad runs");
    std::vector<double> d(size_t(X) * K);
    const double* src = static_cast<const double*>(o.slices);
    for (int64_t x = 0; x < X; ++x) {
      const int64_t pr = r.base + (x / r.run) * r.stride + x % r.run;
      if (pr < 0 || pr >= o.R)
        throw Error(ERR_INVALID_ARGUMENT, "gemm_split_prepacked: runs leave the operand");
      for (int64_t k = 0; k < K; ++k) d[x * K + k] = src[pr * K + k];
    }
    return d;
  };
  std::vector<double> Ad = rows(A, ar, g.M), Bd = rows(B, br, g.N);
  g_pack -= 4;  // nothing is sliced here on the device (gemm_split below counts four)
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  Contraction h = g;
  h.Ki = 0;
  h.A.p = Ad.data(); h.A.s_ro = Mi * K; h.A.s_ri = K; h.A.s_co = 0; h.A.s_ci = 1;
  h.B.p = Bd.data(); h.B.s_ro = 0; h.B.s_ri = 1; h.B.s_co = Ni * K; h.B.s_ci = K;
  gemm_split(h, s, ws);
}

// Plain-loop stand-in for the allocation-free energy entry (host pointers).
int energy_noalloc(const double* T1, const double* T2, const double* V, int64_t o, int64_t v,
                   int cplx, double* out, cudaStream_t, const char** err) {
  if (!T1 || !T2 || !V || !out) { *err = "null pointer"; return ERR_INVALID_ARGUMENT; }
  if (o <= 0 || v <= 0) { *err = "No and Nv must be positive"; return ERR_BAD_SHAPE; }
  if (o * o > 65536) { *err = "No too large"; return ERR_BAD_SHAPE; }
  double acc[4] = {0, 0, 0, 0};
  for (int64_t j = 0; j < o; ++j)
    for (int64_t i = 0; i < o; ++i)
      for (int64_t b = 0; b < v; ++b)
        for (int64_t a = 0; a < v; ++a) {
          const int64_t e = a + v * (b + v * (i + o * j)), ex = b + v * (a + v * (i + o * j));
          const int64_t ai = a + v * i, bj = b + v * j;
          if (!cplx) {
            const double x = T2[e] + T1[ai] * T1[bj];
            acc[0] += x * V[e];
            acc[1] += x * V[ex];
          } else {
            const double xr = T2[2 * e] + T1[2 * ai] * T1[2 * bj] - T1[2 * ai + 1] * T1[2 * bj + 1];
            const double xi = T2[2 * e + 1] + T1[2 * ai] * T1[2 * bj + 1] + T1[2 * ai + 1] * T1[2 * bj];
            acc[0] += xr * V[2 * e] + xi * V[2 * e + 1];
            acc[1] += xr * V[2 * ex] + xi * V[2 * ex + 1];
            acc[2] += xi * V[2 * e] - xr * V[2 * e + 1];
            acc[3] += xi * V[2 * ex] - xr * V[2 * ex + 1];
          }
        }
  out[0] = 2 * acc[0]; out[1] = -acc[1]; out[2] = 2 * acc[2]; out[3] = -acc[3];
  return OK;
}

namespace ops {

double* alloc(size_t elems) {
  void* p = std::calloc(elems ? elems : 1, sizeof(double));
  if (!p) throw Error(ERR_OUT_OF_MEMORY, "host allocation failed");
  return static_cast<double*>(p);
}
void release(void* p) { std::free(p); }
void zero(double* p, size_t n, Stream) { std::memset(p, 0, n * sizeof(double)); }
void h2d(double* d, const double* s, size_t n, Stream) { std::memcpy(d, s, n * sizeof(double)); }
void d2h(double* d, const double* s, size_t n, Stream) { std::memcpy(d, s, n * sizeof(double)); }
void d2d(double* d, const double* s, size_t n, Stream) { std::memmove(d, s, n * sizeof(double)); }
void sync(Stream) {}
Stream stream_create(int) { return nullptr; }
void stream_destroy(Stream) {}
void* event_create() { return nullptr; }
void event_record(void*, Stream) {}
float event_ms(void*, void*) { return 0.f; }
void event_destroy(void*) {}
uint64_t launch_count() { return g_ops; }

void permute4(double* dst, const double* src, const int64_t d[4], const int perm[4],
              double alpha, double beta, Stream) {
  ++g_ops;
  int64_t ss[4];
  ss[3] = 1;
  for (int k = 2; k >= 0; --k) ss[k] = ss[k + 1] * d[k + 1];
  int64_t e[4], es[4];
  for (int k = 0; k < 4; ++k) { e[k] = d[perm[k]]; es[k] = ss[perm[k]]; }
  int64_t o = 0;
  for (int64_t i0 = 0; i0 < e[0]; ++i0)
    for (int64_t i1 = 0; i1 < e[1]; ++i1)
      for (int64_t i2 = 0; i2 < e[2]; ++i2)
        for (int64_t i3 = 0; i3 < e[3]; ++i3, ++o) {
          const double v = alpha * src[i0 * es[0] + i1 * es[1] + i2 * es[2] + i3 * es[3]];
          dst[o] = beta != 0.0 ? v + beta * dst[o] : v;
        }
}

void copy4(double* dst, const int64_t ds[4], const double* src, const int64_t ss[4],
           const int64_t e[4], double alpha, double beta, Stream) {
  ++g_ops;
  if (ds[3] != 1) throw Error(ERR_STATE, "copy4: the destination's inner stride must be 1");
  for (int64_t i0 = 0; i0 < e[0]; ++i0)
    for (int64_t i1 = 0; i1 < e[1]; ++i1)
      for (int64_t i2 = 0; i2 < e[2]; ++i2)
        for (int64_t i3 = 0; i3 < e[3]; ++i3) {
          const double v = alpha * src[i0 * ss[0] + i1 * ss[1] + i2 * ss[2] + i3 * ss[3]];
          double* d = dst + i0 * ds[0] + i1 * ds[1] + i2 * ds[2] + i3;
          *d = beta != 0.0 ? v + beta * *d : v;
        }
}

void axpby(double* out, double a, const double* x, double b, const double* y, double c,
           int64_t n, Stream) {
  ++g_ops;
  for (int64_t e = 0; e < n; ++e) {
    double v = a * x[e];
    if (y) v += b * y[e];
    if (c != 0.0) v += c * out[e];
    out[e] = v;
  }
}

void rank1(double* out, double a, const double* A, double b, const double* t, int64_t n,
           Stream) {
  ++g_ops;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) out[r * n + c] = a * A[r * n + c] + b * t[r] * t[c];
}

void zrank1(double* ore, double* oim, const double* are, const double* aim, const double* tre,
            const double* tim, double b, int64_t n, Stream) {
  ++g_ops;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = 0; c < n; ++c) {
      const int64_t e = r * n + c;
      const double xr = tre[r] * tre[c] - tim[r] * tim[c];
      const double xi = tre[r] * tim[c] + tim[r] * tre[c];
      ore[e] = are[e] + b * xr;
      oim[e] = aim[e] + b * xi;
    }
}

void symmetrize(double* R, int64_t n, Stream) {
  ++g_ops;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t c = r; c < n; ++c) {
      const double s = R[r * n + c] + R[c * n + r];
      R[r * n + c] = s;
      R[c * n + r] = s;
    }
}

void gather_vertex(double* out, const double* in, bool cplx, int part, int64_t NG, int64_t Np,
                   int64_t row0, int64_t nx, int64_t col0, int64_t ny, Stream) {
  ++g_ops;
  const int64_t es = cplx ? 2 : 1;
  for (int64_t g = 0; g < NG; ++g)
    for (int64_t x = 0; x < nx; ++x)
      for (int64_t y = 0; y < ny; ++y)
        out[(g * nx + x) * ny + y] = in[(g + NG * ((row0 + x) + Np * (col0 + y))) * es + part];
}

void jacobi(double* Tnew, double* dT, const double* R, const double* Told, const double* eh,
            const double* ep, const AmpShape& sh, double shift, Stream) {
  ++g_ops;
  const int64_t n1 = sh.n1();
  for (int64_t e = 0; e < sh.total(); ++e) {
    const int64_t q = e % sh.plane();
    double D;
    if (q < n1) {
      D = ep[q / sh.o] - eh[q % sh.o];
    } else {
      const int64_t r = q - n1, ai = r / n1, bj = r % n1;
      D = ep[ai / sh.o] - eh[ai % sh.o] + ep[bj / sh.o] - eh[bj % sh.o];
    }
    double rv = R[e];
    const double told = Told ? Told[e] : 0.0;
    if (Told && shift != 0.0) rv -= shift * told;
    const double tn = rv * (-1.0 / (D + shift));
    Tnew[e] = tn;
    dT[e] = Told ? tn - told : tn;
  }
}

void mp2_energy(const double* Vr, const double* Vi, const double* eh, const double* ep,
                int64_t o, int64_t v, double* out, double*, Stream) {
  ++g_ops;
  const int64_t n1 = v * o;
  double acc[2] = {0, 0};
  for (int64_t r = 0; r < n1; ++r)
    for (int64_t c = 0; c < n1; ++c) {
      const int64_t e = r * n1 + c, a = r / o, i = r % o, b = c / o, j = c % o;
      const double d = eh[i] + eh[j] - ep[a] - ep[b];
      const int64_t ex = (a * o + j) * n1 + b * o + i;
      acc[0] += (Vr[e] * Vr[e] + (Vi ? Vi[e] * Vi[e] : 0.0)) / d;
      acc[1] += (Vr[e] * Vr[ex] + (Vi ? Vi[e] * Vi[ex] : 0.0)) / d;
    }
  out[0] = 2.0 * acc[0];
  out[1] = -acc[1];
}

void energy(const double* T, const double* Vdr, const double* Vdi, const double* Ver,
            const double* Vei, const AmpShape& sh, double* out, double*, Stream) {
  ++g_ops;
  const int64_t n1 = sh.n1();
  const double* t1r = T;
  const double* t2r = T + n1;
  const double* t1i = sh.planes > 1 ? T + sh.plane() : nullptr;
  const double* t2i = sh.planes > 1 ? T + sh.plane() + n1 : nullptr;
  double acc[4] = {0, 0, 0, 0};
  for (int64_t r = 0; r < n1; ++r)
    for (int64_t c = 0; c < n1; ++c) {
      const int64_t e = r * n1 + c;
      // V_baij = Vd[(b,i),(a,j)] when no exchange tensor is given
      const int64_t ex = ((c / sh.o) * sh.o + r % sh.o) * n1 + (r / sh.o) * sh.o + c % sh.o;
      if (!t1i) {
        const double x = t2r[e] + t1r[r] * t1r[c];
        acc[0] += x * Vdr[e];
        acc[1] += x * (Ver ? Ver[e] : Vdr[ex]);
      } else {
        const double xr = t2r[e] + t1r[r] * t1r[c] - t1i[r] * t1i[c];
        const double xi = t2i[e] + t1r[r] * t1i[c] + t1i[r] * t1r[c];
        const double vdi = Vdi ? Vdi[e] : 0.0;
        const double ver = Ver ? Ver[e] : Vdr[ex];
        const double vei = Ver ? (Vei ? Vei[e] : 0.0) : (Vdi ? Vdi[ex] : 0.0);
        acc[0] += xr * Vdr[e] + xi * vdi;
        acc[1] += xr * ver + xi * vei;
        acc[2] += xi * Vdr[e] - xr * vdi;
        acc[3] += xi * ver - xr * vei;
      }
    }
  out[0] = 2.0 * acc[0]; out[1] = -acc[1]; out[2] = 2.0 * acc[2]; out[3] = -acc[3];
}

void dots(const double* x, const double* const* ys, int ny, int64_t n, double* out, double*,
          Stream) {
  ++g_ops;
  for (int k = 0; k < ny; ++k) {
    double s = 0.0;
    for (int64_t e = 0; e < n; ++e) s += x[e] * ys[k][e];
    out[k] = s;
  }
}

void diis_solve(double* B, const double* dots_dev, const int* valid, int N, int next, int count,
                double* coef, int* status, Stream) {
  ++g_ops;
  const int M = N + 1;
  int di = 0;
  for (int i = 0; i < N; ++i) {
    if (!valid[i]) continue;
    const double ov = 2.0 * dots_dev[di++];
    B[(i + 1) * M + next + 1] = ov;
    B[(next + 1) * M + i + 1] = ov;
  }
  const int dim = count + 1;
  std::vector<double> m(dim * dim), x(dim, 0.0);
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) m[r * dim + c] = B[r * M + c];
  x[0] = -1.0;
  int singular = 0;
  for (int k = 0; k < dim; ++k) {
    int piv = k;
    double best = std::fabs(m[k * dim + k]);
    for (int r = k + 1; r < dim; ++r)
      if (std::fabs(m[r * dim + k]) > best) { best = std::fabs(m[r * dim + k]); piv = r; }
    if (!std::isfinite(best)) { singular = 2; break; }
    if (best == 0.0) { singular = 1; break; }
    if (piv != k) {
      for (int c = 0; c < dim; ++c) std::swap(m[k * dim + c], m[piv * dim + c]);
      std::swap(x[k], x[piv]);
    }
    for (int r = k + 1; r < dim; ++r) {
      const double f = m[r * dim + k] / m[k * dim + k];
      for (int c = k; c < dim; ++c) m[r * dim + c] -= f * m[k * dim + c];
      x[r] -= f * x[k];
    }
  }
  if (!singular) {
    for (int k = dim - 1; k >= 0; --k) {
      double s = x[k];
      for (int c = k + 1; c < dim; ++c) s -= m[k * dim + c] * x[c];
      x[k] = s / m[k * dim + k];
    }
    for (int j = 0; j < count; ++j) coef[j] = x[(next + N - j) % N + 1];
  }
  status[0] = singular;
}

void lincomb(double* out, const double* const* xs, const double* const* ys, const double* coef,
             int nx, int64_t n, double* norm2, double*, Stream) {
  ++g_ops;
  double s2 = 0.0;
  for (int64_t e = 0; e < n; ++e) {
    double v = 0.0, w = 0.0;
    for (int k = 0; k < nx; ++k) {
      v += coef[k] * xs[k][e];
      if (ys) w += coef[k] * ys[k][e];
    }
    out[e] = v;
    s2 += w * w;
  }
  if (ys && norm2) norm2[0] = s2;
}

void sum_partials_to(double* dst, const double* ws, int nparts, int nvals, Stream) {
  ++g_ops;
  for (int k = 0; k < nvals; ++k) {
    double v = 0.0;
    for (int b = 0; b < nparts; ++b) v += ws[b * nvals + k];
    dst[k] = v;
  }
}

int scan_vertex(const double* p, int64_t n, bool complex_values, Stream) {
  ++g_ops;
  int f = 0;
  for (int64_t e = 0; e < n; ++e) {
    if (!std::isfinite(p[e])) f |= 1;
    if (complex_values && (e & 1) && p[e] != 0.0) f |= 2;
  }
  return f;
}

// Packed amplitude vectors: per plane [T1 | T2 rows r, columns r..n1-1].
static int64_t packed_index(const AmpShape& sh, int64_t pl, int64_t r, int64_t c) {
  const int64_t n1 = sh.n1();
  return pl * sh.packed_plane() + n1 + r * n1 - r * (r - 1) / 2 + (c - r);
}

void jacobi_packed(double* Tnew, double* dT, const double* R, const double* Told,
                   const double* eh, const double* ep, const AmpShape& sh, double shift,
                   Stream) {
  ++g_ops;
  const int64_t n1 = sh.n1();
  auto upd = [&](int64_t full, int64_t pk, double D) {
    double rv = R[full];
    const double told = Told ? Told[full] : 0.0;
    if (Told && shift != 0.0) rv -= shift * told;
    const double tn = rv * (-1.0 / (D + shift));
    Tnew[pk] = tn;
    dT[pk] = Told ? tn - told : tn;
  };
  for (int64_t pl = 0; pl < sh.planes; ++pl) {
    for (int64_t ai = 0; ai < n1; ++ai)
      upd(pl * sh.plane() + ai, pl * sh.packed_plane() + ai, ep[ai / sh.o] - eh[ai % sh.o]);
    for (int64_t r = 0; r < n1; ++r)
      for (int64_t c = r; c < n1; ++c)
        upd(pl * sh.plane() + n1 + r * n1 + c, packed_index(sh, pl, r, c),
            ep[r / sh.o] - eh[r % sh.o] + ep[c / sh.o] - eh[c % sh.o]);
  }
}

void dots_packed(const double* x, const double* const* ys, int ny, const AmpShape& sh,
                 double* out, double*, Stream) {
  ++g_ops;
  const int64_t n1 = sh.n1();
  for (int k = 0; k < ny; ++k) {
    double s = 0.0;
    for (int64_t pl = 0; pl < sh.planes; ++pl) {
      for (int64_t ai = 0; ai < n1; ++ai) {
        const int64_t e = pl * sh.packed_plane() + ai;
        s += x[e] * ys[k][e];
      }
      for (int64_t r = 0; r < n1; ++r)
        for (int64_t c = r; c < n1; ++c) {
          const int64_t e = packed_index(sh, pl, r, c);
          s += (c == r ? 1.0 : 2.0) * x[e] * ys[k][e];
        }
    }
    out[k] = s;
  }
}

void lincomb_packed(double* out, const double* const* xs, const double* const* ys,
                    const double* coef, int nx, const AmpShape& sh, double* norm2, double*,
                    Stream) {
  ++g_ops;
  const int64_t n1 = sh.n1();
  double s2 = 0.0;
  auto comb = [&](int64_t pk, double& w) {
    double v = 0.0;
    w = 0.0;
    for (int k = 0; k < nx; ++k) {
      v += coef[k] * xs[k][pk];
      if (ys) w += coef[k] * ys[k][pk];
    }
    return v;
  };
  for (int64_t pl = 0; pl < sh.planes; ++pl) {
    double* ob = out + pl * sh.plane();
    for (int64_t ai = 0; ai < n1; ++ai) {
      double w;
      ob[ai] = comb(pl * sh.packed_plane() + ai, w);
      s2 += w * w;
    }
    for (int64_t r = 0; r < n1; ++r)
      for (int64_t c = r; c < n1; ++c) {
        double w;
        const double v = comb(packed_index(sh, pl, r, c), w);
        ob[n1 + r * n1 + c] = v;
        ob[n1 + c * n1 + r] = v;
        s2 += (c == r ? 1.0 : 2.0) * w * w;
      }
  }
  if (ys && norm2) norm2[0] = s2;
}


void fsc_prepare_u(double* ore, double* oim, const double* U, const double* V, int64_t NGG,
                   int64_t NF, Stream) {
  ++g_ops;
  for (int64_t G = 0; G < NGG; ++G)
    for (int64_t F = 0; F < NF; ++F) {
      const int64_t e = F * NGG + G;
      const double re = U ? U[2 * e] : (G == F ? 1.0 : 0.0), im = U ? U[2 * e + 1] : 0.0;
      const double sc = V ? 1.0 / std::sqrt(V[G]) : 1.0;
      ore[G * NF + F] = re * sc;
      oim[G * NF + F] = im * sc;
    }
}

void fsc_stacked_to_complex(double* Qr, double* Qi, const double* Qs, int64_t NF, int parts,
                            Stream) {
  ++g_ops;
  const int64_t S2 = parts * NF;
  for (int64_t F = 0; F < NF; ++F)
    for (int64_t Fp = 0; Fp < NF; ++Fp) {
      const int64_t e = F * NF + Fp;
      if (parts == 2) {
        Qr[e] = Qs[F * S2 + Fp] + Qs[(F + NF) * S2 + Fp + NF];
        Qi[e] = Qs[F * S2 + Fp + NF] - Qs[(F + NF) * S2 + Fp];
      } else {
        Qr[e] = Qs[e];
        Qi[e] = 0.0;
      }
    }
}

static void fsc_direct_emu(const FscGeometry& g, const double v[3], double x[3]) {
  for (int d = 0; d < 3; ++d) x[d] = g.A[3 * d] * v[0] + g.A[3 * d + 1] * v[1] + g.A[3 * d + 2] * v[2];
}

void fsc_box(double* box, const double* S, const double* grid, const FscGeometry& g, Stream) {
  ++g_ops;
  std::memset(box, 0, sizeof(double) * g.dims[0] * g.dims[1] * g.dims[2]);
  for (int64_t e = 0; e < g.NG; ++e) {
    double x[3];
    fsc_direct_emu(g, grid + 3 * e, x);
    int64_t i[3];
    bool in = true;
    for (int d = 0; d < 3; ++d) {
      i[d] = static_cast<int64_t>(std::floor(x[d] + 0.5) - g.origin[d]);
      in = in && i[d] >= 0 && i[d] < g.dims[d];
    }
    if (in) box[i[0] + g.dims[0] * (i[1] + g.dims[1] * i[2])] = S[e];
  }
}

static double fsc_tricubic_emu(const double* box, const FscGeometry& g, const double x[3]) {
  static const double BL[4][4] = {{0.0, -0.5, 1.0, -0.5}, {1.0, 0.0, -2.5, 1.5},
                                  {0.0, 0.5, 2.0, -1.5}, {0.0, 0.0, -0.5, 0.5}};
  double w[3][4];
  int64_t base[3];
  for (int d = 0; d < 3; ++d) {
    const double t = x[d] - g.origin[d];
    int64_t i = static_cast<int64_t>(t);
    i = std::min<int64_t>(std::max<int64_t>(i, 0), g.dims[d] - 1);
    const double u = t - static_cast<double>(i);
    for (int r = 0; r < 4; ++r) w[d][r] = BL[r][0] + BL[r][1] * u + BL[r][2] * u * u + BL[r][3] * u * u * u;
    base[d] = i - 1;
  }
  auto cl = [](int64_t a, int64_t n) { return std::min<int64_t>(std::max<int64_t>(a, 0), n - 1); };
  double total = 0.0;
  for (int sl = 0; sl < 4; ++sl)
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c)
        total += w[0][c] * w[1][r] * w[2][sl] *
                 box[cl(base[0] + c, g.dims[0]) +
                     g.dims[0] * (cl(base[1] + r, g.dims[1]) + g.dims[1] * cl(base[2] + sl, g.dims[2]))];
  return total;
}

void fsc_sums(const double* box, const double* S, const double* grid, const FscGeometry& g,
              double*, double* out, Stream) {
  ++g_ops;
  double acc0 = 0.0, acc1 = 0.0;
  for (int64_t e = 0; e < g.NG; ++e) {
    const double* v = grid + 3 * e;
    const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (std::sqrt(n2) >= 1e-8) acc0 += g.f / n2 * S[e];
  }
  const int64_t n2N = 2 * static_cast<int64_t>(g.N);
  const double inv2N = 1.0 / static_cast<double>(n2N);
  for (int64_t a = -g.N; a < g.N; ++a)
    for (int64_t b = -g.N; b < g.N; ++b)
      for (int64_t c = -g.N; c < g.N; ++c)
        for (int64_t i = 0; i < g.NG; ++i) {
          double v[3];
          for (int d = 0; d < 3; ++d)
            v[d] = g.B[d] * inv2N * double(a) + g.B[3 + d] * inv2N * double(b) +
                   g.B[6 + d] * inv2N * double(c) + grid[3 * i + d];
          const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
          if (std::sqrt(n2) < 1e-8) continue;
          double x[3];
          fsc_direct_emu(g, v, x);
          acc1 += g.f * fsc_tricubic_emu(box, g, x) / n2;
        }
  out[0] = acc0;
  out[1] = acc1;
}

struct TriplesC { double re, im; };

static TriplesC triples_singles_at(const double* t, const double* ti, const double* V,
                                   const double* Vi, int64_t n1, int64_t p1, int64_t p2,
                                   int64_t p3) {
  const int64_t pr[3][3] = {{p1, p2, p3}, {p2, p1, p3}, {p3, p1, p2}};  // t index, V row, V col
  TriplesC s{0.0, 0.0};
  for (const auto& k : pr) {
    const double tr = t[k[0]], tm = ti ? ti[k[0]] : 0.0;
    const double vr = V[k[1] * n1 + k[2]], vm = Vi ? Vi[k[1] * n1 + k[2]] : 0.0;
    s.re += tr * vr - tm * vm;
    s.im += tr * vm + tm * vr;
  }
  return s;
}

void triples_singles(double* S, double* S_im, const double* t1, const double* t1_im,
                     const double* V, const double* V_im, const TriplesBlock& b, Stream) {
  ++g_ops;
  for (int64_t q1 = 0; q1 < b.L[0]; ++q1)
    for (int64_t q2 = 0; q2 < b.L[1]; ++q2)
      for (int64_t q3 = 0; q3 < b.L[2]; ++q3) {
        const int64_t e = (q1 * b.L[1] + q2) * b.L[2] + q3;
        const TriplesC x = triples_singles_at(t1, t1_im, V, V_im, b.n1, b.P[0] + q1,
                                              b.P[1] + q2, b.P[2] + q3);
        S[e] = x.re;
        if (S_im) S_im[e] = x.im;
      }
}

void triples_energy(const double* S, const double* S_im, const double* t1, const double* t1_im,
                    const double* V, const double* V_im, const double* eh, const double* ep,
                    const TriplesBlock& b, const double coef[6], double*, double* out, Stream,
                    const double* M, const double* M_im) {
  ++g_ops;
  static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  const int64_t o = b.o;
  double acc[2] = {0.0, 0.0};
  for (int64_t q1 = 0; q1 < b.L[0]; ++q1)
    for (int64_t q2 = 0; q2 < b.L[1]; ++q2)
      for (int64_t q3 = 0; q3 < b.L[2]; ++q3) {
        const int64_t x[3] = {q1 / o, q2 / o, q3 / o};
        const int64_t y[3] = {q1 % o, q2 % o, q3 % o};
        auto at = [&](const double* A, int64_t r1, int64_t r2, int64_t r3) {
          return A[(r1 * b.L[1] + r2) * b.L[2] + r3];
        };
        const TriplesC sg = triples_singles_at(t1, t1_im, V, V_im, b.n1, b.P[0] + q1,
                                               b.P[1] + q2, b.P[2] + q3);
        double d = 0.0;
        for (int m = 0; m < 3; ++m) d += eh[y[m]] - ep[b.P[m] / o + x[m]];
        double yr = 0.0, yi = 0.0;
        for (int k = 0; k < 6; ++k) {
          const int64_t r1 = x[0] * o + y[perm[k][0]], r2 = x[1] * o + y[perm[k][1]],
                        r3 = x[2] * o + y[perm[k][2]];
          yr += coef[k] * at(S, r1, r2, r3);
          if (S_im) yi += coef[k] * at(S_im, r1, r2, r3);
        }
        const double wr = M ? at(M, q1, q2, q3) : at(S, q1, q2, q3) - sg.re;
        acc[0] += wr * yr / d;
        if (S_im) acc[1] += (M ? at(M_im, q1, q2, q3) : at(S_im, q1, q2, q3) - sg.im) * yi / d;
      }
  out[0] = acc[0];
  out[1] = acc[1];
}

void triples_cr_sums(const double* S, const double* S_im, const double* t1, const double* t1_im,
                     const double* T2, const double* T2_im, const double* eh, const double* ep,
                     const TriplesBlock& b, const double coef[6], double*, double* out, Stream) {
  ++g_ops;
  static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  const int64_t o = b.o;
  double acc[2] = {0.0, 0.0};
  for (int64_t q1 = 0; q1 < b.L[0]; ++q1)
    for (int64_t q2 = 0; q2 < b.L[1]; ++q2)
      for (int64_t q3 = 0; q3 < b.L[2]; ++q3) {
        const int64_t x[3] = {q1 / o, q2 / o, q3 / o};
        const int64_t y[3] = {q1 % o, q2 % o, q3 % o};
        auto at = [&](const double* A, int64_t r1, int64_t r2, int64_t r3) {
          return A[(r1 * b.L[1] + r2) * b.L[2] + r3];
        };
        const int64_t p[3] = {b.P[0] + q1, b.P[1] + q2, b.P[2] + q3};
        const TriplesC ts = triples_singles_at(t1, t1_im, T2, T2_im, b.n1, p[0], p[1], p[2]);
        double pr = t1[p[0]], pi = t1_im ? t1_im[p[0]] : 0.0;
        for (int m = 1; m < 3; ++m) {
          const double r = t1[p[m]], i = t1_im ? t1_im[p[m]] : 0.0;
          const double nr = pr * r - pi * i, ni = pr * i + pi * r;
          pr = nr; pi = ni;
        }
        double d = 0.0;
        for (int m = 0; m < 3; ++m) d += eh[y[m]] - ep[b.P[m] / o + x[m]];
        double zr = 0.0, zi = 0.0;
        for (int k = 0; k < 6; ++k) {
          const int64_t r1 = x[0] * o + y[perm[k][0]], r2 = x[1] * o + y[perm[k][1]],
                        r3 = x[2] * o + y[perm[k][2]];
          zr += coef[k] * at(S, r1, r2, r3);
          if (S_im) zi += coef[k] * at(S_im, r1, r2, r3);
        }
        acc[0] += (ts.re + pr) * zr / d;
        if (S_im) acc[1] += (ts.im + pi) * zi / d;
      }
  out[0] = acc[0];
  out[1] = acc[1];
}

}  // namespace ops
}  // namespace cc4s_b200
