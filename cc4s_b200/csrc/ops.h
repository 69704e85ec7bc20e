// Device operations used by the CoupledCluster schedule.
//
// The CCSD schedule (ccsd_real.cpp) and the iteration driver (driver.cpp) are
// written against this interface only.  The product library implements it with
// CUDA kernels for sm_100a (ops_cuda.cu, gemm_f64.cu).
#pragma once

#include "gemm_f64.cuh"

namespace cc4s_b200 {

using Stream = cudaStream_t;

namespace ops {

// ---- memory ---------------------------------------------------------------
double* alloc(size_t elems);  // throws Error(ERR_OUT_OF_MEMORY) on failure
void release(void* p);
void zero(double* p, size_t elems, Stream s);
void h2d(double* dst, const double* src, size_t elems, Stream s);
void d2h(double* dst, const double* src, size_t elems, Stream s);
void d2d(double* dst, const double* src, size_t elems, Stream s);
void sync(Stream s);
Stream stream_create(int device);
void stream_destroy(Stream s);
void* event_create();
void event_record(void* e, Stream s);
float event_ms(void* start, void* stop);  // synchronises on stop
void event_destroy(void* e);

// ---- bandwidth kernels ----------------------------------------------------
// dst = alpha * permute(src) + beta * dst.  src is row-major with dims d[0..3];
// destination axis k is source axis perm[k].
void permute4(double* dst, const double* src, const int64_t d[4], const int perm[4],
              double alpha, double beta, Stream s);
// Strided 4-index copy: dst[i] = alpha * src[i] + beta * dst[i] over the extents e,
// element i at sum_k i_k ss[k] in src and sum_k i_k ds[k] in dst (ds[3] == 1).
void copy4(double* dst, const int64_t ds[4], const double* src, const int64_t ss[4],
           const int64_t e[4], double alpha, double beta, Stream s);
// out = a*x + b*y + c*out   (y may be null; c == 0 does not read out)
void axpby(double* out, double a, const double* x, double b, const double* y, double c,
           int64_t n, Stream s);
// out[r][c] = a*A[r][c] + b*t[r]*t[c] for an n x n matrix (A may alias out).
void rank1(double* out, double a, const double* A, double b, const double* t, int64_t n,
           Stream s);
// Complex planar version: out = A + b * t t^T (no conjugation); out may alias A.
void zrank1(double* out_re, double* out_im, const double* A_re, const double* A_im,
            const double* t_re, const double* t_im, double b, int64_t n, Stream s);
// R <- R + R^T for an n x n matrix, in place.
void symmetrize(double* R, int64_t n, Stream s);

// Gathers one block of the input Coulomb vertex into a row-major [NG][nx][ny] array:
//   out[g][x][y] = part(Gamma(g, row0 + x, col0 + y)),
// where the input is column-major Gamma[NG][Np][Np] (G fastest), real (part 0 only)
// or complex interleaved (part 0 = real, 1 = imaginary).
void gather_vertex(double* out, const double* in, bool in_complex, int part, int64_t NG,
                   int64_t Np, int64_t row0, int64_t nx, int64_t col0, int64_t ny, Stream s);

// Scans n doubles of a device vector (complex interleaved when complex_values):
// returns bit 0 if any is not finite, bit 1 if any imaginary part is non-zero.
int scan_vertex(const double* p, int64_t n, bool complex_values, Stream s);

// Amplitude vectors: [T1 (v x o, row-major [a][i]) | T2 ((v o) x (v o), row-major [a][i][b][j])],
// repeated once per plane (real plane, then imaginary plane for complex systems).
struct AmpShape {
  int64_t o, v, planes;
  int64_t n1() const { return v * o; }
  int64_t plane() const { return v * o + (v * o) * (v * o); }
  int64_t total() const { return plane() * planes; }
  // Packed form (DIIS history): T2 is a symmetric (vo) x (vo) matrix
  // (T_abij = T_baji), so each plane keeps [T1 | rows r of T2, columns r..n1-1].
  int64_t packed_plane() const { return n1() + n1() * (n1() + 1) / 2; }
  int64_t packed_total() const { return packed_plane() * planes; }
};

// Jacobi update of CoupledCluster::residuumToAmplitudes:
//   Tnew = -(R - shift*Told) / (D + shift),  dT = Tnew - Told   (Told may be null)
// with D_ai = ep[a]-eh[i], D_abij = ep[a]+ep[b]-eh[i]-eh[j].
void jacobi(double* Tnew, double* dT, const double* R, const double* Told, const double* eh,
            const double* ep, const AmpShape& sh, double shift, Stream s);

// The same update written into packed slots (AmpShape::packed_*): R and Told are
// full amplitude vectors with symmetric T2 parts; only their upper triangles are read.
void jacobi_packed(double* Tnew_p, double* dT_p, const double* R, const double* Told,
                   const double* eh, const double* ep, const AmpShape& sh, double shift,
                   Stream s);

// Correlation energy of amplitudes T (AmpShape layout) with the pair-layout integrals
// Vd[(a,i),(b,j)] = V_abij and Ve[(a,i),(b,j)] = V_abji (real and optional imaginary planes).
// Ve_re == nullptr: the exchange integrals are read from Vd itself,
// V_baij = Vd[(b,i),(a,j)] (for real integrals this equals V_abji).
// Writes 4 doubles to out_dev: Re(direct), Re(exchange), Im(direct), Im(exchange).
void energy(const double* T, const double* Vd_re, const double* Vd_im, const double* Ve_re,
            const double* Ve_im, const AmpShape& sh, double* out_dev, double* ws, Stream s);

// Second-order (MP2) energy of the integrals V_abij (pair layout, planar complex
// when Vd_im is given), PerturbativeTriplesStar.hpp:79-99:
//   out_dev[0] = 2 sum Re(conj(V_abij) V_abij) / D_abij,
//   out_dev[1] =  -sum Re(conj(V_abij) V_abji) / D_abij,
// D_abij = eps_i + eps_j - eps_a - eps_b; deterministic order.
void mp2_energy(const double* Vd_re, const double* Vd_im, const double* eh, const double* ep,
                int64_t o, int64_t v, double* out_dev, double* ws, Stream s);

// out_dev[k] = sum_e x[e] * ys[k][e] for k < ny (ny <= 8), deterministic order.
void dots(const double* x, const double* const* ys, int ny, int64_t n, double* out_dev,
          double* ws, Stream s);

// DIIS (DiisMixer.cxx:59-107) on the device:
//   B (device, (N+1)^2, row-major) receives the new overlaps 2*dots[i] at
//   (i+1, next+1) and (next+1, i+1) for the valid slots listed in valid[];
//   the (count+1)^2 corner is solved for rhs (-1, 0, ...) and coef_dev[j]
//   receives the coefficient of slot (next + N - j) % N, j < count.
//   status_dev[0] = 0 on success, 1 if the system is singular (zero pivot),
//   2 if it holds a non-finite entry.
void diis_solve(double* B, const double* dots_dev, const int* valid_host, int N, int next,
                int count, double* coef_dev, int* status_dev, Stream s);

// out = sum_j coef[j] * xs[j]; if ys != null also norm2_out = |sum_j coef[j] ys[j]|^2
// (written to norm2_dev).  Coefficients are read from device memory.
void lincomb(double* out, const double* const* xs, const double* const* ys,
             const double* coef_dev, int nx, int64_t n, double* norm2_dev, double* ws,
             Stream s);

// Packed counterparts of dots and lincomb: the vectors x, ys[k], xs[j] are packed
// (AmpShape::packed_*) and stand for the full symmetric vectors they represent, so
// off-diagonal T2 entries count twice in dot products and norms.  lincomb_packed
// writes the full vector out (both triangles).
void dots_packed(const double* x, const double* const* ys, int ny, const AmpShape& sh,
                 double* out_dev, double* ws, Stream s);
void lincomb_packed(double* out, const double* const* xs, const double* const* ys,
                    const double* coef_dev, int nx, const AmpShape& sh, double* norm2_dev,
                    double* ws, Stream s);

// Small host-visible scalars.
void sum_partials_to(double* dst_dev, const double* ws, int nparts, int nvals, Stream s);

// ---- finite-size correction ---------------------------------------------------
// Planar singular vectors for the structure factor: out_re/out_im [NGG][NF] =
// U[G,F] / sqrt(V[G]) from the caller's column-major complex-interleaved U[G,F]
// (U == null: the identity, NGG == NF; V == null: 1).
void fsc_prepare_u(double* out_re, double* out_im, const double* U, const double* V,
                   int64_t NGG, int64_t NF, Stream s);
// Complex NF x NF matrix from the stacked real one of the real path: rows and
// columns [0, NF) hold the real parts, [NF, 2 NF) the imaginary parts of the
// vertex rows (parts == 2; parts == 1: no imaginary rows):
//   Q = Qs[F][F'] + Qs[F+][F'+] + i (Qs[F][F'+] - Qs[F+][F']).
void fsc_stacked_to_complex(double* Q_re, double* Q_im, const double* Qs, int64_t NF, int parts,
                            Stream s);
// Lattice box of the interpolation: box[x + nx (y + ny z)] = S[g] at the integer
// coordinates round(A . G_g) - origin of each grid vector (other points 0).
struct FscGeometry {
  double A[9];      // rows: inverse of the reciprocal basis (direct coordinates)
  double B[9];      // rows: the reciprocal basis Gi, Gj, Gk
  double origin[3];
  int64_t dims[3];
  int64_t NG;       // grid vectors
  int N;            // interpolationGridSize
  double f;         // Omega / (2 pi^2) times the unit factors
};
void fsc_box(double* box, const double* S, const double* grid, const FscGeometry& g, Stream s);
// out_dev[0] = sum_{|G| >= 1e-8} f S(G) / |G|^2 (uncorrected),
// out_dev[1] = sum over the (2N)^3 NG refined points g != 0 of f S_int(A.g) / |g|^2,
// S_int the Catmull-Rom tricubic interpolation of the box.  ws >= 2 * 148 * 4 doubles.
void fsc_sums(const double* box, const double* S, const double* grid, const FscGeometry& g,
              double* ws, double* out_dev, Stream s);

// ---- perturbative triples ---------------------------------------------------
// One block of the (T) loop: virtual indices a, b, c from three blocks, all
// holes.  The block array is S[q1][q2][q3] with q = local pair index x*o + y
// (x the virtual index within its block, y the hole index); pair q of position
// m is the global pair P[m] + q (= (a, i) -> a*o + i, the layout of T1 rows
// and of the pair-layout integrals V[(a,i),(b,j)], n1 = v*o).
struct TriplesBlock {
  int64_t o = 0, n1 = 0;
  int64_t P[3] = {0, 0, 0};  // global pair offset of each position (block start * o)
  int64_t L[3] = {0, 0, 0};  // pairs per position (block length * o)
};
// S[q] = t[p1] V[p2][p3] + t[p2] V[p1][p3] + t[p3] V[p1][p2]  (p = P + q): the
// disconnected (singles) part, written before the connected terms accumulate.
// Complex: planar operands, imaginary planes S_im, t1_im, V_im (all null on the
// real path); the products are plain complex products.
void triples_singles(double* S, double* S_im, const double* t1, const double* t1_im,
                     const double* V, const double* V_im, const TriplesBlock& b, Stream s);
// With W = S - singles, D = eps_i + eps_j + eps_k - eps_a - eps_b - eps_c and
// Y(q) = sum_pi coef[pi] S(q o pi), where S(q o pi) takes the hole indices of the
// three pairs in the order pi (pi over the six permutations 012, 021, 102, 120,
// 201, 210):  out_dev[0] = sum_q Re W Re Y / D,  out_dev[1] = sum_q Im W Im Y / D.
// ws holds the partial sums (>= 2 * 148 * 4 doubles).  M (planar, may be null):
// a block array of the same layout taking the place of W (the cT branch, whose
// energy is sum M Y / D).
void triples_energy(const double* S, const double* S_im, const double* t1, const double* t1_im,
                    const double* V, const double* V_im, const double* eps_h,
                    const double* eps_p, const TriplesBlock& b, const double coef[6],
                    double* ws, double* out_dev, Stream s, const double* M = nullptr,
                    const double* M_im = nullptr);
// The block-triple part of the CR-(T) denominator of the cT branch (ct::getDenominator,
// CompleteTriples.cxx:138-162, reduced to sum y conj(Z) / D): out_dev[0] = sum Re y Re Z / D,
// out_dev[1] = sum Im y Im Z / D over the block, with
//   y = t_ai t_bj t_ck + t_ai T_bcjk + t_bj T_acik + t_ck T_abij
// (T2 in the pair layout, planar) and Z the hole-permutation combination of S of
// triples_energy; ws as there.
void triples_cr_sums(const double* S, const double* S_im, const double* t1, const double* t1_im,
                     const double* T2, const double* T2_im, const double* eps_h,
                     const double* eps_p, const TriplesBlock& b, const double coef[6],
                     double* ws, double* out_dev, Stream s);

// Number of bandwidth-kernel launches issued so far.
uint64_t launch_count();

}  // namespace ops
}  // namespace cc4s_b200
