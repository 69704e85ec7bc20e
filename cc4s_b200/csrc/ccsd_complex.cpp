// Complex-path CCSD / CCD residual, restated from cc4s Ccsd<Complex>::getResiduum
// (src/main/algorithms/coupledcluster/Ccsd.cxx:382-633) as FP64 tensor-core
// contractions on planar complex tensors.
//
// Integrals follow VertexCoulombIntegrals.cxx:143-190:
//   V_pqsr = sum_G conj(Gamma_G,s,p) Gamma_G,q,r.
// Layouts as on the real path: pair [a][i][b][j] storage, other pairings as
// two-level strided views (strides a: o*vo, i: vo, b: o, j: 1).  Exact
// rearrangements relative to the reference:
//   * Vphhh T1 and Vphhp T1 T1 (Ccsd.cxx:490-491) are contracted through the
//     vertex: sum_G conj(Gamma_G,i,a) sum_k T_bk (Gamma_G,k,j + sum_c Gamma_G,k,c T_cj);
//   * Vphhp T1 and Vphph T1 in the singles (Ccsd.cxx:620-621) likewise;
//   * the ring (Ccsd.cxx:494-502) contracts the vertex part as
//     cTdGamma^T (Gamma (2T - T^x)) without forming Xakic;
//   * the crossed ring's second term is written into the exchange pairing;
//   * the ladder runs on a >= b slabs as on the real path.
#include "ccsd_complex.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

namespace cc4s_b200 {

CcsdComplex::CcsdComplex(const ComplexSystem& sys, const RealOptions& opt, Stream s)
    : Schedule(s), sys_(sys), opt_(opt) {
  so_ = sys.o; sv_ = sys.v; sG_ = sys.G; scplx_ = true; sGph_ = sys.Gph; sGhp_ = sys.Ghp;
  const int64_t o = sys.o, v = sys.v, G = sys.G, n1 = v * o, D2 = n1 * n1;
  if (o <= 0 || v <= 0 || G <= 0) throw Error(ERR_BAD_SHAPE, "CcsdComplex: empty dimension");
  D2_ = D2;
  try {
    scratch_.elems = static_cast<size_t>(std::max<int64_t>(int64_t(1) << 22,
                                                           std::min<int64_t>(64 * v * v, int64_t(1) << 25)));
    scratch_.p = take(scratch_.elems);
    auto z = [&](int64_t n) { return take(2 * n); };
    Vd_ = z(D2); Vh4_ = z(D2); M2_ = z(D2);
    Vhhhh_ = z(o * o * o * o); Vhhhp_ = z(o * o * o * v); Vh2_ = z(o * o * o * v);
    Xd_ = z(D2); Y_ = z(D2); EX_ = z(D2);
    W8_ = Vt_ = EX2_ = W8s_ = EX_;
    Yx_ = Y_;
    adjoint_ = opt.adjoint;
    Kki_ = z(o * o); Kac_ = z(v * v); Lac_ = z(v * v); Lki_ = z(o * o); jG_ = z(G);
    U_ = z(G * n1); cTdGph_ = z(G * n1); W_ = z(G * n1); SQ_ = z(G * n1); W1_ = z(G * n1);
    F_ = z(G * n1); cTdGpp_ = z(G * v * v); dGpp_ = z(G * v * v); dGhh_ = z(G * o * o);
    Xkl1_ = z(o * o * o * o); Xkl2_ = z(o * o * o * o); kck_ = z(n1); P1_ = z(o * o);
    P_ = z(G * o * v);
    cTdGph2_ = cTdGph_;
    if (adjoint_) {  // every recorded value keeps its own buffer
      W8_ = z(D2); Vt_ = z(D2); EX2_ = z(D2); W8s_ = z(D2); Yx_ = z(D2);
      cTdGph2_ = z(G * n1); zt_ = take(n1);
    }
    // The ladder slices follow integralsSliceSize (default No) exactly: the
    // reference mirrors each a > b slice pair into (b,a,j,i), which equals the
    // directly computed block only for a Hermitian vertex, so for a general
    // complex vertex the result depends on the slicing (Ccsd.cxx:553-598).
    // Panels of c (slab V[x][y][c-panel][d] within 2^28 complex values, or
    // CC4S_PPL_SLAB_DOUBLES) split the sum over c exactly and change nothing.
    const int64_t sl = opt.slab > 0 ? opt.slab : o;
    slab_rows_ = std::min(sl, v);
    int64_t budget = int64_t(1) << 28;
    if (const char* e = std::getenv("CC4S_PPL_SLAB_DOUBLES")) {
      const long long b = std::atoll(e);
      if (b > 0) budget = b;
    }
    const int64_t cmax = std::max<int64_t>(
        1, std::min<int64_t>(v, budget / (slab_rows_ * slab_rows_ * v)));
    const int64_t npanels = (v + cmax - 1) / cmax;
    slab_cols_ = (v + npanels - 1) / npanels;
    if (opt.ppl) slab_ = z(slab_rows_ * slab_rows_ * slab_cols_ * v);
  } catch (...) {
    release_all();
    throw;
  }
  count_flops_ = false;
  taping_ = adjoint_;
  build_integrals();
  taping_ = false;
  integrals_tape_.swap(tape_);
  tape_.clear();
  count_flops_ = true;
}

// Xr = Tr + a (tr tr^T - ti ti^T),  Xi = Ti + a (tr ti^T + ti tr^T).  While taping,
// as recorded real rank-1 updates (tr ti^T + ti tr^T = (tr+ti)(tr+ti)^T - tr tr^T
// - ti ti^T); otherwise one fused kernel.
void CcsdComplex::zrank1_(double* Xr, double* Xi, const double* Tr, const double* Ti,
                          const double* tr, const double* ti, double alpha, int64_t n) {
  if (!taping_) {
    ops::zrank1(Xr, Xi, Tr, Ti, tr, ti, alpha, n, s_);
    return;
  }
  rank1_(Xr, 1.0, Tr, alpha, tr, n);
  rank1_(Xr, 1.0, Xr, -alpha, ti, n);
  axpby_(zt_, 1.0, tr, 1.0, ti, 0.0, n);
  rank1_(Xi, 1.0, Ti, alpha, zt_, n);
  rank1_(Xi, 1.0, Xi, -alpha, tr, n);
  rank1_(Xi, 1.0, Xi, -alpha, ti, n);
}

void CcsdComplex::zperm(double* dst, int64_t dst_im, const double* src, int64_t src_im,
                        const int64_t d[4], const int p[4], double alpha, double beta,
                        bool conj) {
  perm_(dst, src, d, p, alpha, beta);
  perm_(dst + dst_im, src + src_im, d, p, conj ? -alpha : alpha, beta);
}

// out = a x + b y on both planes; every operand has its imaginary plane at +n.
void CcsdComplex::zaxpby(double* out, double a, const double* x, double b, const double* y,
                         int64_t n) {
  axpby_(out, a, x, b, y, 0.0, n);
  axpby_(out + n, a, x + n, b, y ? y + n : nullptr, 0.0, n);
}

// Iteration-independent integrals (VertexCoulombIntegrals.cxx:143-190).
void CcsdComplex::build_integrals() {
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o, D2 = D2_;
  const int64_t gph = G * n1;
  double *Gph = sys_.Gph, *Ghh = sys_.Ghh, *Ghp = sys_.Ghp;
  {  // Vd[(a,i),(b,j)] = V_abij = sum_G conj(Ghp[G][i][a]) Gph[G][b][j]
    Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o;
    c.A = vw(Ghp, 1, v, 0, n1);
    c.B = rm(Gph, n1);
    c.C = vw(Vd_, o * n1, n1, 0, 1);
    zgemm(c, gph, gph, D2, true, false);
  }
  {  // Vh4[k][l][c][d] = V_klcd = sum_G conj(Gph[G][c][k]) Ghp[G][l][d]
    Contraction c; c.M = o * v; c.N = o * v; c.K = G; c.Mi = v; c.Ni = v;
    c.A = vw(Gph, 1, o, 0, n1);
    c.B = vw(Ghp, 0, n1, v, 1);
    c.C = vw(Vh4_, o * v * v, v, v * v, 1);
    zgemm(c, gph, gph, D2, true, false);
  }
  const int64_t dh[4] = {o, o, v, v};  // Vh4 [k][l][c][d]
  {  // M2[(c,k),(d,l)] = V_lkdc - V_lkcd / 2  (V_lkcd itself is read as a view of Vh4)
    const int pa[4] = {3, 1, 2, 0}, pb[4] = {2, 1, 3, 0};
    zperm(M2_, D2, Vh4_, D2, dh, pa, 1.0, 0.0);
    zperm(M2_, D2, Vh4_, D2, dh, pb, -0.5, 1.0);
  }
  const int64_t o4 = o * o * o * o, o3v = o * o * o * v;
  {  // Vhhhh[k][l][i][j] = sum_G conj(Ghh[G][i][k]) Ghh[G][l][j]
    Contraction c; c.M = o * o; c.N = o * o; c.K = G; c.Mi = o; c.Ni = o;
    c.A = vw(Ghh, 1, o, 0, o * o);
    c.B = vw(Ghh, 0, o * o, o, 1);
    c.C = vw(Vhhhh_, o * o * o, o, o * o, 1);
    zgemm(c, G * o * o, G * o * o, o4, true, false);
  }
  {  // Vhhhp[k][l][i][c] = sum_G conj(Ghh[G][i][k]) Ghp[G][l][c]
    Contraction c; c.M = o * o; c.N = o * v; c.K = G; c.Mi = o; c.Ni = v;
    c.A = vw(Ghh, 1, o, 0, o * o);
    c.B = vw(Ghp, 0, o * v, v, 1);
    c.C = vw(Vhhhp_, o * o * v, v, o * v, 1);
    zgemm(c, G * o * o, gph, o3v, true, false);
  }
  {  // Vh2[i][k][c][l] = 2 V_klic - V_lkic
    const int64_t dv[4] = {o, o, o, v};
    const int pa[4] = {2, 0, 3, 1}, pb[4] = {2, 1, 3, 0};
    zperm(Vh2_, o3v, Vhhhp_, o3v, dv, pa, 2.0, 0.0);
    zperm(Vh2_, o3v, Vhhhp_, o3v, dv, pb, -1.0, 1.0);
  }
}

void CcsdComplex::residual(const double* T, double* R) {
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o, D2 = D2_;
  const int64_t pl = n1 + D2;  // imaginary plane of amplitude vectors
  double* R1 = R;
  double* R2 = R + n1;
  if (!T) {  // Ccsd.cxx:404-409
    zero_(R1, n1);
    zero_(R1 + pl, n1);
    copy_(R2, Vd_, D2);
    copy_(R2 + pl, Vd_ + D2, D2);
    return;
  }
  const bool ccd = opt_.ccd;
  flops_ = 0.0;
  double* t = cp(T);
  double* Td = cp(T + n1);
  double *Gpp = sys_.Gpp, *Gph = sys_.Gph, *Ghh = sys_.Ghh, *Ghp = sys_.Ghp;
  const int64_t gpp = G * v * v, gph = G * n1, ghh = G * o * o, o4 = o * o * o * o,
                o3v = o * o * o * v, gov = G * o * v;
  const int64_t d4[4] = {v, o, v, o};
  const int64_t dh[4] = {o, o, v, v};  // Vh4 [k][l][c][d]
  const int p_ex[4] = {0, 3, 2, 1};
  const int64_t sA = o * n1, sI = n1, sB = o;  // pair-layout strides

  // ---- X = T2 + T1 T1 (Ccsd.cxx:460-461) ----------------------------------------
  if (ccd) { copy_(Xd_, Td, D2); copy_(Xd_ + D2, Td + pl, D2); }
  else zrank1_(Xd_, Xd_ + D2, Td, Td + pl, t, t + pl, 1.0, n1);
  // ---- Kac, Kki (Ccsd.cxx:465-473) ---------------------------------------------
  {  // Vt[(c,k),(d,l)] = 2 V_klcd - V_kldc
    const int pa[4] = {2, 0, 3, 1}, pb[4] = {3, 0, 2, 1};
    zperm(Vt_, D2, Vh4_, D2, dh, pa, 2.0, 0.0);
    zperm(Vt_, D2, Vh4_, D2, dh, pb, -1.0, 1.0);
  }
  {  // Kki[k][i] = sum_{c,(d,l)} Vt[(c,k),(d,l)] X[(c,i),(d,l)]
    Contraction c; c.M = o; c.N = o; c.K = v * n1; c.Ki = n1;
    c.A = vw(Vt_, 0, sI, sA, 1); c.B = vw(Xd_, sA, 1, 0, sI); c.C = rm(Kki_, o);
    zgemm(c, D2, D2, o * o);
  }
  {  // Kac[a][c] = -sum_{k,(d,l)} X[(a,k),(d,l)] Vt[(c,k),(d,l)]
    Contraction c; c.M = v; c.N = v; c.K = o * n1; c.Ki = n1;
    c.A = vw(Xd_, 0, sA, sI, 1); c.B = vw(Vt_, sI, 1, 0, sA); c.C = rm(Kac_, v); c.alpha = -1.0;
    zgemm(c, D2, D2, v * v);
  }
  if (!ccd) {  // kck[(c,k)] = sum_{(d,l)} Vt[(c,k),(d,l)] t[d][l]  (for the singles)
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(Vt_, n1); c.B = vw(t, 0, 1, 0, 0); c.C = vw(kck_, 0, 1, 0, 0);
    zgemm(c, D2, pl, n1);
  }
  // ---- Lac (Ccsd.cxx:468-470) ----------------------------------------------------
  copy_(Lac_, Kac_, 2 * v * v);
  if (!ccd) {
    {  // jG[G] = sum_{k,d} Ghp[G][k][d] t[d][k]
      Contraction c; c.M = G; c.N = 1; c.K = n1; c.Ki = v;
      c.A = vw(Ghp, 0, n1, v, 1); c.B = vw(t, 1, o, 0, 0); c.C = vw(jG_, 0, 1, 0, 0);
      zgemm(c, gph, pl, G);
    }
    {  // Lac[a][c] += 2 sum_G conj(Gpp[G][c][a]) jG[G]
      Contraction c; c.M = v * v; c.N = 1; c.K = G; c.Mi = v;
      c.A = vw(Gpp, v, 1, 0, v * v); c.B = vw(jG_, 0, 1, 0, 0); c.C = vw(Lac_, 1, v, 0, 0);
      c.alpha = 2.0; c.beta = 1.0;
      zgemm(c, gpp, G, v * v, true, false);
    }
    {  // U[G][a][k] = sum_d conj(Gpp[G][d][a]) t[d][k]
      Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(tr(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(U_, o), n1);
      zgemm(c, gpp, pl, gph, true, false);
    }
    {  // Lac[a][c] -= sum_{G,k} U[G][a][k] Ghp[G][k][c]
      Contraction c; c.M = v; c.N = v; c.K = G * o; c.Ki = o;
      c.A = vw(U_, 0, o, n1, 1); c.B = vw(Ghp, o * v, v, 0, 1); c.C = rm(Lac_, v);
      c.alpha = -1.0; c.beta = 1.0;
      zgemm(c, gph, gph, v * v);
    }
  }
  // ---- Lki (Ccsd.cxx:476-478) ----------------------------------------------------
  copy_(Lki_, Kki_, 2 * o * o);
  if (!ccd) {
    Contraction c; c.M = o * o; c.N = 1; c.K = v * o; c.Mi = o; c.Ki = o;
    c.A = vw(Vh2_, v * o * o, v * o, o, 1); c.B = vw(t, o, 1, 0, 0); c.C = vw(Lki_, 1, o, 0, 0);
    c.beta = 1.0;
    zgemm(c, o3v, pl, o * o);
  }
  // ---- R2 = Lac T2 - Lki T2 (Ccsd.cxx:481-484) ------------------------------------
  {
    Contraction c; c.M = v; c.N = o * n1; c.K = v;
    c.A = rm(Lac_, v); c.B = rm(Td, o * n1); c.C = rm(R2, o * n1);
    zgemm(c, v * v, pl, pl);
  }
  {
    Contraction c; c.M = o; c.N = n1; c.K = o; c.batch = v;
    c.A = tr(Lki_, o); c.B = with_batch(rm(Td, n1), o * n1); c.C = with_batch(rm(R2, n1), o * n1);
    c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, o * o, pl, pl);
  }
  // ---- T1-dressed vertex terms (Ccsd.cxx:487-491) -------------------------------
  {
    const int64_t dg[4] = {1, G, o, v};
    const int pt[4] = {0, 1, 3, 2};
    zperm(cTdGph_, gph, Ghp, gph, dg, pt, 1.0, 0.0, true);  // conj(Ghp[G][i][a]) -> [G][a][i]
  }
  copy_(dGhh_, Ghh, 2 * ghh);
  if (!ccd) {
    {  // cTdGph[G][a][i] -= sum_k t[a][k] conj(Ghh[G][i][k])
      Contraction c; c.M = v; c.N = o; c.K = o; c.batch = G;
      c.A = rm(t, o); c.B = with_batch(tr(Ghh, o), o * o); c.C = with_batch(rm(cTdGph_, o), n1);
      c.alpha = -1.0; c.beta = 1.0;
      zgemm(c, pl, ghh, gph, false, true);
    }
    {  // W[G][b][j] = sum_c Gpp[G][b][c] t[c][j]
      Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(rm(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(W_, o), n1);
      zgemm(c, gpp, pl, gph);
    }
    {  // R2 += cTdGph^T W
      Contraction c; c.M = n1; c.N = n1; c.K = G;
      c.A = tr(cTdGph_, n1); c.B = rm(W_, n1); c.C = rm(R2, n1); c.beta = 1.0;
      zgemm(c, gph, gph, pl, false, false, true);
    }
    {  // dGhh[G][k][i] += sum_d Ghp[G][k][d] t[d][i]
      Contraction c; c.M = o; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(rm(Ghp, v), o * v); c.B = rm(t, o); c.C = with_batch(rm(dGhh_, o), o * o);
      c.beta = 1.0;
      zgemm(c, gph, pl, ghh);
    }
    {  // SQ[G][b][j] = sum_k t[b][k] dGhh[G][k][j]
      Contraction c; c.M = v; c.N = o; c.K = o; c.batch = G;
      c.A = rm(t, o); c.B = with_batch(rm(dGhh_, o), o * o); c.C = with_batch(rm(SQ_, o), n1);
      zgemm(c, pl, ghh, gph);
    }
    {  // R2 -= sum_G conj(Ghp[G][i][a]) SQ[G][b][j]   (Vphhh T1 + Vphhp T1 T1)
      Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o;
      c.A = vw(Ghp, 1, v, 0, n1); c.B = rm(SQ_, n1); c.C = vw(R2, o * n1, n1, 0, 1);
      c.alpha = -1.0; c.beta = 1.0;
      zgemm(c, gph, gph, pl, true, false, true);
    }
  }
  // ---- ring Xakic (Ccsd.cxx:494-502) -----------------------------------------------
  if (ccd) { copy_(W8_, Td, D2); copy_(W8_ + D2, Td + pl, D2); }
  else zrank1_(W8_, W8_ + D2, Td, Td + pl, t, t + pl, 2.0, n1);
  zperm(Yx_, D2, W8_, D2, d4, p_ex, 1.0, 0.0);  // (T2 + 2 T1 T1)^x
  // the second dressing of the ring vertex (in place on the fast path)
  if (cTdGph2_ != cTdGph_) copy_(cTdGph2_, cTdGph_, 2 * gph);
  if (!ccd) {  // cTdGph[G][a][i] += sum_d conj(Gpp[G][d][a]) t[d][i]
    Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
    c.A = with_batch(tr(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(cTdGph2_, o), n1);
    c.beta = 1.0;
    zgemm(c, gpp, pl, gph, true, false);
  }
  {  // cTdGph -= 1/2 sum_{dl} conj(Gph[G][d][l]) Y_dail
    Contraction c; c.M = G; c.N = n1; c.K = n1;
    c.A = rm(Gph, n1); c.B = rm(Yx_, n1); c.C = rm(cTdGph2_, n1); c.alpha = -0.5; c.beta = 1.0;
    zgemm(c, gph, D2, gph, true, false, true);
  }
  zperm(Y_, D2, Td, pl, d4, p_ex, -1.0, 0.0);                 // -T^x
  axpby_(Y_, 2.0, Td, 1.0, Y_, 0.0, D2);                      // Y = 2T - T^x
  axpby_(Y_ + D2, 2.0, Td + pl, 1.0, Y_ + D2, 0.0, D2);
  {  // W1[G][(b,j)] = sum_{c,k} Ghp[G][k][c] Y[(c,k),(b,j)]
    Contraction c; c.M = G; c.N = n1; c.K = n1; c.Ki = o;
    c.A = vw(Ghp, 0, n1, 1, v); c.B = vw(Y_, o * n1, n1, 0, 1); c.C = rm(W1_, n1);
    zgemm(c, gph, D2, gph, false, false, true);
  }
  {  // R2 += cTdGph^T W1
    Contraction c; c.M = n1; c.N = n1; c.K = G;
    c.A = tr(cTdGph2_, n1); c.B = rm(W1_, n1); c.C = rm(R2, n1); c.beta = 1.0;
    zgemm(c, gph, gph, pl, false, false, true);
  }
  {  // EX = T M2^T ;  R2 += EX Y
    Contraction c; c.M = n1; c.N = n1; c.K = n1;
    c.A = rm(Td, n1); c.B = tr(M2_, n1); c.C = rm(EX_, n1);
    zgemm(c, pl, D2, D2, false, false, true);
    Contraction d; d.M = n1; d.N = n1; d.K = n1;
    d.A = rm(EX_, n1); d.B = rm(Y_, n1); d.C = rm(R2, n1); d.beta = 1.0;
    zgemm(d, D2, D2, pl, false, false, true);
  }
  // ---- crossed ring Xakci (Ccsd.cxx:509-517) ----------------------------------------
  {
    const int64_t dg[4] = {1, G, v, v};
    const int pt[4] = {0, 1, 3, 2};
    zperm(cTdGpp_, gpp, Gpp, gpp, dg, pt, 1.0, 0.0, true);  // conj(Gpp[G][c][a]) -> [G][a][c]
  }
  if (!ccd) {  // cTdGpp[G][a][c] -= sum_l t[a][l] conj(Gph[G][c][l])
    Contraction c; c.M = v; c.N = v; c.K = o; c.batch = G;
    c.A = rm(t, o); c.B = with_batch(tr(Gph, o), n1); c.C = with_batch(rm(cTdGpp_, v), v * v);
    c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, pl, gph, gpp, false, true);
  }
  {  // EX[(a,i),(c,k)] = -1/2 sum_{l,d} T_adli V_lkcd   (k = (l, d); T^x and Vh4 views)
    Contraction c; c.M = n1; c.N = n1; c.K = n1; c.Mi = o; c.Ki = v; c.Ni = o;
    c.A = vw(Td, sA, 1, sI, sB);                   // T_adli = T[(a,l),(d,i)]
    c.B = vw(Vh4_, o * v * v, 1, v, v * v);        // V_lkcd = Vh4[l][k][c][d]
    c.C = vw(EX2_, sA, sI, o, 1); c.alpha = -0.5;
    zgemm(c, pl, D2, D2, false, false, true);
  }
  {  // EX[a][i][c][k] += sum_G cTdGpp[G][a][c] dGhh[G][k][i]
    Contraction c; c.M = v * v; c.N = o * o; c.K = G; c.Mi = v; c.Ni = o;
    c.A = vw(cTdGpp_, v, 1, 0, v * v); c.B = vw(dGhh_, 0, o * o, o, 1);
    c.C = vw(EX2_, o * n1, o, 1, n1); c.beta = 1.0;
    zgemm(c, gpp, ghh, D2, false, false, true);
  }
  {  // R2 -= EX T
    Contraction c; c.M = n1; c.N = n1; c.K = n1;
    c.A = rm(EX2_, n1); c.B = rm(Td, n1); c.C = rm(R2, n1); c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, D2, pl, pl, false, false, true);
  }
  {  // R2_abij -= sum_ck T_ackj X_bkci   (exchange pairing)
    Contraction c; c.M = n1; c.N = n1; c.K = n1; c.Mi = o; c.Ni = o; c.Ki = o;
    c.A = vw(Td, sA, 1, sB, sI);                   // T_ackj = T[(a,k),(c,j)]
    c.B = vw(EX2_, sB, 1, sA, sI);                 // X_bkci = EX[(b,i),(c,k)]
    c.C = vw(R2, sA, 1, sB, sI); c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, pl, D2, pl, false, false, true);
  }
  // ---- symmetrisation, +V (Ccsd.cxx:520,529) -----------------------------------
  sym_(R2, n1);
  sym_(R2 + pl, n1);
  axpby_(R2, 1.0, R2, 1.0, Vd_, 0.0, D2);
  axpby_(R2 + pl, 1.0, R2 + pl, 1.0, Vd_ + D2, 0.0, D2);
  // ---- hole-hole ladder (Ccsd.cxx:534-546) ----------------------------------------
  copy_(Xkl1_, Vhhhh_, 2 * o4);
  if (!ccd) {
    {
      Contraction c; c.M = o * o * o; c.N = o; c.K = v;
      c.A = rm(Vhhhp_, v); c.B = rm(t, o); c.C = rm(Xkl1_, o); c.beta = 1.0;
      zgemm(c, o3v, pl, o4);
    }
    {
      Contraction c; c.M = o * o; c.N = o; c.K = v; c.batch = o; c.Mi = o;
      c.A = vw(Vhhhp_, o * v, v, 0, 1, 0, o * o * v); c.B = rm(t, o);
      c.C = vw(Xkl1_, o * o * o, 1, 0, o, 0, o * o); c.beta = 1.0;
      zgemm(c, o3v, pl, o4);
    }
  }
  {  // Xkl2[kl][ij] = sum_cd V_klcd X_cdij   (k = (c,d))
    Contraction c; c.M = o * o; c.N = o * o; c.K = v * v; c.Ki = v; c.Ni = o;
    c.A = vw(Vh4_, 0, v * v, v, 1);
    c.B = vw(Xd_, sA, sB, sI, 1);                  // X_cdij = X[(c,i),(d,j)]
    c.C = vw(Xkl2_, 0, o * o, o, 1);
    zgemm(c, D2, D2, o4, false, false, true);
  }
  {  // R2 += Xkl1 X_abkl, R2 += Xkl2 T_abkl (or X_abkl)   (m = (a,b), k = (k,l))
    Contraction c; c.M = v * v; c.N = o * o; c.K = o * o; c.Mi = v; c.Ki = o; c.Ni = o;
    c.A = vw(Xd_, sA, sB, sI, 1); c.B = vw(Xkl1_, o * o * o, o * o, o, 1);
    c.C = vw(R2, sA, sB, sI, 1); c.beta = 1.0;
    zgemm(c, D2, o4, pl, false, false, true);
    c.B.p = Xkl2_;
    if (opt_.ppl) {
      c.A.p = cp(Td);
      zgemm(c, pl, o4, pl, false, false, true);
    } else {
      zgemm(c, D2, o4, pl, false, false, true);
    }
  }
  // ---- particle-particle ladder (Ccsd.cxx:549-601) ---------------------------------
  if (opt_.ppl) {
    copy_(dGpp_, Gpp, 2 * gpp);
    if (!ccd) {  // dGpp[G][a][b] -= sum_k t[a][k] Ghp[G][k][b]
      Contraction c; c.M = v; c.N = v; c.K = o; c.batch = G;
      c.A = rm(t, o); c.B = with_batch(rm(Ghp, v), o * v); c.C = with_batch(rm(dGpp_, v), v * v);
      c.alpha = -1.0; c.beta = 1.0;
      zgemm(c, pl, gph, gpp);
    }
    const int64_t s = slab_rows_, cn = slab_cols_, nb = (v + s - 1) / s;
    const int64_t sz = s * s * cn * v;  // imaginary plane of the slab
    for (int64_t c0 = 0; c0 < v; c0 += cn) {
      const int64_t nc = std::min(cn, v - c0);
      for (int64_t X = 0; X < nb; ++X)
        for (int64_t Yb = 0; Yb <= X; ++Yb) {
          const int64_t x0 = X * s, sx = std::min(s, v - x0);
          const int64_t y0 = Yb * s, sy = std::min(s, v - y0);
          const size_t t_build = tape_.size();
          {  // slab[x][y][c'][d], m = (x, c'), n = (y, d)
            Contraction c; c.M = sx * nc; c.N = sy * v; c.K = G; c.Mi = nc; c.Ni = v;
            c.A = vw(cTdGpp_ + x0 * v + c0, v, 1, 0, v * v);
            c.B = vw(dGpp_ + y0 * v, 0, v * v, v, 1);
            c.C = vw(slab_, sy * nc * v, v, nc * v, 1);
            zgemm(c, gpp, gpp, sz, false, false, true);
          }
          std::vector<Contraction> build_ops;
          for (size_t k = t_build; taping_ && k < tape_.size(); ++k) build_ops.push_back(tape_[k].c);
          {  // m = (x, y), k = (c', d), n = (i, j)
            Contraction c; c.M = sx * sy; c.N = o * o; c.K = nc * v; c.Mi = sy; c.Ki = v; c.Ni = o;
            c.A = vw(slab_, sy * nc * v, nc * v, v, 1);
            c.B = vw(Xd_ + c0 * sA, sA, sB, sI, 1);   // X_cdij = X[(c,i),(d,j)]
            c.C = vw(R2 + x0 * o * n1 + y0 * o, o * n1, o, n1, 1);
            if (X != Yb) c.C2 = vw(R2 + y0 * o * n1 + x0 * o, o, o * n1, 1, n1);
            c.beta = 1.0;
            zgemm(c, sz, D2, pl, false, false, true);
          }
          if (taping_ && !build_ops.empty()) {  // the slab is rebuilt before the adjoints
            TapeOp& last = tape_.back();        // of this pair's contractions (the last
            last.recompute = true;              // recorded one is reversed first)
            last.pre = build_ops[0];
            last.pres.assign(build_ops.begin() + 1, build_ops.end());
            last.zero_p = slab_;
            last.zero_n = 2 * sz;
          }
        }
    }
  }
  if (ccd) {
    zero_(R1, n1);
    zero_(R1 + pl, n1);
    profile_finish();
    return;
  }
  // ---- singles (Ccsd.cxx:607-629) ------------------------------------------------------
  {
    Contraction c; c.M = v; c.N = o; c.K = v;
    c.A = rm(Kac_, v); c.B = rm(t, o); c.C = rm(R1, o);
    zgemm(c, v * v, pl, pl);
    Contraction d; d.M = v; d.N = o; d.K = o;
    d.A = rm(t, o); d.B = rm(Kki_, o); d.C = rm(R1, o); d.alpha = -1.0; d.beta = 1.0;
    zgemm(d, pl, o * o, pl);
  }
  {  // R1 += (2T - T^x) kck
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(Y_, n1); c.B = vw(kck_, 0, 1, 0, 0); c.C = vw(R1, 0, 1, 0, 0); c.beta = 1.0;
    zgemm(c, D2, n1, pl);
  }
  {  // R1 += t (kck^T t)
    Contraction c; c.M = o; c.N = o; c.K = v;
    c.A = tr(kck_, o); c.B = rm(t, o); c.C = rm(P1_, o);
    zgemm(c, n1, pl, o * o);
    Contraction d; d.M = v; d.N = o; d.K = o;
    d.A = rm(t, o); d.B = rm(P1_, o); d.C = rm(R1, o); d.beta = 1.0;
    zgemm(d, pl, o * o, pl);
  }
  {  // R1 += 2 sum_G conj(Ghp[G][i][a]) jG[G]   (2 Vphhp T1)
    Contraction c; c.M = n1; c.N = 1; c.K = G; c.Mi = o;
    c.A = vw(Ghp, 1, v, 0, n1); c.B = vw(jG_, 0, 1, 0, 0); c.C = vw(R1, o, 1, 0, 0);
    c.alpha = 2.0; c.beta = 1.0;
    zgemm(c, gph, G, pl, true, false);
  }
  {  // P[G][i][c] = sum_k Ghh[G][k][i] t[c][k];  R1[a][i] -= sum_{G,c} conj(Gpp[G][c][a]) P[G][i][c]
    Contraction c; c.M = o; c.N = v; c.K = o; c.batch = G;
    c.A = with_batch(tr(Ghh, o), o * o); c.B = tr(t, o); c.C = with_batch(rm(P_, v), o * v);
    zgemm(c, ghh, pl, gov);
    Contraction d; d.M = v; d.N = o; d.K = G * v; d.Ki = v;
    d.A = vw(Gpp, 0, 1, v * v, v); d.B = vw(P_, o * v, 1, 0, v); d.C = rm(R1, o);
    d.alpha = -1.0; d.beta = 1.0;
    zgemm(d, gpp, gov, pl, true, false);
  }
  {  // F = Ghp' (2X - X^x);  R1[a][i] += sum_{G,x} conj(Gpp[G][x][a]) F[G][x][i]
    zperm(W8s_, D2, Xd_, D2, d4, p_ex, 1.0, 0.0);
    axpby_(W8s_, 2.0, Xd_, -1.0, W8s_, 0.0, D2);
    axpby_(W8s_ + D2, 2.0, Xd_ + D2, -1.0, W8s_ + D2, 0.0, D2);
    Contraction c; c.M = G; c.N = n1; c.K = n1; c.Ki = o;
    c.A = vw(Ghp, 0, n1, 1, v); c.B = vw(W8s_, o * n1, n1, 0, 1); c.C = rm(F_, n1);
    zgemm(c, gph, D2, gph, false, false, true);
    Contraction d; d.M = v; d.N = o; d.K = G * v; d.Ki = v;
    d.A = vw(Gpp, 0, 1, v * v, v); d.B = vw(F_, n1, o, 0, 1); d.C = rm(R1, o); d.beta = 1.0;
    zgemm(d, gpp, gph, pl, true, false);
  }
  {  // R1[a][i] -= sum_{k,(c,l)} X[(a,k),(c,l)] Vh2[i][k][c][l]
    Contraction c; c.M = v; c.N = o; c.K = o * n1; c.Ki = n1;
    c.A = vw(Xd_, 0, sA, sI, 1); c.B = vw(Vh2_, n1, 1, 0, o * n1); c.C = rm(R1, o);
    c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, D2, o3v, pl);
  }
  profile_finish();
}

}  // namespace cc4s_b200

namespace cc4s_b200 {

// E = sum Re[(2 conj(V_abij) - conj(V_baij)) X_abij], X = T2 + T1 T1, over both planes:
//   dE/dX_re = 2 V_re - V^x_re,  dE/dX_im = 2 V_im - V^x_im  (V^x_abij = V_baij),
//   dE/dT2 = dE/dX,  dE/dT1 (re + i im) = 2 (dE/dX) conj(t),
//   dE/dVd = 2 X - X^x on each plane.
void CcsdComplex::energy_gradients(const double* T, double* g, double* Vd_bar) {
  const int64_t o = sys_.o, v = sys_.v, n1 = v * o, D2 = D2_, pl = n1 + D2;
  const int64_t d4[4] = {v, o, v, o};
  const int p_ex[4] = {0, 3, 2, 1};
  for (int q = 0; q < 2; ++q) {
    double* g2 = g + q * pl + n1;
    const double* V = Vd_ + q * D2;
    ops::permute4(g2, V, d4, p_ex, -1.0, 0.0, s_);
    ops::axpby(g2, 2.0, V, 1.0, g2, 0.0, D2, s_);
  }
  {
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(g + n1, n1); c.B = vw(cp(T), 0, 1, 0, 0); c.C = vw(g, 0, 1, 0, 0); c.alpha = 2.0;
    zgemm(c, pl, pl, pl, false, true);
  }
  if (Vd_bar) {  // X staged in the forward output buffer (never read by the reverse sweep)
    if (!Rf_) Rf_ = take(2 * pl);
    double* Xr = Rf_ + n1;
    double* Xi = Rf_ + pl + n1;
    ops::zrank1(Xr, Xi, T + n1, T + pl + n1, T, T + pl, 1.0, n1, s_);
    const double* X[2] = {Xr, Xi};
    for (int q = 0; q < 2; ++q) {
      double* b = Vd_bar + q * D2;
      ops::permute4(b, X[q], d4, p_ex, -1.0, 0.0, s_);
      ops::axpby(b, 2.0, X[q], 1.0, b, 0.0, D2, s_);
    }
  }
}

void CcsdComplex::prepare_vjp(const double* T) {
  if (!adjoint_) throw Error(ERR_STATE, "reverse mode needs a schedule built in adjoint mode");
  if (!T) throw Error(ERR_INVALID_ARGUMENT, "prepare_vjp: no amplitudes");
  const int64_t n1 = sys_.v * sys_.o, pl = n1 + D2_;
  if (!Rf_) Rf_ = take(2 * pl);
  tape_.clear();
  taping_ = true;
  try {
    residual(T, Rf_);
  } catch (...) {
    taping_ = false;
    throw;
  }
  taping_ = false;
  Tprep_ = T;
}

void CcsdComplex::vjp(const double* Rbar, double* Tbar, const VertexBar* gbar,
                      const double* extra_Vd_bar) {
  if (!Tprep_) throw Error(ERR_STATE, "vjp before prepare_vjp");
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o, D2 = D2_, pl = n1 + D2,
                n = 2 * pl;
  while (bar_bufs_.size() < owned_.size()) {
    const size_t k = bar_bufs_.size();
    bar_bufs_.push_back(owned_[k] == scratch_.p ? nullptr : ops::alloc(owned_n_[k]));
  }
  regions_.clear();
  for (size_t k = 0; k < owned_.size(); ++k) {
    if (!bar_bufs_[k]) continue;
    ops::zero(bar_bufs_[k], owned_n_[k], s_);
    regions_.push_back({owned_[k], static_cast<int64_t>(owned_n_[k]), bar_bufs_[k]});
  }
  ops::zero(Tbar, n, s_);
  regions_.push_back({Tprep_, n, Tbar});
  if (gbar) {  // planar complex vertex blocks: two planes each
    if (gbar->Gpp) regions_.push_back({sys_.Gpp, 2 * G * v * v, gbar->Gpp});
    if (gbar->Gph) regions_.push_back({sys_.Gph, 2 * G * n1, gbar->Gph});
    if (gbar->Ghh) regions_.push_back({sys_.Ghh, 2 * G * o * o, gbar->Ghh});
    if (gbar->Ghp) regions_.push_back({sys_.Ghp, 2 * G * n1, gbar->Ghp});
  }
  ops::d2d(bar_of(Rf_), Rbar, n, s_);
  try {
    reverse(tape_);
    // the amplitudes are symmetric, T_abij = T_baji: project the T2 adjoint (both planes)
    for (int q = 0; q < 2; ++q) {
      double* t2 = Tbar + q * pl + n1;
      ops::symmetrize(t2, n1, s_);
      ops::axpby(t2, 0.5, t2, 0.0, nullptr, 0.0, D2, s_);
    }
    if (gbar) {
      if (extra_Vd_bar)
        ops::axpby(bar_of(Vd_), 1.0, bar_of(Vd_), 1.0, extra_Vd_bar, 0.0, 2 * D2, s_);
      reverse(integrals_tape_);
    }
  } catch (...) {
    regions_.clear();
    throw;
  }
  regions_.clear();
}

}  // namespace cc4s_b200
