// Real-path CCSD / CCD residual, restated from cc4s Ccsd<Real>::getResiduum
// (src/main/algorithms/coupledcluster/Ccsd.cxx:77-378) as a schedule of FP64
// tensor-core contractions on HBM-resident tensors.
//
// Layouts (row-major, all FP64):
//   T1, R1        [a][i]                         (v x o)
//   T2, R2 "pair" [a][i][b][j]  = X_abij          ((vo) x (vo), symmetric matrix)
//   vertex        Gpp[G][a][b], Gph[G][a][i], Ghh[G][k][i], Ghp[G][i][a]
// Only four (vo)^2 buffers are stored besides T and R (Vd, X, Y, EX): the other
// pairings a contraction needs -- exchange A_abji, pp order A_abij with (a,b) and
// (i,j) as matrix indices -- are two-level strided views of the pair layout
// (strides a: o*vo, i: vo, b: o, j: 1), which the contraction kernels read directly.
//
// Exact algebraic rearrangements relative to the reference (each term is the
// same sum, only the contraction order changes):
//   * ring (Ccsd.cxx:215-229): the two V_dclk terms are folded into the
//     vertex, Z_Gai = sum_dl Gamma_Gdl (T_adil - X'_dail/2), and the vertex part of
//     Xakic is contracted as (dGamma + Z)^T (Gamma (2T - T^x)) without forming
//     the v^2 o^2 intermediate; only the exchange part -V_cdlk T_adil / 2 is a
//     (vo)^3 contraction;
//   * crossed ring (Ccsd.cxx:233-253): the second term, sum Xbkci T_ackj, is
//     written straight into the exchange pairing of R2;
//   * the particle-particle ladder (Ccsd.cxx:283-333) is evaluated on square
//     blocks of the virtual index pair (a >= b blocks, mirrored into (b,a,j,i))
//     and panels of c, V_abcd built per slab from the dressed vertex and never
//     stored whole;
//   * singles (Ccsd.cxx:339-375): the Gamma.Gamma.X pair shares one
//     Gamma (2X - X^x) intermediate.
#include "ccsd_real.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace cc4s_b200 {

CcsdReal::CcsdReal(const RealSystem& sys, const RealOptions& opt, Stream s)
    : Schedule(s), sys_(sys), opt_(opt) {
  so_ = sys.o; sv_ = sys.v; sG_ = sys.G; scplx_ = false; sGph_ = sys.Gph; sGhp_ = sys.Ghp;
  const int64_t o = sys.o, v = sys.v, G = sys.G, n1 = v * o, D2 = n1 * n1;
  if (o <= 0 || v <= 0 || G <= 0) throw Error(ERR_BAD_SHAPE, "CcsdReal: empty dimension");
  try {
    // split-K scratch
    scratch_.elems = static_cast<size_t>(std::max<int64_t>(int64_t(1) << 22,
                                                           std::min<int64_t>(64 * v * v, int64_t(1) << 25)));
    scratch_.p = take(scratch_.elems);
    Vd_ = take(D2);
    Vhhhh_ = take(o * o * o * o); Vhhhp_ = take(o * o * o * v); Vh2_ = take(o * o * o * v);
    Xd_ = take(D2); Y_ = take(D2); EX_ = take(D2);
    // Roles that share EX, Y and dGph on the fast path get their own buffers in
    // adjoint mode, where every recorded value must survive the residual.
    adjoint_ = opt.adjoint;
    Vt_ = EX2_ = W8r_ = W8s_ = EX_;
    Yx_ = Y_;
    if (adjoint_) {
      Vt_ = take(D2); EX2_ = take(D2); W8r_ = take(D2); W8s_ = take(D2); Yx_ = take(D2);
    }
    Kki_ = take(o * o); Kac_ = take(v * v); Lac_ = take(v * v); Lki_ = take(o * o);
    jG_ = take(G);
    U_ = take(G * n1); dGph_ = take(G * n1); W_ = take(G * n1); Z_ = take(G * n1);
    W1_ = take(G * n1); F_ = take(G * n1);
    dGpp_ = take(G * v * v); dGhh_ = take(G * o * o);
    A2_ = adjoint_ ? take(G * n1) : dGph_;
    Q_ = take(n1 * o * o); Xkl1_ = take(o * o * o * o); Xkl2_ = take(o * o * o * o);
    kck_ = take(n1); P1_ = take(o * o); P_ = take(G * o * v);
    // Ladder slabs: blocks of s virtual orbitals (s^2 rows of the contraction,
    // 64 by default) times a panel of c_n values of c, sized so that one slab
    // V[x][y][c][d] (s^2 c_n v doubles) stays within the budget (2^28 doubles;
    // CC4S_PPL_SLAB_DOUBLES overrides it).
    int64_t sl = opt.slab > 0 ? opt.slab : 64;
    slab_rows_ = std::max<int64_t>(1, std::min(sl, v));
    int64_t budget = int64_t(1) << 28;
    if (const char* e = std::getenv("CC4S_PPL_SLAB_DOUBLES")) {
      const long long b = std::atoll(e);
      if (b > 0) budget = b;
    }
    const int64_t cmax = std::max<int64_t>(
        1, std::min<int64_t>(v, budget / (slab_rows_ * slab_rows_ * v)));
    const int64_t npanels = (v + cmax - 1) / cmax;
    slab_cols_ = (v + npanels - 1) / npanels;
    if (opt.ppl) slab_ = take(slab_rows_ * slab_rows_ * slab_cols_ * v);
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

// Iteration-independent integrals (VertexCoulombIntegrals.cxx:87-121).
void CcsdReal::build_integrals() {
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o;
  // Vd[(a,i),(b,j)] = V_abij = sum_G Gph[G][a][i] Gph[G][b][j]
  {
    Contraction c; c.M = n1; c.N = n1; c.K = G;
    c.A = tr(sys_.Gph, n1); c.B = rm(sys_.Gph, n1); c.C = rm(Vd_, n1);
    gemm_(c);
  }
  // Vhhhh[k][l][i][j] = sum_G Ghh[G][k][i] Ghh[G][l][j]
  {
    Contraction c; c.M = o * o; c.N = o * o; c.K = G; c.Mi = o; c.Ni = o;
    c.A = vw(sys_.Ghh, o, 1, 0, o * o);            // (m=(k,i), G)
    c.B = vw(sys_.Ghh, 0, o * o, o, 1);            // (G, n=(l,j))
    c.C = vw(Vhhhh_, o * o * o, o, o * o, 1);      // [k][l][i][j]
    gemm_(c);
  }
  // Vhhhp[k][l][i][c] = sum_G Ghh[G][k][i] Ghp[G][l][c]
  {
    Contraction c; c.M = o * o; c.N = o * v; c.K = G; c.Mi = o; c.Ni = v;
    c.A = vw(sys_.Ghh, o, 1, 0, o * o);
    c.B = vw(sys_.Ghp, 0, o * v, v, 1);
    c.C = vw(Vhhhp_, o * o * v, v, o * v, 1);
    gemm_(c);
  }
  // Vh2[i][k][c][l] = 2 V_klic - V_lkic
  {
    const int64_t dh[4] = {o, o, o, v};
    const int pa[4] = {2, 0, 3, 1};
    const int pb[4] = {2, 1, 3, 0};
    perm_(Vh2_, Vhhhp_, dh, pa, 2.0, 0.0);
    perm_(Vh2_, Vhhhp_, dh, pb, -1.0, 1.0);
  }
}

void CcsdReal::residual(const double* T, double* R) {
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o, D2 = n1 * n1;
  double* R1 = R;
  double* R2 = R + n1;
  if (!T) {  // Ccsd.cxx:97-102
    ops::zero(R1, n1, s_);
    ops::d2d(R2, Vd_, D2, s_);
    return;
  }
  const bool ccd = opt_.ccd;
  flops_ = 0.0;
  double* t = cp(T);
  double* Td = cp(T + n1);
  double* Gpp = sys_.Gpp;
  double* Gph = sys_.Gph;
  double* Ghh = sys_.Ghh;
  const int64_t d4[4] = {v, o, v, o};
  const int p_ex[4] = {0, 3, 2, 1};   // pair -> exchange (i <-> j)
  // strides of the pair layout [a][i][b][j]
  const int64_t sA = o * n1, sI = n1, sB = o;

  // ---- X = T2 + T1 T1 (Ccsd.cxx:169-170) -----------------------------------
  if (ccd) copy_(Xd_, Td, D2);
  else rank1_(Xd_, 1.0, Td, 1.0, t, n1);

  // ---- Kki, Kac (Ccsd.cxx:172-178) -------------------------------------------
  // EX <- Vt[(c,k),(d,l)] = 2 V_cdkl - V_cdlk  (= 2 V_cdkl - V_dckl)
  perm_(Vt_, Vd_, d4, p_ex, -1.0, 0.0);
  axpby_(Vt_, 2.0, Vd_, 1.0, Vt_, 0.0, D2);
  {  // Kki[k][i] = sum_{c,(d,l)} Vt[(c,k),(d,l)] X[(c,i),(d,l)]
    Contraction c; c.M = o; c.N = o; c.K = v * n1; c.Ki = n1;
    c.A = vw(Vt_, 0, sI, sA, 1);
    c.B = vw(Xd_, sA, 1, 0, sI);
    c.C = rm(Kki_, o);
    gemm_(c);
  }
  {  // Kac[a][c] = -sum_{k,(d,l)} X[(a,k),(d,l)] Vt[(c,k),(d,l)]
    Contraction c; c.M = v; c.N = v; c.K = o * n1; c.Ki = n1;
    c.A = vw(Xd_, 0, sA, sI, 1);
    c.B = vw(Vt_, sI, 1, 0, sA);
    c.C = rm(Kac_, v);
    c.alpha = -1.0;
    gemm_(c);
  }
  // ---- Lac (Ccsd.cxx:180-189) --------------------------------------------------
  copy_(Lac_, Kac_, v * v);
  if (!ccd) {
    {  // jG[G] = sum_{dk} Gph[G][dk] t[dk]
      Contraction c; c.M = G; c.N = 1; c.K = n1;
      c.A = rm(Gph, n1); c.B = vw(t, 0, 1, 0, 0); c.C = vw(jG_, 0, 1, 0, 0);
      gemm_(c);
    }
    {  // Lac[a][c] += 2 sum_G Gpp[G][c][a] jG[G]      (m = (c,a))
      Contraction c; c.M = v * v; c.N = 1; c.K = G; c.Mi = v;
      c.A = vw(Gpp, v, 1, 0, v * v);
      c.B = vw(jG_, 0, 1, 0, 0);
      c.C = vw(Lac_, 1, v, 0, 0);
      c.alpha = 2.0; c.beta = 1.0;
      gemm_(c);
    }
    {  // U[G][a][k] = sum_d Gpp[G][d][a] t[d][k]
      Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(tr(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(U_, o), n1);
      gemm_(c);
    }
    {  // Lac[a][c] -= sum_{G,k} U[G][a][k] Gph[G][c][k]
      Contraction c; c.M = v; c.N = v; c.K = G * o; c.Ki = o;
      c.A = vw(U_, 0, o, n1, 1);
      c.B = vw(Gph, n1, 1, 0, o);
      c.C = rm(Lac_, v);
      c.alpha = -1.0; c.beta = 1.0;
      gemm_(c);
    }
  }
  // ---- Lki (Ccsd.cxx:175,192-193) --------------------------------------------
  copy_(Lki_, Kki_, o * o);
  if (!ccd) {  // Lki[k][i] += sum_{c,l} (2 V_klic - V_lkic) t[c][l]
    Contraction c; c.M = o * o; c.N = 1; c.K = v * o; c.Mi = o; c.Ki = o;
    c.A = vw(Vh2_, v * o * o, v * o, o, 1);   // Vh2[i][k][c][l]: m = (i,k), k = (c,l)
    c.B = vw(t, o, 1, 0, 0);
    c.C = vw(Lki_, 1, o, 0, 0);
    c.beta = 1.0;
    gemm_(c);
  }
  // ---- R2 = Lac T2 - Lki T2 (Ccsd.cxx:195-197) ---------------------------------
  {
    Contraction c; c.M = v; c.N = o * n1; c.K = v;
    c.A = rm(Lac_, v); c.B = rm(Td, o * n1); c.C = rm(R2, o * n1);
    gemm_(c);
  }
  {
    Contraction c; c.M = o; c.N = n1; c.K = o; c.batch = v;
    c.A = tr(Lki_, o); c.B = with_batch(rm(Td, n1), o * n1); c.C = with_batch(rm(R2, n1), o * n1);
    c.alpha = -1.0; c.beta = 1.0;
    gemm_(c);
  }
  // ---- T1-dressed vertex terms (Ccsd.cxx:201-210) ----------------------------
  copy_(dGph_, Gph, G * n1);
  if (!ccd) {
    {  // dGph[G][a][i] -= sum_k t[a][k] Ghh[G][k][i]
      Contraction c; c.M = v; c.N = o; c.K = o; c.batch = G;
      c.A = rm(t, o); c.B = with_batch(rm(Ghh, o), o * o); c.C = with_batch(rm(dGph_, o), n1);
      c.alpha = -1.0; c.beta = 1.0;
      gemm_(c);
    }
    {  // W[G][b][j] = sum_c Gpp[G][b][c] t[c][j]
      Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(rm(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(W_, o), n1);
      gemm_(c);
    }
    {  // R2 += dGph^T W
      Contraction c; c.M = n1; c.N = n1; c.K = G;
      c.A = tr(dGph_, n1); c.B = rm(W_, n1); c.C = rm(R2, n1); c.beta = 1.0;
      tc_(c);
    }
    {  // R2[a][i][b][j] -= sum_k Vhhhp[j][i][k][a] t[b][k]      (batch j, m = (a,i))
      Contraction c; c.M = n1; c.N = v; c.K = o; c.batch = o; c.Mi = o;
      c.A = vw(Vhhhp_, 1, o * v, 0, v, 0, o * o * v);
      c.B = tr(t, o);
      c.C = vw(R2, o * n1, n1, 0, o, 0, 1);
      c.alpha = -1.0; c.beta = 1.0;
      gemm_(c);
    }
    {  // Q[(a,i)][k][j] = sum_c Vd[(a,i)][c][k] t[c][j]
      Contraction c; c.M = o; c.N = o; c.K = v; c.batch = n1;
      c.A = with_batch(tr(Vd_, o), n1); c.B = rm(t, o); c.C = with_batch(rm(Q_, o), o * o);
      gemm_(c);
    }
    {  // R2[(a,i)][b][j] -= sum_k t[b][k] Q[(a,i)][k][j]
      Contraction c; c.M = v; c.N = o; c.K = o; c.batch = n1;
      c.A = rm(t, o); c.B = with_batch(rm(Q_, o), o * o); c.C = with_batch(rm(R2, o), n1);
      c.alpha = -1.0; c.beta = 1.0;
      gemm_(c);
    }
  }
  // ---- ring Xakic (Ccsd.cxx:215-229) -------------------------------------------
  if (ccd) copy_(W8r_, Td, D2);
  else rank1_(W8r_, 1.0, Td, 2.0, t, n1);                        // X' = T2 + 2 T1 T1
  perm_(Yx_, W8r_, d4, p_ex, 1.0, 0.0);                          // X'^x
  axpby_(W8r_, 1.0, Td, -0.5, Yx_, 0.0, D2);                     // M1 = T - X'^x / 2
  perm_(Y_, Td, d4, p_ex, -1.0, 0.0);                            // -T^x
  axpby_(Y_, 2.0, Td, 1.0, Y_, 0.0, D2);                         // Y = 2T - T^x
  {  // Z = Gph M1
    Contraction c; c.M = G; c.N = n1; c.K = n1;
    c.A = rm(Gph, n1); c.B = rm(W8r_, n1); c.C = rm(Z_, n1);
    tc_(c);
  }
  // A2 = dGph + Gpp t + Z (in place in dGph on the fast path)
  if (A2_ != dGph_) copy_(A2_, dGph_, G * n1);
  if (!ccd) {  // A2[G][a][i] += sum_d Gpp[G][a][d] t[d][i]
    Contraction c; c.M = v; c.N = o; c.K = v; c.batch = G;
    c.A = with_batch(rm(Gpp, v), v * v); c.B = rm(t, o); c.C = with_batch(rm(A2_, o), n1);
    c.beta = 1.0;
    gemm_(c);
  }
  axpby_(A2_, 1.0, A2_, 1.0, Z_, 0.0, G * n1);
  {  // W1 = Gph Y
    Contraction c; c.M = G; c.N = n1; c.K = n1;
    c.A = rm(Gph, n1); c.B = rm(Y_, n1); c.C = rm(W1_, n1);
    tc_(c);
  }
  {  // R2 += A2^T W1
    Contraction c; c.M = n1; c.N = n1; c.K = G;
    c.A = tr(A2_, n1); c.B = rm(W1_, n1); c.C = rm(R2, n1); c.beta = 1.0;
    tc_(c);
  }
  {  // EX[(a,i),(c,k)] = -1/2 sum_{(b,j)} T[(a,i),(b,j)] V_bckj,  V_bckj = Vd[(b,k),(c,j)]
    Contraction c; c.M = n1; c.N = n1; c.K = n1; c.Ki = o; c.Ni = o;
    c.A = vw(Td, 0, n1, o, 1);
    c.B = vw(Vd_, sA, 1, sB, sI);
    c.C = vw(EX_, 0, n1, o, 1);
    c.alpha = -0.5;
    tc_(c);
  }
  {  // R2 += EX Y
    Contraction c; c.M = n1; c.N = n1; c.K = n1;
    c.A = rm(EX_, n1); c.B = rm(Y_, n1); c.C = rm(R2, n1); c.beta = 1.0;
    tc_(c);
  }
  // ---- crossed ring Xakci (Ccsd.cxx:233-253) ------------------------------------
  copy_(dGpp_, Gpp, G * v * v);
  copy_(dGhh_, Ghh, G * o * o);
  if (!ccd) {
    {  // dGpp[G][a][c] -= sum_l t[a][l] Gph[G][c][l]
      Contraction c; c.M = v; c.N = v; c.K = o; c.batch = G;
      c.A = rm(t, o); c.B = with_batch(tr(Gph, o), n1); c.C = with_batch(rm(dGpp_, v), v * v);
      c.alpha = -1.0; c.beta = 1.0;
      gemm_(c);
    }
    {  // dGhh[G][k][i] += sum_d Gph[G][d][k] t[d][i]
      Contraction c; c.M = o; c.N = o; c.K = v; c.batch = G;
      c.A = with_batch(tr(Gph, o), n1); c.B = rm(t, o); c.C = with_batch(rm(dGhh_, o), o * o);
      c.beta = 1.0;
      gemm_(c);
    }
  }
  {  // EX[(a,i),(c,k)] = -1/2 sum_{(b,j)} T_abji V_bckj = -1/2 T^x Ve (views of T and Vd)
    Contraction c; c.M = n1; c.N = n1; c.K = n1; c.Mi = o; c.Ki = o; c.Ni = o;
    c.A = vw(Td, sA, 1, sB, sI);
    c.B = vw(Vd_, sA, 1, sB, sI);
    c.C = vw(EX2_, sA, sI, o, 1);
    c.alpha = -0.5;
    tc_(c);
  }
  {  // EX[a][i][c][k] += sum_G dGpp[G][a][c] dGhh[G][k][i]      (m = (a,c), n = (k,i))
    Contraction c; c.M = v * v; c.N = o * o; c.K = G; c.Mi = v; c.Ni = o;
    c.A = vw(dGpp_, v, 1, 0, v * v);
    c.B = vw(dGhh_, 0, o * o, o, 1);
    c.C = vw(EX2_, o * n1, o, 1, n1);
    c.beta = 1.0;
    tc_(c);
  }
  {  // R2 -= EX T
    Contraction c; c.M = n1; c.N = n1; c.K = n1;
    c.A = rm(EX2_, n1); c.B = rm(Td, n1); c.C = rm(R2, n1);
    c.alpha = -1.0; c.beta = 1.0;
    tc_(c);
  }
  {  // R2_abij -= sum_ck T_ackj X_bkci : exchange pairing m = (a,j), n = (b,i)
    Contraction c; c.M = n1; c.N = n1; c.K = n1; c.Mi = o; c.Ni = o; c.Ki = o;
    c.A = vw(Td, sA, 1, sB, sI);           // T_ackj = T[(a,k),(c,j)]
    c.B = vw(EX2_, sB, 1, sA, sI);          // X_bkci = EX[(b,i),(c,k)]
    c.C = vw(R2, sA, 1, sB, sI);
    c.alpha = -1.0; c.beta = 1.0;
    tc_(c);
  }
  // ---- particle-particle ladder (Ccsd.cxx:283-333), before the symmetrisation:
  // L_abij = L_baji holds exactly on the real path, so the a >= b half of the
  // ladder (diagonal blocks at weight 1/2) is completed by P(ab,ij) below ------
  if (opt_.ppl) ppl(Xd_, R2, dGpp_);
  // ---- P(ab,ij) symmetrisation and +V (Ccsd.cxx:256,263) ----------------------
  sym_(R2, n1);
  axpby_(R2, 1.0, R2, 1.0, Vd_, 0.0, D2);
  // ---- hole-hole ladder (Ccsd.cxx:267-281) --------------------------------------
  copy_(Xkl1_, Vhhhh_, o * o * o * o);
  if (!ccd) {
    {  // Xkl1[k][l][i][j] += sum_c Vhhhp[k][l][i][c] t[c][j]
      Contraction c; c.M = o * o * o; c.N = o; c.K = v;
      c.A = rm(Vhhhp_, v); c.B = rm(t, o); c.C = rm(Xkl1_, o); c.beta = 1.0;
      gemm_(c);
    }
    {  // Xkl1[k][l][i][j] += sum_c Vhhhp[l][k][j][c] t[c][i]     (batch l, m = (k,j))
      Contraction c; c.M = o * o; c.N = o; c.K = v; c.batch = o; c.Mi = o;
      c.A = vw(Vhhhp_, o * v, v, 0, 1, 0, o * o * v);
      c.B = rm(t, o);
      c.C = vw(Xkl1_, o * o * o, 1, 0, o, 0, o * o);
      c.beta = 1.0;
      gemm_(c);
    }
  }
  {  // Xkl2[kl][ij] = sum_cd V_cdkl X_cdij  (m = (k,l), k = (c,d), n = (i,j))
    Contraction c; c.M = o * o; c.N = o * o; c.K = v * v; c.Mi = o; c.Ki = v; c.Ni = o;
    c.A = vw(Vd_, sI, 1, sA, sB);          // V_cdkl = Vd[(c,k),(d,l)]
    c.B = vw(Xd_, sA, sB, sI, 1);          // X_cdij = X[(c,i),(d,j)]
    c.C = vw(Xkl2_, o * o * o, o * o, o, 1);
    tc_(c);
  }
  {  // R2 += Xkl1 X_abkl  (m = (a,b), k = (k,l), n = (i,j))
    Contraction c; c.M = v * v; c.N = o * o; c.K = o * o; c.Mi = v; c.Ki = o; c.Ni = o;
    c.A = vw(Xd_, sA, sB, sI, 1);          // X_abkl = X[(a,k),(b,l)]
    c.B = vw(Xkl1_, o * o * o, o * o, o, 1);
    c.C = vw(R2, sA, sB, sI, 1);
    c.beta = 1.0;
    tc_(c);
    c.A.p = opt_.ppl ? cp(Td) : Xd_;       // T_abkl (ppl) or X_abkl, same view
    c.B.p = Xkl2_;
    tc_(c);
  }
  if (ccd) {
    zero_(R1, n1);
    profile_finish();
    return;
  }
  // ---- singles (Ccsd.cxx:339-375) ------------------------------------------------
  {
    Contraction c; c.M = v; c.N = o; c.K = v;
    c.A = rm(Kac_, v); c.B = rm(t, o); c.C = rm(R1, o);
    gemm_(c);
  }
  {
    Contraction c; c.M = v; c.N = o; c.K = o;
    c.A = rm(t, o); c.B = rm(Kki_, o); c.C = rm(R1, o); c.alpha = -1.0; c.beta = 1.0;
    gemm_(c);
  }
  {  // kck = 2 Vd t - Ve t,  Ve[(a,i),(b,j)] = V_abji = Vd[(a,j),(b,i)]
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(Vd_, n1); c.B = vw(t, 0, 1, 0, 0); c.C = vw(kck_, 0, 1, 0, 0); c.alpha = 2.0;
    gemm_(c);
    Contraction e; e.M = n1; e.N = 1; e.K = n1; e.Mi = o; e.Ki = o;
    e.A = vw(Vd_, sA, 1, sB, sI);
    e.B = vw(t, o, 1, 0, 0);
    e.C = vw(kck_, o, 1, 0, 0);
    e.alpha = -1.0; e.beta = 1.0;
    gemm_(e);
  }
  {  // R1 += (2T - T^x) kck
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(Y_, n1); c.B = vw(kck_, 0, 1, 0, 0); c.C = vw(R1, 0, 1, 0, 0); c.beta = 1.0;
    gemm_(c);
  }
  {  // P1[k][i] = sum_c kck[c][k] t[c][i];  R1 += t P1
    Contraction c; c.M = o; c.N = o; c.K = v;
    c.A = tr(kck_, o); c.B = rm(t, o); c.C = rm(P1_, o);
    gemm_(c);
    Contraction d; d.M = v; d.N = o; d.K = o;
    d.A = rm(t, o); d.B = rm(P1_, o); d.C = rm(R1, o); d.beta = 1.0;
    gemm_(d);
  }
  {  // R1 += 2 Vd t
    Contraction c; c.M = n1; c.N = 1; c.K = n1;
    c.A = rm(Vd_, n1); c.B = vw(t, 0, 1, 0, 0); c.C = vw(R1, 0, 1, 0, 0);
    c.alpha = 2.0; c.beta = 1.0;
    gemm_(c);
  }
  {  // P[G][i][c] = sum_k Ghh[G][i][k] t[c][k];  R1[a][i] -= sum_{G,c} Gpp[G][c][a] P[G][i][c]
    Contraction c; c.M = o; c.N = v; c.K = o; c.batch = G;
    c.A = with_batch(rm(Ghh, o), o * o); c.B = tr(t, o); c.C = with_batch(rm(P_, v), o * v);
    gemm_(c);
    Contraction d; d.M = v; d.N = o; d.K = G * v; d.Ki = v;
    d.A = vw(Gpp, 0, 1, v * v, v);
    d.B = vw(P_, o * v, 1, 0, v);
    d.C = rm(R1, o);
    d.alpha = -1.0; d.beta = 1.0;
    gemm_(d);
  }
  {  // F = Gph (2X - X^x);  R1[a][i] += sum_{G,x} Gpp[G][x][a] F[G][x][i]
    perm_(W8s_, Xd_, d4, p_ex, 1.0, 0.0);
    axpby_(W8s_, 2.0, Xd_, -1.0, W8s_, 0.0, D2);
    Contraction c; c.M = G; c.N = n1; c.K = n1;
    c.A = rm(Gph, n1); c.B = rm(W8s_, n1); c.C = rm(F_, n1);
    tc_(c);
    Contraction d; d.M = v; d.N = o; d.K = G * v; d.Ki = v;
    d.A = vw(Gpp, 0, 1, v * v, v);
    d.B = vw(F_, n1, o, 0, 1);
    d.C = rm(R1, o);
    d.beta = 1.0;
    gemm_(d);
  }
  {  // R1[a][i] -= sum_{k,(c,l)} X[(a,k),(c,l)] Vh2[i][k][c][l]
    Contraction c; c.M = v; c.N = o; c.K = o * n1; c.Ki = n1;
    c.A = vw(Xd_, 0, sA, sI, 1);
    c.B = vw(Vh2_, n1, 1, 0, o * n1);
    c.C = rm(R1, o);
    c.alpha = -1.0; c.beta = 1.0;
    gemm_(c);
  }
  profile_finish();
}

// Particle-particle ladder on virtual-pair slabs: for blocks X >= Y of s virtual
// orbitals and panels of c_n values of c,
//   V[x][y][c'][d] = sum_G dGpp[G][x0+x][c0+c'] dGpp[G][y0+y][d]      (GEMM, K = G)
//   R_{x y i j} += w sum_{c',d} V[x][y][c'][d] X_{c0+c',d,i,j}        (GEMM, K = c_n v)
// with w = 1/2 on diagonal blocks; added before R <- R + R^T, which supplies the
// mirrored blocks R_{y x j i} (the reference copies them, Ccsd.cxx:318-330).  Panelling c keeps the
// slab small enough for wide blocks (s^2 = 4096 rows), and each panel reads only
// its c-range of X.
void CcsdReal::ppl(const double* Xd, double* R2, const double* dGpp) {
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o;
  const int64_t s = slab_rows_, cn = slab_cols_;
  const int64_t nb = (v + s - 1) / s;
  // m = (x, y), k = (c', d), n = (i, j): the contraction of one block pair
  auto contraction = [&](int64_t x0, int64_t sx, int64_t y0, int64_t sy, int64_t c0, int64_t nc) {
    Contraction c; c.M = sx * sy; c.N = o * o; c.K = nc * v; c.Mi = sy; c.Ki = v; c.Ni = o;
    c.A = vw(slab_, sy * nc * v, nc * v, v, 1);
    c.B = vw(cp(Xd) + c0 * o * n1, o * n1, o, n1, 1);   // X_cdij = X[(c,i),(d,j)]
    c.C = vw(R2 + x0 * o * n1 + y0 * o, o * n1, o, n1, 1);
    c.alpha = x0 == y0 ? 0.5 : 1.0;  // the symmetrisation that follows adds the mirror
    c.beta = 1.0;
    return c;
  };
  auto build_of = [&](int64_t x0, int64_t sx, int64_t y0, int64_t sy, int64_t c0, int64_t nc) {
    Contraction build;  // m = (x, c'), n = (y, d), slab[x][y][c'][d]
    build.M = sx * nc; build.N = sy * v; build.K = G; build.Mi = nc; build.Ni = v;
    build.A = vw(cp(dGpp) + x0 * v + c0, v, 1, 0, v * v);
    build.B = vw(cp(dGpp) + y0 * v, 0, v * v, v, 1);
    build.C = vw(slab_, sy * nc * v, v, nc * v, 1);
    return build;
  };
  // Split form: the X panel (operand B of every contraction of one c range, shared
  // by all block pairs: B depends on N = o^2, K = c_n v and the X view only) is
  // sliced once per c range into a region kept beside the per-contraction scratch.
  const Contraction c_first = contraction(0, std::min(s, v), 0, std::min(s, v), 0, std::min(cn, v));
  const bool prepack = !taping_ && split_ok(c_first) && split_single_panel(c_first) && nb > 1;
  if (prepack) {
    size_t regular = 0;
    for (int64_t c0 = 0; c0 < v; c0 += cn) {
      const int64_t nc = std::min(cn, v - c0);
      for (int64_t X = 0; X < nb; ++X) {
        const int64_t sx = std::min(s, v - X * s);
        for (int64_t Yb = 0; Yb <= X; ++Yb) {
          const int64_t sy = std::min(s, v - Yb * s);
          const Contraction b = build_of(X * s, sx, Yb * s, sy, c0, nc);
          const Contraction c = contraction(X * s, sx, Yb * s, sy, c0, nc);
          if (split_ok(b)) regular = std::max(regular, gemm_split_scratch_bytes(b));
          if (split_ok(c)) regular = std::max(regular, split_scratch_bytes_packed_b(c));
        }
      }
    }
    split_reserve(regular, split_packed_b_bytes(c_first));
  }
  for (int64_t c0 = 0; c0 < v; c0 += cn) {
    const int64_t nc = std::min(cn, v - c0);
    SplitPackedB pb;
    if (prepack) {  // timed with the split contractions (no flops of its own)
      const bool prof = profile_ && count_flops_;
      const size_t k = ev_flops_.size();
      if (prof) {
        while (ev_.size() < 2 * (k + 1)) ev_.push_back(ops::event_create());
        ev_flops_.push_back(0.0);
        ev_split_.push_back(1);
        ev_shape_.push_back({0, o * o, nc * v, 1});
        ops::event_record(ev_[2 * k], s_);
      }
      pb = split_pack_b(contraction(0, s, 0, s, c0, nc), split_extra_, s_);
      if (prof) ops::event_record(ev_[2 * k + 1], s_);
    }
    for (int64_t X = 0; X < nb; ++X) {
      for (int64_t Yb = 0; Yb <= X; ++Yb) {
        const int64_t x0 = X * s, sx = std::min(s, v - x0);
        const int64_t y0 = Yb * s, sy = std::min(s, v - y0);
        const Contraction build = build_of(x0, sx, y0, sy, c0, nc);
        tc_(build);
        {
          const Contraction c = contraction(x0, sx, y0, sy, c0, nc);
          if (prepack && split_ok(c)) tc_packed_b_(c, pb);
          else tc_(c);
          if (taping_) {  // the slab is rebuilt before this contraction's adjoint
            tape_.back().recompute = true;
            tape_.back().pre = build;
            tape_.back().zero_p = slab_;
            tape_.back().zero_n = slab_rows_ * slab_rows_ * slab_cols_ * v;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Reverse mode: the residual at T recorded once, replayed backwards per vjp.
void CcsdReal::energy_gradients(const double* T, double* g, double* Vd_bar) {
  const int64_t o = sys_.o, v = sys_.v, n1 = v * o, D2 = n1 * n1;
  const int64_t d4[4] = {v, o, v, o};
  const int p_ex[4] = {0, 3, 2, 1};
  double* g2 = g + n1;
  ops::permute4(g2, Vd_, d4, p_ex, -1.0, 0.0, s_);       // dE/dT2 = 2 Vd - Vd^x
  ops::axpby(g2, 2.0, Vd_, 1.0, g2, 0.0, D2, s_);
  Contraction c; c.M = n1; c.N = 1; c.K = n1;           // dE/dT1 = 2 (dE/dT2) T1
  c.A = rm(g2, n1); c.B = vw(cp(T), 0, 1, 0, 0); c.C = vw(g, 0, 1, 0, 0); c.alpha = 2.0;
  gemm(c, s_, scratch_);
  if (Vd_bar) {  // dE/dVd = 2 X - X^x, X staged in the forward output buffer (never
                 // read by the reverse sweep)
    if (!Rf_) Rf_ = take(n1 + D2);
    double* X = Rf_ + n1;
    ops::rank1(X, 1.0, T + n1, 1.0, T, n1, s_);
    ops::permute4(Vd_bar, X, d4, p_ex, -1.0, 0.0, s_);
    ops::axpby(Vd_bar, 2.0, X, 1.0, Vd_bar, 0.0, D2, s_);
  }
}

void CcsdReal::prepare_vjp(const double* T) {
  if (!adjoint_) throw Error(ERR_STATE, "reverse mode needs a schedule built in adjoint mode");
  if (!T) throw Error(ERR_INVALID_ARGUMENT, "prepare_vjp: no amplitudes");
  const int64_t n1 = sys_.v * sys_.o;
  if (!Rf_) Rf_ = take(n1 + n1 * n1);
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

void CcsdReal::vjp(const double* Rbar, double* Tbar, const VertexBar* gbar,
                   const double* extra_Vd_bar) {
  if (!Tprep_) throw Error(ERR_STATE, "vjp before prepare_vjp");
  const int64_t o = sys_.o, v = sys_.v, G = sys_.G, n1 = v * o, n = n1 + n1 * n1;
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
  if (gbar) {
    if (gbar->Gpp) regions_.push_back({sys_.Gpp, G * v * v, gbar->Gpp});
    if (gbar->Gph) regions_.push_back({sys_.Gph, G * n1, gbar->Gph});
    if (gbar->Ghh) regions_.push_back({sys_.Ghh, G * o * o, gbar->Ghh});
    if (gbar->Ghp) regions_.push_back({sys_.Ghp, G * n1, gbar->Ghp});
  }
  ops::d2d(bar_of(Rf_), Rbar, n, s_);
  try {
    reverse(tape_);
    // the amplitudes are symmetric, T_abij = T_baji: project the T2 adjoint
    ops::symmetrize(Tbar + n1, n1, s_);
    ops::axpby(Tbar + n1, 0.5, Tbar + n1, 0.0, nullptr, 0.0, n1 * n1, s_);
    if (gbar) {
      if (extra_Vd_bar) ops::axpby(bar_of(Vd_), 1.0, bar_of(Vd_), 1.0, extra_Vd_bar, 0.0, n1 * n1, s_);
      reverse(integrals_tape_);
    }
  } catch (...) {
    regions_.clear();
    throw;
  }
  regions_.clear();
}

}  // namespace cc4s_b200
