// Direct-ring CCD residual, restated from cc4s Drccd::getResiduum
// (src/main/algorithms/coupledcluster/Drccd.cxx:31-104):
//   R2 = 2 Vphhp_akic T_cbkj;  R2 += R2^(ba,ji);  R2 += Vpphh;
//   R2 += 2 W_klcd T_acik T_dblj,  W = 2 Vhhpp (- Vhhpp_lkcd with adjacentPairsExchange).
// The ring term is contracted through the vertex (Gamma^T (Gamma T)) without
// forming Vphhp; the quadratic term is T (W T) with W built once.
#include "drccd.h"

namespace cc4s_b200 {

Drccd::Drccd(int64_t o, int64_t v, int64_t G, bool complex_path, double* Gph, double* Ghp,
             const DrccdOptions& opt, Stream s)
    : Schedule(s), o_(o), v_(v), G_(G), D2_(o * v * o * v), cplx_(complex_path), Gph_(Gph),
      Ghp_(Ghp), opt_(opt) {
  so_ = o; sv_ = v; sG_ = G; scplx_ = complex_path; sGph_ = Gph; sGhp_ = Ghp;
  const int64_t n1 = o * v, D2 = D2_, pl = cplx_ ? 2 : 1;
  const int64_t gi = cplx_ ? G * n1 : 0;  // imaginary plane of Gph / Ghp
  const int64_t di = cplx_ ? D2 : 0;
  try {
    scratch_.elems = static_cast<size_t>(int64_t(1) << 22);
    scratch_.p = take(scratch_.elems);
    Vd_ = take(pl * D2); Ve_ = take(pl * D2); Wq_ = take(pl * D2); Q_ = take(pl * D2);
    W1_ = take(pl * G * n1);
  } catch (...) {
    release_all();
    throw;
  }
  count_flops_ = false;
  {  // Vd = V_abij (real: Gph^T Gph; complex: conj(Ghp)^T Gph)
    Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o;
    c.A = cplx_ ? vw(Ghp, 1, v, 0, n1) : vw(Gph, o, 1, 0, n1);
    c.B = rm(Gph, n1);
    c.C = vw(Vd_, o * n1, n1, 0, 1);  // m = (a,i) split like the A view
    zgemm(c, gi, gi, di, cplx_, false);
  }
  {
    const int64_t d4[4] = {v, o, v, o};
    const int pm[4] = {2, 1, 0, 3};  // Ve[(a,i),(b,j)] = V_baij
    ops::permute4(Ve_, Vd_, d4, pm, 1.0, 0.0, s_);
    if (cplx_) ops::permute4(Ve_ + D2, Vd_ + D2, d4, pm, 1.0, 0.0, s_);
  }
  {  // Wq[(c,k),(d,l)] = 2 Vhhpp_klcd
    Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o; c.Ni = o;
    c.A = cplx_ ? vw(Gph, o, 1, 0, n1) : vw(Ghp, 1, v, 0, n1);
    c.B = vw(Ghp, 0, n1, 1, v);
    c.C = vw(Wq_, o * n1, n1, o, 1);
    c.alpha = 2.0;
    zgemm(c, gi, gi, di, cplx_, false);
  }
  if (opt_.adjacent_pairs_exchange) {  // Wq[(c,k),(d,l)] -= Vhhpp_lkcd
    Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o; c.Ni = v;
    c.A = cplx_ ? vw(Gph, o, 1, 0, n1) : vw(Ghp, 1, v, 0, n1);
    c.B = vw(Ghp, 0, n1, v, 1);
    c.C = vw(Wq_, o * n1, 1, n1, o);
    c.alpha = -1.0; c.beta = 1.0;
    zgemm(c, gi, gi, di, cplx_, false);
  }
  count_flops_ = true;
}

void Drccd::residual(const double* T, double* R) {
  const int64_t o = o_, v = v_, G = G_, n1 = o * v, D2 = D2_;
  const int64_t pl = n1 + D2;                 // imaginary plane of amplitude vectors
  const int64_t ti = cplx_ ? pl : 0, gi = cplx_ ? G * n1 : 0, di = cplx_ ? D2 : 0;
  double* R1 = R;
  double* R2 = R + n1;
  ops::zero(R1, n1, s_);
  if (cplx_) ops::zero(R1 + pl, n1, s_);
  if (!T) {  // Drccd.cxx:61-66
    ops::d2d(R2, Vd_, D2, s_);
    if (cplx_) ops::d2d(R2 + pl, Vd_ + D2, D2, s_);
    return;
  }
  flops_ = 0.0;
  double* Td = cp(T + n1);
  {  // W1[G][(b,j)] = sum_{c,k} Ghp[G][k][c] T[(c,k),(b,j)]
    Contraction c; c.M = G; c.N = n1; c.K = n1; c.Ki = o;
    c.A = vw(Ghp_, 0, n1, 1, v); c.B = vw(Td, o * n1, n1, 0, 1); c.C = rm(W1_, n1);
    zgemm(c, gi, ti, cplx_ ? G * n1 : 0, false, false, true);
  }
  {  // R2 = 2 Vphhp_akic T_cbkj = 2 sum_G (Gph | conj Ghp^T)[G][(a,i)] W1[G][(b,j)]
    Contraction c; c.M = n1; c.N = n1; c.K = G; c.Mi = o;
    c.A = cplx_ ? vw(Ghp_, 1, v, 0, n1) : vw(Gph_, o, 1, 0, n1);
    c.B = rm(W1_, n1); c.C = vw(R2, o * n1, n1, 0, 1); c.alpha = 2.0;
    zgemm(c, gi, cplx_ ? G * n1 : 0, ti, cplx_, false, true);
  }
  ops::symmetrize(R2, n1, s_);
  ops::axpby(R2, 1.0, R2, 1.0, Vd_, 0.0, D2, s_);
  if (cplx_) {
    ops::symmetrize(R2 + pl, n1, s_);
    ops::axpby(R2 + pl, 1.0, R2 + pl, 1.0, Vd_ + D2, 0.0, D2, s_);
  }
  if (!opt_.linearized) {
    {  // Q = Wq T
      Contraction c; c.M = n1; c.N = n1; c.K = n1;
      c.A = rm(Wq_, n1); c.B = rm(Td, n1); c.C = rm(Q_, n1);
      zgemm(c, di, ti, di, false, false, true);
    }
    {  // R2 += 2 T Q
      Contraction c; c.M = n1; c.N = n1; c.K = n1;
      c.A = rm(Td, n1); c.B = rm(Q_, n1); c.C = rm(R2, n1); c.alpha = 2.0; c.beta = 1.0;
      zgemm(c, ti, di, ti, false, false, true);
    }
  }
  profile_finish();
}

}  // namespace cc4s_b200
