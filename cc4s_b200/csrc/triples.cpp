// Perturbative triples (T) energy, real and complex paths (triples.h).
#include "triples.h"

#include <algorithm>
#include <array>
#include <set>
#include <vector>

namespace cc4s_b200 {

namespace {
// Block array budget: planes * (block * o)^3 doubles, below the 126 MB L2 of the B200.
constexpr int64_t BLOCK_BUDGET_DOUBLES = int64_t(12) << 20;
const int PERMS[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

int perm_index(const int p[3]) {
  for (int k = 0; k < 6; ++k)
    if (PERMS[k][0] == p[0] && PERMS[k][1] == p[1] && PERMS[k][2] == p[2]) return k;
  return -1;
}
// (a . b)[m] = a[b[m]]: taking the hole indices in the order b, then a.
void compose(const int a[3], const int b[3], int out[3]) {
  for (int m = 0; m < 3; ++m) out[m] = a[b[m]];
}
void invert(const int a[3], int out[3]) {
  for (int m = 0; m < 3; ++m) out[a[m]] = m;
}
}  // namespace

int64_t Triples::auto_block(int64_t o, int64_t v, int planes) {
  int64_t nb = 1;
  while (nb < v) {
    const int64_t L = (nb + 1) * o;
    if (planes * L * L * L > BLOCK_BUDGET_DOUBLES) break;
    ++nb;
  }
  return nb;
}

void Triples::coefficients(int64_t A, int64_t B, int64_t C, double coef[6]) {
  const int64_t blk[3] = {A, B, C};
  static const int T23[3] = {0, 2, 1};
  static const int CINV[3] = {2, 0, 1};  // inverse of the left rotation (1, 2, 0)
  for (int k = 0; k < 6; ++k) coef[k] = 0.0;
  std::set<std::array<int64_t, 3>> seen;
  for (const auto& s : PERMS) {
    const std::array<int64_t, 3> key = {blk[s[0]], blk[s[1]], blk[s[2]]};
    if (!seen.insert(key).second) continue;
    int si[3], t[3], u[3];
    invert(s, si);
    coef[0] += 4.0 / 3.0;
    compose(s, T23, t);
    compose(t, si, u);
    coef[perm_index(u)] += -2.0;
    compose(s, CINV, t);
    compose(t, si, u);
    coef[perm_index(u)] += 2.0 / 3.0;
  }
}

Triples::Triples(const RealSystem& sys, const ComplexSystem* cs, const TriplesOptions& opt,
                 Stream s)
    : Schedule(s), sys_(sys), cplx_(cs != nullptr), reference_form_(opt.reference_form) {
  o_ = sys.o; v_ = sys.v; n1_ = o_ * v_;
  const int64_t o = o_, v = v_, n1 = n1_, G = sys.G;
  const int pl = cplx_ ? 2 : 1;
  nb_ = opt.block > 0 ? std::min(opt.block, v) : auto_block(o, v, pl);
  const int64_t nbk = (v + nb_ - 1) / nb_;
  ntri_ = nbk * (nbk + 1) * (nbk + 2) / 6;
  const int64_t L = nb_ * o;
  if (cplx_) {
    vi_pphh_ = n1 * n1; vi_ppph_ = v * n1 * v; vi_hhhp_ = o * n1 * o; si_ = L * L * L;
  }
  try {
    scratch_.elems = static_cast<size_t>(int64_t(1) << 22);
    scratch_.p = take(scratch_.elems);
    Vpphh_ = take(pl * n1 * n1);
    Vppph_ = take(pl * v * n1 * v);
    Vhhhp_ = take(pl * o * n1 * o);
    S_ = take(pl * L * L * L);
    ws_ = take(2048);
    slots_ = take(2 * ntri_ + 2);
  } catch (...) {
    release_all();
    throw;
  }
  // Vertex slices Gamma[G][p][q] (q fastest); complex: imaginary plane after the real one.
  double* Gpp = cplx_ ? cs->Gpp : sys.Gpp;
  double* Gph = cplx_ ? cs->Gph : sys.Gph;
  double* Ghh = cplx_ ? cs->Ghh : sys.Ghh;
  double* Ghp = cplx_ ? cs->Ghp : sys.Ghp;
  const int64_t gpp = cplx_ ? G * v * v : 0, gph = cplx_ ? G * n1 : 0, ghh = cplx_ ? G * o * o : 0;
  void* e0 = ops::event_create();
  void* e1 = ops::event_create();
  ops::event_record(e0, s_);
  {  // V_abij: real sum_G Gamma_Gai Gamma_Gbj; complex sum_G conj(Gamma_Gia) Gamma_Gbj
    Contraction c; c.M = n1; c.Mi = o; c.N = n1; c.K = G;
    c.A = cplx_ ? vw(Ghp, 1, v, 0, n1) : vw(Gph, o, 1, 0, n1);
    c.B = vw(Gph, 0, n1, 0, 1);
    c.C = vw(Vpphh_, o * n1, n1, 0, 1);
    zgemm(c, gph, gph, vi_pphh_, cplx_, false, true);
  }
  {  // V_bcdk as [b][(c,k)][d]: real sum_G Gamma_Gbd Gamma_Gck; complex conj(Gamma_Gdb) Gamma_Gck
    Contraction c; c.M = n1; c.N = v * v; c.Ni = v; c.K = G;
    c.A = vw(Gph, 0, 1, 0, n1);
    c.B = cplx_ ? vw(Gpp, 0, v * v, 1, v) : vw(Gpp, 0, v * v, v, 1);
    c.C = vw(Vppph_, 0, v, n1 * v, 1);
    zgemm(c, gph, gpp, vi_ppph_, false, cplx_, true);
  }
  {  // V_jklc as [j][(c,k)][l]: real sum_G Gamma_Gjl Gamma_Gkc; complex conj(Gamma_Glj) Gamma_Gkc
    Contraction c; c.M = n1; c.Mi = o; c.N = o * o; c.Ni = o; c.K = G;
    c.A = vw(Ghp, 1, v, 0, o * v);
    c.B = cplx_ ? vw(Ghh, 0, o * o, 1, o) : vw(Ghh, 0, o * o, o, 1);
    c.C = vw(Vhhhp_, o * o, o, n1 * o, 1);
    zgemm(c, gph, ghh, vi_hhhp_, false, cplx_, true);
  }
  ops::event_record(e1, s_);
  setup_seconds_ = ops::event_ms(e0, e1) * 1e-3;
  ops::event_destroy(e0);
  ops::event_destroy(e1);
}

void Triples::residual(const double*, double*) {
  throw Error(ERR_STATE, "the triples schedule has no residual");
}

// S += the six permutations of the base term X for one block triple.  Term
// (p, q, r): the pair (x1, y1) of X is the pair at block position p, x2 and y2
// are the virtual and hole index at position q, the pair (x3, y3) is position r.
// particle = true: the six d sums; false: the six l sums.
void Triples::connected(const double* T2, const ops::TriplesBlock& b, const int64_t X[3],
                        const int64_t n[3], bool particle) {
  static const int PQR[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}};
  const int64_t o = o_, v = v_, n1 = n1_;
  const int64_t sP[3] = {b.L[1] * b.L[2], b.L[2], 1};
  const int64_t ti = cplx_ ? n1 + n1 * n1 : 0;  // imaginary plane of the amplitude vector
  double* T = cp(T2);
  for (const auto& t : PQR) {
    const int p = t[0], q = t[1], r = t[2];
    if (particle) {  // + sum_d T[(x1,y1),(d,y2)] V[x2][(x3,y3)][d]
      Contraction c;
      c.M = b.L[p] * o; c.N = n[q] * b.L[r]; c.Ni = b.L[r]; c.K = v;
      if (p == 2) {  // pair p is the output's contiguous index: make it the inner row level
        c.Mi = b.L[p];
        c.A = vw(T + b.P[p] * n1, 1, n1, 0, o);
        c.C = vw(S_, sP[q], sP[p], o * sP[q], sP[r]);
      } else {
        c.Mi = o;
        c.A = vw(T + b.P[p] * n1, n1, 1, 0, o);
        c.C = vw(S_, sP[p], sP[q], o * sP[q], sP[r]);
      }
      c.B = vw(Vppph_ + X[q] * n1 * v + b.P[r] * v, 0, 1, n1 * v, v);
      c.alpha = 1.0; c.beta = 1.0;
      zgemm(c, ti, vi_ppph_, si_, false, false, true);
    } else {  // - sum_l T[(x1,y1),(x2,l)] V[y2][(x3,y3)][l]   (conj(V) on the complex path)
      Contraction c;
      c.M = b.L[p] * n[q]; c.N = o * b.L[r]; c.K = o;
      if (p == 2) {  // rows (virtual q, pair p) with pair p inner
        c.Mi = b.L[p];
        c.A = vw(T + b.P[p] * n1 + X[q] * o, o, n1, 0, 1);
        c.C = vw(S_, o * sP[q], sP[p], 0, 0);
      } else {
        c.Mi = n[q];
        c.A = vw(T + b.P[p] * n1 + X[q] * o, n1, o, 0, 1);
        c.C = vw(S_, sP[p], o * sP[q], 0, 0);
      }
      if (q == 2) {  // hole q is the output's contiguous index: columns (pair r, hole q)
        c.Ni = o;
        c.B = vw(Vhhhp_ + b.P[r] * o, 0, 1, o, n1 * o);
        c.C.s_co = sP[r]; c.C.s_ci = sP[q];
      } else {
        c.Ni = b.L[r];
        c.B = vw(Vhhhp_ + b.P[r] * o, 0, 1, n1 * o, o);
        c.C.s_co = sP[q]; c.C.s_ci = sP[r];
      }
      c.alpha = -1.0; c.beta = 1.0;
      zgemm(c, ti, vi_hhhp_, si_, false, cplx_, true);
    }
  }
}

TriplesOutcome Triples::run(const double* T) {
  const int64_t o = o_, v = v_, n1 = n1_, nb = nb_;
  const int64_t nbk = (v + nb - 1) / nb;
  const int64_t plane = n1 + n1 * n1;
  const double* t1 = T;
  const double* t1i = cplx_ ? T + plane : nullptr;
  const double* T2 = T + n1;
  const double* Vi = cplx_ ? Vpphh_ + vi_pphh_ : nullptr;
  double* Si = cplx_ ? S_ + si_ : nullptr;
  TriplesOutcome out;
  out.block = nb;
  out.block_triples = ntri_;
  out.setup_seconds = setup_seconds_;
  out.flops = 2.0 * double(o) * o * o * double(v) * v * v * double(o + v);
  void* e0 = ops::event_create();
  void* e1 = ops::event_create();
  // profile: events around the four phases of every block triple
  std::vector<void*> pev;
  if (profile_) {
    pev.resize(5 * static_cast<size_t>(ntri_));
    for (auto& e : pev) e = ops::event_create();
  }
  ops::event_record(e0, s_);
  int64_t t = 0;
  for (int64_t A = 0; A < nbk; ++A)
    for (int64_t B = A; B < nbk; ++B)
      for (int64_t C = B; C < nbk; ++C, ++t) {
        const int64_t X[3] = {A * nb, B * nb, C * nb};
        const int64_t n[3] = {std::min(nb, v - X[0]), std::min(nb, v - X[1]),
                              std::min(nb, v - X[2])};
        ops::TriplesBlock b;
        b.o = o; b.n1 = n1;
        for (int m = 0; m < 3; ++m) { b.P[m] = X[m] * o; b.L[m] = n[m] * o; }
        if (profile_) ops::event_record(pev[5 * t], s_);
        ops::triples_singles(S_, Si, t1, t1i, Vpphh_, Vi, b, s_);
        if (profile_) ops::event_record(pev[5 * t + 1], s_);
        connected(T2, b, X, n, true);
        if (profile_) ops::event_record(pev[5 * t + 2], s_);
        connected(T2, b, X, n, false);
        if (profile_) ops::event_record(pev[5 * t + 3], s_);
        double coef[6];
        coefficients(A, B, C, coef);
        ops::triples_energy(S_, Si, t1, t1i, Vpphh_, Vi, sys_.eh, sys_.ep, b, coef, ws_,
                            slots_ + 2 * t, s_);
        if (profile_) ops::event_record(pev[5 * t + 4], s_);
        out.executed_flops += (cplx_ ? 4.0 : 1.0) * 12.0 * double(n[0] * n[1] * n[2]) * o * o * o *
                              double(v + o);
      }
  ops::sum_partials_to(slots_ + 2 * ntri_, slots_, static_cast<int>(ntri_), 2, s_);
  ops::event_record(e1, s_);
  out.seconds = ops::event_ms(e0, e1) * 1e-3;
  ops::event_destroy(e0);
  ops::event_destroy(e1);
  for (int64_t k = 0; k < static_cast<int64_t>(pev.size()) / 5; ++k)
    for (int ph = 0; ph < 4; ++ph)
      out.phase_seconds[ph] += 1e-3 * ops::event_ms(pev[5 * k + ph], pev[5 * k + ph + 1]);
  for (void* e : pev) ops::event_destroy(e);
  double sums[2];
  ops::d2h(sums, slots_ + 2 * ntri_, 2, s_);
  ops::sync(s_);
  if (device_error()) throw Error(ERR_TIMEOUT, "tensor-core kernel wait expired in (T)");
  // Re conj(W) Z = ReW ReZ + ImW ImZ;  Re conj(W) conj(Z) = ReW ReZ - ImW ImZ
  out.energy = reference_form_ ? sums[0] - sums[1] : sums[0] + sums[1];
  return out;
}

}  // namespace cc4s_b200
