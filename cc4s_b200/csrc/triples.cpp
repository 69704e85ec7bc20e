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
    : Schedule(s), sys_(sys), cs_(cs), cplx_(cs != nullptr), reference_form_(opt.reference_form),
      complete_(opt.complete) {
  o_ = sys.o; v_ = sys.v; n1_ = o_ * v_;
  const int64_t o = o_, v = v_, n1 = n1_, G = sys.G;
  const int pl = cplx_ ? 2 : 1;
  nb_ = opt.block > 0 ? std::min(opt.block, v) : auto_block(o, v, pl * (complete_ ? 2 : 1));
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
    kc_ = v + o;
    ai_ = cplx_ ? n1 * o * kc_ : 0;
    bi_ = cplx_ ? v * n1 * kc_ : 0;
    Ac_ = take(pl * n1 * o * kc_);
    Bc_ = take(pl * v * n1 * kc_);
    if (complete_) {
      Ip_ = take(pl * v * n1 * v);
      Ih_ = take(pl * o * n1 * o);
      Mb_ = take(pl * L * L * L);
      AcM_ = take(pl * n1 * o * kc_);
      BcM_ = take(pl * v * n1 * kc_);
    }
    ws_ = take(2048);
    slots_ = take(2 * ntri_ + 2);
    if (complete_) cr_slots_ = take(2 * ntri_ + 2);
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

// S += the six permutations of the base term X for one block triple, the particle
// and the hole half of each in one contraction over K = v + o.  Term (p, q, r): the
// pair (x1, y1) of X is the pair at block position p, x2 and y2 are the virtual and
// hole index at position q, the pair (x3, y3) is position r.  Its particle half
//   + sum_d T[(x1,y1),(d,y2)] V^p[x2][(x3,y3)][d]
// has rows (pair p, hole q) and columns (virtual q, pair r); the hole half of the
// term (r, q, p),
//   - sum_l T[(x3,y3),(x2,l)] V^h[y2][(x1,y1)][l]   (conj(V^h) on the complex path),
// writes the same elements of S with the same rows and columns (its transpose), so
// rows of Ac hold [T | -V^h] and columns of Bc hold [V^p | T] along K.
void Triples::connected(const ops::TriplesBlock& b, const int64_t X[3], const int64_t n[3],
                        const double* Ac, const double* Bc, double* S) {
  static const int PQR[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}};
  const int64_t o = o_, n1 = n1_, kc = kc_;
  const int64_t sP[3] = {b.L[1] * b.L[2], b.L[2], 1};
  for (const auto& t : PQR) {
    const int p = t[0], q = t[1], r = t[2];
    Contraction c;
    c.M = b.L[p] * o; c.N = n[q] * b.L[r]; c.Ni = b.L[r]; c.K = kc;
    double* A0 = cp(Ac) + b.P[p] * o * kc;
    if (p == 2) {  // pair p is the output's contiguous index: make it the inner row level
      c.Mi = b.L[p];
      c.A = vw(A0, kc, o * kc, 0, 1);
      c.C = vw(S, sP[q], sP[p], o * sP[q], sP[r]);
    } else {
      c.Mi = o;
      c.A = vw(A0, o * kc, kc, 0, 1);
      c.C = vw(S, sP[p], sP[q], o * sP[q], sP[r]);
    }
    c.B = vw(cp(Bc) + (X[q] * n1 + b.P[r]) * kc, 0, 1, n1 * kc, kc);
    c.alpha = 1.0; c.beta = 1.0;
    zgemm(c, ai_, bi_, si_, false, false, true);
  }
}

void Triples::pack_operands(int w, const double* Ac, const double* Bc) {
  const int64_t o = o_, v = v_, n1 = n1_, kc = kc_;
  const int planes = cplx_ ? 2 : 1;
  const size_t ba = split_operand_bytes(n1 * o, kc), bb = split_operand_bytes(v * n1, kc);
  const size_t per = 2 * ba + bb;
  if (!sl_mem_[w]) sl_mem_[w] = take((planes * per + 7) / 8);
  unsigned char* p = reinterpret_cast<unsigned char*>(sl_mem_[w]);
  for (int pl = 0; pl < planes; ++pl, p += per) {
    const double* A = Ac + pl * ai_;
    const double* B = Bc + pl * bi_;
    Sliced& s = sl_[w][pl];
    s.A = split_pack_operand(A, n1 * o, 0, 0, kc, kc, 1, p, s_);
    s.A2 = split_pack_operand(A, o * n1, n1, kc, o * kc, kc, 1, p + ba, s_);
    s.B = split_pack_operand(B, v * n1, 0, 0, kc, kc, 1, p + 2 * ba, s_);
  }
}

void Triples::connected_packed(const ops::TriplesBlock& b, const int64_t X[3], const int64_t n[3],
                               int w, double* S) {
  static const int PQR[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}};
  const int64_t o = o_, n1 = n1_;
  const int64_t sP[3] = {b.L[1] * b.L[2], b.L[2], 1};
  for (const auto& t : PQR) {
    const int p = t[0], q = t[1], r = t[2];
    Contraction c;
    c.M = b.L[p] * o; c.N = n[q] * b.L[r]; c.Ni = b.L[r]; c.K = kc_;
    SplitRuns ar, br;
    const bool inner_pair = p == 2;  // rows (hole q, pair p): pair p contiguous in S
    if (inner_pair) {
      c.Mi = b.L[p];
      c.C = vw(S, sP[q], sP[p], o * sP[q], sP[r]);
      ar.base = b.P[p]; ar.run = b.L[p]; ar.stride = n1;
    } else {
      c.Mi = o;
      c.C = vw(S, sP[p], sP[q], o * sP[q], sP[r]);
      ar.base = b.P[p] * o; ar.run = c.M; ar.stride = 0;
    }
    br.base = X[q] * n1 + b.P[r]; br.run = b.L[r]; br.stride = n1;
    c.alpha = 1.0; c.beta = 1.0;
    if (c.M < 64 || c.N < 64) {  // too small for the split form (a ragged last block): FP64
      const double* Ac = w ? AcM_ : Ac_;
      const double* Bc = w ? BcM_ : Bc_;
      c.A = inner_pair ? vw(cp(Ac) + b.P[p] * o * kc_, kc_, o * kc_, 0, 1)
                       : vw(cp(Ac) + b.P[p] * o * kc_, o * kc_, kc_, 0, 1);
      c.B = vw(cp(Bc) + (X[q] * n1 + b.P[r]) * kc_, 0, 1, n1 * kc_, kc_);
      zgemm(c, ai_, bi_, si_, false, false, false);
      continue;
    }
    const Sliced& re = sl_[w][0];
    auto A = [&](const Sliced& s) -> const SplitOperand& { return inner_pair ? s.A2 : s.A; };
    tc_prepacked_(c, A(re), ar, re.B, br);
    if (cplx_) {  // Re C -= Im A Im B; Im C += Re A Im B + Im A Re B
      const Sliced& im = sl_[w][1];
      Contraction d = c;
      d.alpha = -1.0;
      tc_prepacked_(d, A(im), ar, im.B, br);
      d = c;
      d.C.p = S + si_;
      tc_prepacked_(d, A(re), ar, im.B, br);
      tc_prepacked_(d, A(im), ar, re.B, br);
    }
  }
}

void Triples::concat_operands(const double* T, const double* Vp, const double* Vh, double* Ac,
                              double* Bc) {
  const int64_t o = o_, v = v_, n1 = n1_, kc = kc_;
  const int64_t plane = n1 + n1 * n1;
  for (int pl = 0; pl < (cplx_ ? 2 : 1); ++pl) {
    const double* T2 = T + pl * plane + n1;
    double* A = Ac + pl * ai_;
    double* B = Bc + pl * bi_;
    {  // Ac[P][y][d] = T2[P][(d, y)]
      const int64_t e[4] = {1, n1, o, v}, ds[4] = {0, o * kc, kc, 1}, ss[4] = {0, n1, 1, o};
      ops::copy4(A, ds, T2, ss, e, 1.0, 0.0, s_);
    }
    {  // Ac[P][y][v + l] = -conj(V^h[y][P][l])
      const int64_t e[4] = {1, n1, o, o}, ds[4] = {0, o * kc, kc, 1}, ss[4] = {0, o, n1 * o, 1};
      ops::copy4(A + v, ds, Vh + pl * vi_hhhp_, ss, e, pl == 0 ? -1.0 : 1.0, 0.0, s_);
    }
    {  // Bc[x][P][d] = V^p[x][P][d]
      const int64_t e[4] = {1, v, n1, v}, ds[4] = {0, n1 * kc, kc, 1}, ss[4] = {0, n1 * v, v, 1};
      ops::copy4(B, ds, Vp + pl * vi_ppph_, ss, e, 1.0, 0.0, s_);
    }
    {  // Bc[x][P][v + l] = T2[P][(x, l)]
      const int64_t e[4] = {1, v, n1, o}, ds[4] = {0, n1 * kc, kc, 1}, ss[4] = {0, o, n1, 1};
      ops::copy4(B + v, ds, T2, ss, e, 1.0, 0.0, s_);
    }
  }
}

void Triples::vslice(const char* name, const char* lab, double alpha, double beta, const Ten& C) {
  // V_pqsr = sum_G L_Gps R_Gqr with L = Gamma^{LO LI} (real half-grid rows) or
  // conj(Gamma^{LI LO})^T (complex), R = Gamma^{RO RI}: VertexCoulombIntegrals.cxx:55-197.
  const int64_t o = o_, v = v_, G = sys_.G;
  auto gam = [&](char X, char Y, char x, char y, bool conj) {
    Ten t;
    const bool px = X == 'p', py = Y == 'p';
    const RealSystem& r = sys_;
    double* base = px ? (py ? (cplx_ ? cs_->Gpp : r.Gpp) : (cplx_ ? cs_->Gph : r.Gph))
                      : (py ? (cplx_ ? cs_->Ghp : r.Ghp) : (cplx_ ? cs_->Ghh : r.Ghh));
    t.p = base;
    t.labels = std::string("#") + x + y;
    t.dims = {G, px ? v : o, py ? v : o};
    t.im = cplx_ ? G * t.dims[1] * t.dims[2] : 0;
    t.conj = conj;
    return t;
  };
  const char LO = name[0], RO = name[1], LI = name[2], RI = name[3];
  const Ten L = cplx_ ? gam(LI, LO, lab[2], lab[0], true) : gam(LO, LI, lab[0], lab[2], false);
  const Ten R = gam(RO, RI, lab[1], lab[3], false);
  ein(alpha, L, R, beta, C);
}

// ct::getCompleteTriples (CompleteTriples.cxx:11-118) on the device: every statement
// of :51-114 as one labelled contraction (ein), the integral slices from the vertex.
// Pair-layout amplitudes T_abij sit in memory as [a][i][b][j]; I_bcek is stored in
// the layout of Vppph_ ([b][c][k][e]) and I_mcjk in that of Vhhhp_ ([j][c][k][m]),
// so that the block contractions of V take them unchanged.
void Triples::complete_intermediates(const double* T) {
  const int64_t o = o_, v = v_, n1 = n1_;
  const int64_t plane = n1 + n1 * n1;
  const int pl = cplx_ ? 2 : 1;
  auto ext = [&](char c) { return c == 'p' ? v : o; };
  // A tensor named by the reference's labels `lab` of its type (e.g. "hhhp"), held in
  // memory in the order `perm` of the reference positions.
  struct Buf {
    double* p;
    std::string type, perm;
    int64_t size;
  };
  auto buf = [&](const char* type, const char* perm = nullptr) {
    Buf b;
    b.type = type;
    b.perm = perm ? perm : std::string("0123").substr(0, b.type.size());
    b.size = 1;
    for (char c : b.type) b.size *= ext(c);
    b.p = nullptr;
    return b;
  };
  auto R = [&](const Buf& b, const char* lab) {
    Ten t;
    t.p = b.p;
    for (char k : b.perm) {
      const int q = k - '0';
      t.labels += lab[q];
      t.dims.push_back(ext(b.type[q]));
    }
    t.im = cplx_ ? b.size : 0;
    return t;
  };
  Buf t1 = buf("ph"), t2 = buf("pphh", "0213");
  t1.p = cp(T);
  t2.p = cp(T) + n1;
  auto T1 = [&](const char* l) { Ten x = R(t1, l); x.im = cplx_ ? plane : 0; return x; };
  auto T2 = [&](const char* l) { Ten x = R(t2, l); x.im = cplx_ ? plane : 0; return x; };
  Buf Ip = buf("ppph", "0132"), Ih = buf("hphh", "2130");
  Ip.p = Ip_;
  Ih.p = Ih_;
  Buf Vhhhp = buf("hhhp", "0312");  // Vhhhp_: V_jklc as [j][c][k][l]
  Vhhhp.p = Vhhhp_;
  Buf Vhp = buf("hhpp"), Xk = buf("hhhp"), Xa = buf("phpp"), I = buf("hp"), P1 = buf("hphp"),
      P2 = buf("hpph"), Vhhph = buf("hhph"), Vhhhh = buf("hhhh"), Y = buf("ph");
  Y.type = "#ph";  // Y_Gck = sum_f Gamma^pp_Gcf t_fk
  Y.perm = "012";
  Y.size = sys_.G * v * o;
  for (Buf* b : {&Vhp, &Xk, &Xa, &I, &P1, &P2, &Vhhph, &Vhhhh, &Y}) b->p = take(pl * b->size);
  auto RY = [&](const char* lab) {
    Ten t;
    t.p = Y.p; t.labels = lab; t.dims = {sys_.G, v, o}; t.im = cplx_ ? Y.size : 0;
    return t;
  };
  vslice("hhpp", "ijab", 1.0, 0.0, R(Vhp, "ijab"));
  // :53-55  Xijka = Vhhhp + T_fk Vhhpp_ijfa
  vslice("hhhp", "ijka", 1.0, 0.0, R(Xk, "ijka"));
  ein(1.0, T1("fk"), R(Vhp, "ijfa"), 1.0, R(Xk, "ijka"));
  // :57-59  pXaibc = Vphpp - 1/2 T_al Vhhpp_libc
  vslice("phpp", "aibc", 1.0, 0.0, R(Xa, "aibc"));
  ein(-0.5, T1("al"), R(Vhp, "libc"), 1.0, R(Xa, "aibc"));
  // :61-63  Iia = 2 Vhhpp_ilaf T_fl - Vhhpp_ilfa T_fl
  ein(2.0, R(Vhp, "ilaf"), T1("fl"), 0.0, R(I, "ia"));
  ein(-1.0, R(Vhp, "ilfa"), T1("fl"), 1.0, R(I, "ia"));
  // :66-69  pXiajb = Vhphp - 1/2 Vhhhp_iljb T_al + T_fj pXaibc_aibf
  vslice("hphp", "iajb", 1.0, 0.0, R(P1, "iajb"));
  ein(-0.5, R(Vhhhp, "iljb"), T1("al"), 1.0, R(P1, "iajb"));
  ein(1.0, T1("fj"), R(Xa, "aibf"), 1.0, R(P1, "iajb"));
  // :71-74  pXiabj = Vhpph - 1/2 Vhhph_ilbj T_al + pXaibc_aifb T_fj
  vslice("hhph", "ilbj", 1.0, 0.0, R(Vhhph, "ilbj"));
  vslice("hpph", "iabj", 1.0, 0.0, R(P2, "iabj"));
  ein(-0.5, R(Vhhph, "ilbj"), T1("al"), 1.0, R(P2, "iabj"));
  ein(1.0, R(Xa, "aifb"), T1("fj"), 1.0, R(P2, "iabj"));
  // :76-78  Xaibc = pXaibc - 1/2 T_al Vhhpp_libc
  ein(-0.5, T1("al"), R(Vhp, "libc"), 1.0, R(Xa, "aibc"));
  // :90-101  dpIbcek
  copy_(Ip_, Vppph_, pl * v * n1 * v);
  {  // V_bcef T_fk = sum_G L_Gbe Y_Gck without forming V_pppp
    auto gpp = [&](const char* lab, bool conj) {
      Ten g;
      g.p = cplx_ ? cs_->Gpp : sys_.Gpp;
      g.labels = lab;
      g.dims = {sys_.G, v, v};
      g.im = cplx_ ? sys_.G * v * v : 0;
      g.conj = conj;
      return g;
    };
    ein(1.0, gpp("#cf", false), T1("fk"), 0.0, RY("#ck"));
    ein(1.0, cplx_ ? gpp("#eb", true) : gpp("#be", false), RY("#ck"), 1.0, R(Ip, "bcek"));
  }
  ein(-1.0, R(P1, "lbke"), T1("cl"), 1.0, R(Ip, "bcek"));
  ein(-1.0, T1("bl"), R(P2, "lcek"), 1.0, R(Ip, "bcek"));
  ein(-1.0, T2("bclk"), R(I, "le"), 1.0, R(Ip, "bcek"));
  ein(2.0, R(Xa, "blef"), T2("cfkl"), 1.0, R(Ip, "bcek"));
  ein(-1.0, R(Xa, "blef"), T2("fckl"), 1.0, R(Ip, "bcek"));
  ein(-1.0, R(Xa, "blfe"), T2("fclk"), 1.0, R(Ip, "bcek"));
  ein(-1.0, T2("fbkl"), R(Xa, "clfe"), 1.0, R(Ip, "bcek"));
  ein(1.0, T2("cbln"), R(Xk, "lnke"), 1.0, R(Ip, "bcek"));
  // :80-83  dpXiajb = Vhphp - Vhhhp_iljb T_al + 1/2 T_fj Xaibc_aibf
  vslice("hphp", "iajb", 1.0, 0.0, R(P1, "iajb"));
  ein(-1.0, R(Vhhhp, "iljb"), T1("al"), 1.0, R(P1, "iajb"));
  ein(0.5, T1("fj"), R(Xa, "aibf"), 1.0, R(P1, "iajb"));
  // :85-88  dpXiabj = Vhpph - Vhhph_ilbj T_al + 1/2 Xaibc_aifb T_fj
  vslice("hpph", "iabj", 1.0, 0.0, R(P2, "iabj"));
  ein(-1.0, R(Vhhph, "ilbj"), T1("al"), 1.0, R(P2, "iabj"));
  ein(0.5, R(Xa, "aifb"), T1("fj"), 1.0, R(P2, "iabj"));
  // :103-113  dpImcjk
  vslice("hhhh", "mljk", 1.0, 0.0, R(Vhhhh, "mljk"));
  vslice("hphh", "mcjk", 1.0, 0.0, R(Ih, "mcjk"));
  ein(-1.0, R(Vhhhh, "mljk"), T1("cl"), 1.0, R(Ih, "mcjk"));
  ein(1.0, R(P1, "mcjf"), T1("fk"), 1.0, R(Ih, "mcjk"));
  ein(1.0, T1("fj"), R(P2, "mcfk"), 1.0, R(Ih, "mcjk"));
  ein(2.0, R(Xk, "mljf"), T2("cfkl"), 1.0, R(Ih, "mcjk"));
  ein(-1.0, R(Xk, "mljf"), T2("fckl"), 1.0, R(Ih, "mcjk"));
  ein(-1.0, R(Xk, "lmjf"), T2("fclk"), 1.0, R(Ih, "mcjk"));
  ein(-1.0, T2("cflj"), R(Xk, "lmkf"), 1.0, R(Ih, "mcjk"));
  ein(1.0, T2("dfkj"), R(Xa, "cmdf"), 1.0, R(Ih, "mcjk"));
}

double Triples::cr_amplitude_terms(const double* T) {
  const int64_t o = o_, v = v_, n1 = n1_, n2 = n1 * n1;
  const int64_t plane = n1 + n2;
  const int pl = cplx_ ? 2 : 1;
  double* X = take(pl * n2);   // T2 + t1 t1^T
  double* Tx = take(pl * n2);  // T_baij in the pair layout
  double* r = take(8);
  const int64_t d[4] = {v, o, v, o};
  const int perm[4] = {2, 1, 0, 3};
  if (cplx_) {
    ops::zrank1(X, X + n2, T + n1, T + plane + n1, T, T + plane, 1.0, n1, s_);
  } else {
    ops::rank1(X, 1.0, T + n1, 1.0, T, n1, s_);
  }
  for (int p = 0; p < pl; ++p) {
    ops::permute4(Tx + p * n2, T + p * plane + n1, d, perm, 1.0, 0.0, s_);
    const double* ys[2] = {T + p * plane + n1, Tx + p * n2};
    ops::dots(X + p * n2, ys, 2, n2, r + 2 * p, ws_, s_);
    const double* t1s[1] = {T + p * plane};
    ops::dots(T + p * plane, t1s, 1, n1, r + 4 + p, ws_, s_);
  }
  double h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  ops::d2h(h, r, 8, s_);
  ops::sync(s_);
  // Re sum (2T - T^x) X = sum over planes with the sign of Re(a b) = ReRe - ImIm
  const double wc = (2.0 * h[0] - h[1]) - (cplx_ ? 2.0 * h[2] - h[3] : 0.0);
  const double tt = h[4] - (cplx_ ? h[5] : 0.0);
  return 1.0 + 2.0 * tt + wc;
}

TriplesOutcome Triples::run(const double* T) {
  const int64_t o = o_, v = v_, n1 = n1_, nb = nb_;
  const int64_t nbk = (v + nb - 1) / nb;
  const int64_t plane = n1 + n1 * n1;
  const double* t1 = T;
  const double* t1i = cplx_ ? T + plane : nullptr;
  const double* Vi = cplx_ ? Vpphh_ + vi_pphh_ : nullptr;
  double* Si = cplx_ ? S_ + si_ : nullptr;
  TriplesOutcome out;
  out.block = nb;
  out.block_triples = ntri_;
  out.setup_seconds = setup_seconds_;
  out.flops = 2.0 * double(o) * o * o * double(v) * v * v * double(o + v);
  void* e0 = ops::event_create();
  void* e1 = ops::event_create();
  ops::event_record(e0, s_);
  if (complete_) complete_intermediates(T);
  concat_operands(T, Vppph_, Vhhhp_, Ac_, Bc_);
  if (complete_) concat_operands(T, Ip_, Ih_, AcM_, BcM_);
  // split form (the contractions' K = v + o long enough for it): both operands sliced once here
  const bool packed = precision_ == 3 && kc_ >= 64;
  if (packed) {
    pack_operands(0, Ac_, Bc_);
    if (complete_) pack_operands(1, AcM_, BcM_);
  }
  ops::event_record(e1, s_);
  out.setup_seconds += ops::event_ms(e0, e1) * 1e-3;
  const int64_t Lm = nb * o;
  double* Mi = complete_ && cplx_ ? Mb_ + si_ : nullptr;
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
        if (complete_) zero_(Mb_, (cplx_ ? 2 : 1) * Lm * Lm * Lm);
        if (profile_) ops::event_record(pev[5 * t + 1], s_);
        if (packed) {
          connected_packed(b, X, n, 0, S_);
          if (complete_) connected_packed(b, X, n, 1, Mb_);
        } else {
          connected(b, X, n, Ac_, Bc_, S_);
          if (complete_) connected(b, X, n, AcM_, BcM_, Mb_);
        }
        if (profile_) ops::event_record(pev[5 * t + 2], s_);
        // (the hole terms ride in the contractions above: the hole phase stays empty)
        if (profile_) ops::event_record(pev[5 * t + 3], s_);
        double coef[6];
        coefficients(A, B, C, coef);
        ops::triples_energy(S_, Si, t1, t1i, Vpphh_, Vi, sys_.eh, sys_.ep, b, coef, ws_,
                            slots_ + 2 * t, s_, complete_ ? Mb_ : nullptr, Mi);
        if (complete_)
          ops::triples_cr_sums(S_, Si, t1, t1i, T + n1, cplx_ ? T + plane + n1 : nullptr, sys_.eh,
                               sys_.ep, b, coef, ws_, cr_slots_ + 2 * t, s_);
        if (profile_) ops::event_record(pev[5 * t + 4], s_);
        out.executed_flops += (complete_ ? 2.0 : 1.0) * (cplx_ ? 4.0 : 1.0) * 12.0 *
                              double(n[0] * n[1] * n[2]) * o * o * o * double(v + o);
      }
  ops::sum_partials_to(slots_ + 2 * ntri_, slots_, static_cast<int>(ntri_), 2, s_);
  if (complete_)
    ops::sum_partials_to(cr_slots_ + 2 * ntri_, cr_slots_, static_cast<int>(ntri_), 2, s_);
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
  // Re conj(W) Z = ReW ReZ + ImW ImZ;  Re conj(W) conj(Z) = ReW ReZ - ImW ImZ;
  // cT: Re M conj(Z) = ReM ReZ + ImM ImZ
  out.energy = reference_form_ && !complete_ ? sums[0] - sums[1] : sums[0] + sums[1];
  if (complete_) {
    double cr[2];
    ops::d2h(cr, cr_slots_ + 2 * ntri_, 2, s_);
    ops::sync(s_);
    // Re y conj(Z) / D = Re y Re Z / D + Im y Im Z / D
    out.cr_denominator = cr_amplitude_terms(T) + cr[0] + cr[1];
  }
  return out;
}

}  // namespace cc4s_b200
