#include "schedule.h"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <vector>

namespace cc4s_b200 {

Schedule::~Schedule() { release_all(); }

void Schedule::release_all() {
  for (void* e : ev_) ops::event_destroy(e);
  ev_.clear();
  if (split_mem_) ops::release(split_mem_);
  split_mem_ = nullptr;
  split_ = SplitScratch();
  split_extra_ = nullptr;
  split_extra_bytes_ = 0;
  for (double* p : owned_) ops::release(p);
  owned_.clear();
  owned_n_.clear();
  for (double* p : bar_bufs_) ops::release(p);
  bar_bufs_.clear();
}

double* Schedule::take(size_t elems) {
  double* p = ops::alloc(elems);
  owned_.push_back(p);
  owned_n_.push_back(elems);
  bytes_ += elems * sizeof(double);
  return p;
}

void Schedule::gemm_(const Contraction& c) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::GEMM;
    op.c = c;
    tape_.push_back(op);
  }
  const double f = 2.0 * double(c.M) * double(c.N) * double(c.K) * double(c.batch);
  if (count_flops_) flops_ += f;
  if (profile_ && count_flops_) {
    const size_t k = ev_flops_.size();
    while (ev_.size() < 2 * (k + 1)) ev_.push_back(ops::event_create());
    ev_flops_.push_back(f);
    ev_split_.push_back(0);
    ev_shape_.push_back({c.M, c.N, c.K, c.batch});
    ops::event_record(ev_[2 * k], s_);
    gemm(c, s_, scratch_);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  gemm(c, s_, scratch_);
}

namespace {
constexpr size_t kSplitDataOffset = 128;  // doubles: 1 KiB
}  // namespace

bool Schedule::split_ok(const Contraction& c) const {
  return precision_ != 0 && c.batch == 1 && c.K >= 64 && c.M >= 64 && c.N >= 64;
}

void Schedule::split_reserve(size_t regular, size_t extra) {
  regular = (regular + 1023) / 1024 * 1024;
  extra = (extra + 1023) / 1024 * 1024;
  if (regular <= split_.bytes && extra <= split_extra_bytes_) return;
  regular = std::max(regular, split_.bytes);
  extra = std::max(extra, split_extra_bytes_);
  ops::sync(s_);
  if (split_mem_) ops::release(split_mem_);
  split_mem_ = nullptr;
  split_extra_ = nullptr;
  split_extra_bytes_ = 0;
  // The error word sits in the first double; the packed slices start 1 KiB in,
  // so every TMA row request of the contraction kernel begins on a sector and
  // line boundary (a 16-byte offset made each 64-byte row touch three sectors).
  const size_t doubles = (regular + extra) / 8 + kSplitDataOffset;
  split_mem_ = ops::alloc(doubles);
  split_.p = split_mem_ + kSplitDataOffset;
  split_.bytes = regular;
  split_.error = reinterpret_cast<int*>(split_mem_);
  if (extra) {
    split_extra_ = static_cast<unsigned char*>(split_.p) + regular;
    split_extra_bytes_ = extra;
  }
  ops::zero(split_mem_, 2, s_);
}

void Schedule::split_exec(const Contraction& c) {
  const size_t need = gemm_split_scratch_bytes(c);
  // growing keeps the size of the extra region (not its contents: no pre-packed
  // operand is live across a contraction that needs more than the reserved part)
  if (need > split_.bytes) split_reserve(need, split_extra_bytes_);
  gemm_split(c, s_, split_);
}

void Schedule::tc_packed_b_(const Contraction& c, const SplitPackedB& b) {
  if (taping_) throw Error(ERR_STATE, "pre-packed split operands are not recorded");
  const double f = 2.0 * double(c.M) * double(c.N) * double(c.K);
  if (count_flops_) flops_ += f;
  if (profile_ && count_flops_) {
    const size_t k = ev_flops_.size();
    while (ev_.size() < 2 * (k + 1)) ev_.push_back(ops::event_create());
    ev_flops_.push_back(f);
    ev_split_.push_back(1);
    ev_shape_.push_back({c.M, c.N, c.K, c.batch});
    ops::event_record(ev_[2 * k], s_);
    gemm_split_packed_b(c, b, s_, split_);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  gemm_split_packed_b(c, b, s_, split_);
}

void Schedule::tc_prepacked_(const Contraction& c, const SplitOperand& A, const SplitRuns& ar,
                             const SplitOperand& B, const SplitRuns& br) {
  if (taping_) throw Error(ERR_STATE, "pre-packed split operands are not recorded");
  if (!split_.error) split_reserve(size_t(1) << 16, split_extra_bytes_);  // the error word
  const double f = 2.0 * double(c.M) * double(c.N) * double(c.K);
  if (count_flops_) flops_ += f;
  if (profile_ && count_flops_) {
    const size_t k = ev_flops_.size();
    while (ev_.size() < 2 * (k + 1)) ev_.push_back(ops::event_create());
    ev_flops_.push_back(f);
    ev_split_.push_back(1);
    ev_shape_.push_back({c.M, c.N, c.K, c.batch});
    ops::event_record(ev_[2 * k], s_);
    gemm_split_prepacked(c, A, ar, B, br, s_, split_);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  gemm_split_prepacked(c, A, ar, B, br, s_, split_);
}

// A contraction of the reverse sweep (or a recomputed forward one): split
// precision under the same rule as tc_, else FP64; neither recorded nor counted.
void Schedule::exec_(const Contraction& c) {
  if (split_ok(c)) split_exec(c);
  else gemm(c, s_, scratch_);
}

void Schedule::tc_(const Contraction& c) {
  if (!split_ok(c)) {
    gemm_(c);
    return;
  }
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::GEMM;
    op.c = c;
    tape_.push_back(op);
  }
  const double f = 2.0 * double(c.M) * double(c.N) * double(c.K);
  if (count_flops_) flops_ += f;
  if (profile_ && count_flops_) {
    const size_t k = ev_flops_.size();
    while (ev_.size() < 2 * (k + 1)) ev_.push_back(ops::event_create());
    ev_flops_.push_back(f);
    ev_split_.push_back(1);
    ev_shape_.push_back({c.M, c.N, c.K, c.batch});
    ops::event_record(ev_[2 * k], s_);
    split_exec(c);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  split_exec(c);
}

void Schedule::zgemm(Contraction c, int64_t a_im, int64_t b_im, int64_t c_im, bool conjA,
                     bool conjB, bool big) {
  auto run = [&](const Contraction& x) { if (big) tc_(x); else gemm_(x); };
  const double sA = conjA ? -1.0 : 1.0, sB = conjB ? -1.0 : 1.0;
  const double al = c.alpha, be = c.beta;
  double* Ar = c.A.p;
  double* Br = c.B.p;
  double* Cr = c.C.p;
  double* C2r = c.C2.p;
  // real plane: Re(A) Re(B) - sA sB Im(A) Im(B)
  run(c);
  if (a_im && b_im) {
    Contraction r = c;
    r.A.p = Ar + a_im; r.B.p = Br + b_im; r.alpha = -al * sA * sB; r.beta = 1.0;
    run(r);
  }
  if (!c_im) return;  // real result (both operands real)
  // imaginary plane: sB Re(A) Im(B) + sA Im(A) Re(B)
  Contraction i = c;
  i.C.p = Cr + c_im;
  if (C2r) i.C2.p = C2r + c_im;
  bool wrote = false;
  if (b_im) {
    i.B.p = Br + b_im; i.alpha = al * sB; i.beta = be;
    run(i);
    wrote = true;
  }
  if (a_im) {
    i.A.p = Ar + a_im; i.B.p = Br; i.alpha = al * sA; i.beta = wrote ? 1.0 : be;
    run(i);
    wrote = true;
  }
  if (!wrote) throw Error(ERR_STATE, "zgemm: complex result from real operands");
}

namespace {
// One index of an ein() operand: label id, extent, element stride.
struct EinAx {
  int id;
  int64_t n, s;
};
struct EinOps {
  double* p[3];
  std::vector<EinAx> ax[3];  // memory order, outer first
};
int ein_find(const std::vector<EinAx>& v, int id) {
  for (size_t k = 0; k < v.size(); ++k)
    if (v[k].id == id) return static_cast<int>(k);
  return -1;
}
// Fuses index pairs (x, y) that are adjacent (y right after x, stride_x = n_y stride_y)
// in every operand holding either of them.
void ein_fuse(EinOps& e, int& next_id) {
  for (bool again = true; again;) {
    again = false;
    for (int t = 0; t < 3 && !again; ++t)
      for (size_t k = 0; k + 1 < e.ax[t].size() && !again; ++k) {
        const int x = e.ax[t][k].id, y = e.ax[t][k + 1].id;
        bool ok = true;
        for (int u = 0; u < 3 && ok; ++u) {
          const int px = ein_find(e.ax[u], x), py = ein_find(e.ax[u], y);
          if ((px < 0) != (py < 0)) ok = false;
          else if (px >= 0)
            ok = py == px + 1 && e.ax[u][px].s == e.ax[u][py].n * e.ax[u][py].s;
        }
        if (!ok) continue;
        const int id = next_id++;
        for (int u = 0; u < 3; ++u) {
          const int px = ein_find(e.ax[u], x);
          if (px < 0) continue;
          EinAx& a = e.ax[u][px];
          const EinAx b = e.ax[u][px + 1];
          a = EinAx{id, a.n * b.n, b.s};
          e.ax[u].erase(e.ax[u].begin() + px + 1);
        }
        again = true;
      }
  }
}
// Groups the indices, loops on the host over one index of any group wider than
// two levels (the smallest such index; a summed one accumulates), and hands one
// contraction per launch to `launch`.
void ein_run(EinOps e, int& next_id, double alpha, double beta,
             const std::function<void(const Contraction&)>& launch) {
  ein_fuse(e, next_id);
  std::vector<int> g[4];  // M (A, C), N (B, C), K (A, B), batch (all three)
  auto has = [&](int t, int id) { return ein_find(e.ax[t], id) >= 0; };
  for (int t = 0; t < 3; ++t)
    for (const auto& a : e.ax[t]) {
      const bool inA = has(0, a.id), inB = has(1, a.id), inC = has(2, a.id);
      const int grp = inA && inB && inC ? 3 : inA && inC ? 0 : inB && inC ? 1 : inA && inB ? 2 : -1;
      if (grp < 0) throw Error(ERR_STATE, "ein: a label appears in one operand only");
      if (std::find(g[grp].begin(), g[grp].end(), a.id) == g[grp].end()) g[grp].push_back(a.id);
    }
  for (int k = 0; k < 4; ++k) {
    if (g[k].size() <= 2) continue;
    int best = -1;
    int64_t bn = 0;
    for (int id : g[k]) {
      for (int t = 0; t < 3; ++t) {
        const int q = ein_find(e.ax[t], id);
        if (q >= 0 && (best < 0 || e.ax[t][q].n < bn)) { best = id; bn = e.ax[t][q].n; }
      }
    }
    for (int64_t x = 0; x < bn; ++x) {
      EinOps f = e;
      for (int t = 0; t < 3; ++t) {
        const int q = ein_find(f.ax[t], best);
        if (q < 0) continue;
        f.p[t] += x * f.ax[t][q].s;
        f.ax[t].erase(f.ax[t].begin() + q);
      }
      ein_run(f, next_id, alpha, k == 2 && x > 0 ? 1.0 : beta, launch);
    }
    return;
  }
  // extent, inner extent (0: one level) and the outer / inner strides in operand t
  auto level = [&](const std::vector<int>& ids, int t, int64_t& so, int64_t& si) {
    so = si = 0;
    if (ids.empty()) return;
    const EinAx& in = e.ax[t][ein_find(e.ax[t], ids.back())];
    si = in.s;
    if (ids.size() == 2) so = e.ax[t][ein_find(e.ax[t], ids.front())].s;
  };
  auto extent = [&](const std::vector<int>& ids, int64_t& n, int64_t& ni) {
    n = 1; ni = 0;
    for (int id : ids)
      for (int t = 0; t < 3; ++t) {
        const int q = ein_find(e.ax[t], id);
        if (q >= 0) { n *= e.ax[t][q].n; if (ids.size() == 2 && id == ids.back()) ni = e.ax[t][q].n; break; }
      }
  };
  // inner level of M and N: the index with the smaller stride in C
  for (int k : {0, 1})
    if (g[k].size() == 2 && e.ax[2][ein_find(e.ax[2], g[k][0])].s <
                                e.ax[2][ein_find(e.ax[2], g[k][1])].s)
      std::swap(g[k][0], g[k][1]);
  Contraction c;
  extent(g[0], c.M, c.Mi);
  extent(g[1], c.N, c.Ni);
  extent(g[2], c.K, c.Ki);
  extent(g[3], c.batch, c.Bi);
  c.A.p = e.p[0]; c.B.p = e.p[1]; c.C.p = e.p[2];
  level(g[0], 0, c.A.s_ro, c.A.s_ri);
  level(g[2], 0, c.A.s_co, c.A.s_ci);
  level(g[2], 1, c.B.s_ro, c.B.s_ri);
  level(g[1], 1, c.B.s_co, c.B.s_ci);
  level(g[0], 2, c.C.s_ro, c.C.s_ri);
  level(g[1], 2, c.C.s_co, c.C.s_ci);
  for (int t = 0; t < 3; ++t) {
    View& v = t == 0 ? c.A : t == 1 ? c.B : c.C;
    level(g[3], t, v.s_bo, v.s_bi);
  }
  c.alpha = alpha;
  c.beta = beta;
  launch(c);
}
}  // namespace

void Schedule::ein(double alpha, const Ten& A, const Ten& B, double beta, const Ten& C, bool big) {
  EinOps e;
  const Ten* T[3] = {&A, &B, &C};
  std::map<char, int> ids;
  std::map<int, int64_t> ext;
  for (int t = 0; t < 3; ++t) {
    const Ten& x = *T[t];
    if (x.labels.size() != x.dims.size())
      throw Error(ERR_STATE, "ein: labels and extents differ in number");
    e.p[t] = x.p;
    int64_t stride = 1;
    std::vector<EinAx> v(x.labels.size());
    for (size_t k = x.labels.size(); k-- > 0;) {
      const char c = x.labels[k];
      auto it = ids.find(c);
      const int id = it == ids.end() ? (ids[c] = static_cast<int>(ids.size())) : it->second;
      auto et = ext.find(id);
      if (et != ext.end() && et->second != x.dims[k])
        throw Error(ERR_STATE, std::string("ein: extents of label ") + c + " differ");
      ext[id] = x.dims[k];
      v[k] = EinAx{id, x.dims[k], stride};
      stride *= x.dims[k];
    }
    e.ax[t] = v;
  }
  for (int t = 0; t < 3; ++t)
    for (size_t k = 0; k < e.ax[t].size(); ++k)
      if (ein_find(e.ax[t], e.ax[t][k].id) != static_cast<int>(k))
        throw Error(ERR_STATE, "ein: repeated label in one operand");
  if (C.conj || (C.im != 0) != (A.im != 0 || B.im != 0))
    throw Error(ERR_STATE, "ein: output must be complex exactly when an operand is");
  int next_id = static_cast<int>(ids.size());
  ein_run(e, next_id, alpha, beta, [&](const Contraction& c) {
    zgemm(c, A.im, B.im, C.im, A.conj, B.conj, big);
  });
}

// W[G][(a,i)] = sum_{b,j} Gamma^hp_Gjb M[(b,j),(a,i)] with M = 2X - X^x, X = T2 + T1 T1
// (adjW_; M stays in adjX_ + planes * D2 for the gradient).
void Schedule::structure_factor_w(const double* T) {
  const int64_t o = so_, v = sv_, G = sG_, n1 = o * v, D2 = n1 * n1;
  if (!T || !sGph_) throw Error(ERR_STATE, "structure factor: no amplitudes or vertex");
  const int64_t planes = scplx_ ? 2 : 1, pl = n1 + D2;
  if (!adjX_) {
    adjX_ = take(2 * planes * D2);
    adjW_ = take(planes * G * n1);
  }
  double* X = adjX_;             // X = T2 + T1 T1, then M = 2X - X^x
  double* M = adjX_ + planes * D2;
  const double* t = T;
  const double* Td = T + n1;
  if (scplx_) ops::zrank1(X, X + D2, Td, Td + pl, t, t + pl, 1.0, n1, s_);
  else ops::rank1(X, 1.0, Td, 1.0, t, n1, s_);
  const int64_t d4[4] = {v, o, v, o};
  const int p_ex[4] = {0, 3, 2, 1};
  for (int64_t p = 0; p < planes; ++p) {
    ops::permute4(M + p * D2, X + p * D2, d4, p_ex, -1.0, 0.0, s_);
    ops::axpby(M + p * D2, 2.0, X + p * D2, 1.0, M + p * D2, 0.0, D2, s_);
  }
  const int64_t gi = scplx_ ? G * n1 : 0, mi = scplx_ ? D2 : 0;
  Contraction c; c.M = G; c.N = n1; c.K = n1; c.Ki = o;
  c.A = vw(sGhp_, 0, n1, 1, v); c.B = vw(M, o * n1, n1, 0, 1); c.C = rm(adjW_, n1);
  zgemm(c, gi, mi, gi, false, false, true);
}

void Schedule::structure_factor(const double* T, double* S_dev, double* dGph_dev) {
  structure_factor_w(T);
  const int64_t o = so_, v = sv_, G = sG_, n1 = o * v, D2 = n1 * n1;
  const int64_t planes = scplx_ ? 2 : 1;
  const int64_t gi = scplx_ ? G * n1 : 0;
  {  // S[G] = Re sum_r conj(Gamma^ph_G,r) W_G,r   (batched dot products)
    Contraction c; c.M = 1; c.N = 1; c.K = n1; c.batch = G;
    c.A = vw(sGph_, 0, 0, 0, 1, 0, n1); c.B = vw(adjW_, 0, 1, 0, 0, 0, n1);
    c.C = vw(S_dev, 0, 0, 0, 0, 0, 1);
    zgemm(c, gi, gi, 0, scplx_, false);
  }
  if (dGph_dev) {
    if (scplx_) throw Error(ERR_UNSUPPORTED, "dE/dGamma is provided on the real path only");
    double* M = adjX_ + planes * D2;
    Contraction c; c.M = G; c.N = n1; c.K = n1;  // dE/dGph = 2 Gph M
    c.A = rm(sGph_, n1); c.B = rm(M, n1); c.C = rm(dGph_dev, n1); c.alpha = 2.0;
    tc_(c);
  }
  (void)v;
}

void Schedule::structure_factor_pw(const double* T, const double* Uw, int64_t NGG, int64_t NF,
                                   double* S_dev) {
  structure_factor_w(T);
  const int64_t G = sG_, n1 = so_ * sv_;
  const int parts = scplx_ ? 1 : static_cast<int>(G / NF);
  if (G != NF * parts || parts < 1 || parts > 2)
    throw Error(ERR_BAD_SHAPE, "structure factor: vertex rows do not match the singular vectors");
  std::vector<double*> tmp;
  auto tk = [&](int64_t n) { double* p = ops::alloc(n); tmp.push_back(p); return p; };
  try {
    double* Qs = tk(scplx_ ? 2 * G * G : G * G);
    double* Q = tk(2 * NF * NF);
    double* Y = tk(2 * NGG * NF);
    {  // Qs[F][F'] = sum_r conj(Gamma^ph_F,r) W_F',r  (vertex rows of this schedule)
      Contraction c; c.M = G; c.N = G; c.K = n1;
      c.A = rm(sGph_, n1); c.B = vw(adjW_, 0, 1, 0, n1); c.C = rm(Qs, G);
      zgemm(c, scplx_ ? G * n1 : 0, scplx_ ? G * n1 : 0, scplx_ ? G * G : 0, scplx_, false);
    }
    if (scplx_) {
      ops::d2d(Q, Qs, 2 * NF * NF, s_);
    } else {
      ops::fsc_stacked_to_complex(Q, Q + NF * NF, Qs, NF, parts, s_);
    }
    {  // Y[G][F'] = sum_F conj(Uw_GF) Q_FF'
      Contraction c; c.M = NGG; c.N = NF; c.K = NF;
      c.A = rm(cp(Uw), NF); c.B = rm(Q, NF); c.C = rm(Y, NF);
      zgemm(c, NGG * NF, NF * NF, NGG * NF, true, false);
    }
    {  // S[G] = Re sum_F' Y[G][F'] Uw[G][F']
      Contraction c; c.M = 1; c.N = 1; c.K = NF; c.batch = NGG;
      c.A = vw(Y, 0, 0, 0, 1, 0, NF); c.B = vw(cp(Uw), 0, 1, 0, 0, 0, NF);
      c.C = vw(S_dev, 0, 0, 0, 0, 0, 1);
      zgemm(c, NGG * NF, NGG * NF, 0, false, false);
    }
    ops::sync(s_);
  } catch (...) {
    for (double* p : tmp) ops::release(p);
    throw;
  }
  for (double* p : tmp) ops::release(p);
}

int Schedule::device_error() {
  if (!split_.error) return 0;
  double v = 0.0;
  ops::d2h(&v, split_mem_, 1, s_);
  ops::sync(s_);
  int e;
  std::memcpy(&e, &v, sizeof(int));
  return e;
}

void Schedule::profile_finish() {
  if (!profile_) return;
  Profile p;
  for (size_t k = 0; k < ev_flops_.size(); ++k) {
    const double sec = 1e-3 * ops::event_ms(ev_[2 * k], ev_[2 * k + 1]);
    p.gemm_seconds += sec;
    p.gemm_flops += ev_flops_[k];
    if (ev_flops_[k] > p.top_flops) { p.top_flops = ev_flops_[k]; p.top_seconds = sec; }
    if (ev_split_[k]) {
      p.split_seconds += sec;
      p.split_flops += ev_flops_[k];
      ++p.split_launches;
    }
  }
  p.launches = static_cast<int>(ev_flops_.size());
  // CC4S_PROFILE_LOG: append a per-shape summary of this residual's contractions
  if (const char* path = std::getenv("CC4S_PROFILE_LOG")) {
    std::map<std::array<int64_t, 5>, std::array<double, 3>> agg;  // count, seconds, flops
    for (size_t k = 0; k < ev_flops_.size(); ++k) {
      const auto& sh = ev_shape_[k];
      auto& a = agg[{ev_split_[k] ? 1 : 0, sh[0], sh[1], sh[2], sh[3]}];
      a[0] += 1;
      a[1] += 1e-3 * ops::event_ms(ev_[2 * k], ev_[2 * k + 1]);
      a[2] += ev_flops_[k];
    }
    std::vector<std::pair<double, std::array<int64_t, 5>>> order;
    for (const auto& kv : agg) order.push_back({kv.second[1], kv.first});
    std::sort(order.rbegin(), order.rend());
    if (FILE* f = std::fopen(path, "a")) {
      std::fprintf(f, "# residual: %d launches, %.4f s, %.4g flops\n", p.launches, p.gemm_seconds,
                   p.gemm_flops);
      std::fprintf(f, "# kind M N K batch count seconds TFLOP/s(fp64-equivalent)\n");
      for (const auto& e : order) {
        const auto& a = agg[e.second];
        std::fprintf(f, "%s %lld %lld %lld %lld %d %.5f %.2f\n", e.second[0] ? "split" : "dmma",
                     (long long)e.second[1], (long long)e.second[2], (long long)e.second[3],
                     (long long)e.second[4], (int)a[0], a[1], a[2] / a[1] / 1e12);
      }
      std::fclose(f);
    }
  }
  ev_split_.clear();
  ev_flops_.clear();
  ev_shape_.clear();
  prof_ = p;
}


// ---------------------------------------------------------------------------
// Reverse mode.

void Schedule::perm_(double* dst, const double* src, const int64_t d[4], const int p[4],
                     double alpha, double beta) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::PERM;
    op.dst = dst; op.x = src; op.a = alpha; op.b = beta;
    for (int k = 0; k < 4; ++k) { op.d[k] = d[k]; op.perm[k] = p[k]; }
    tape_.push_back(op);
  }
  ops::permute4(dst, src, d, p, alpha, beta, s_);
}

void Schedule::axpby_(double* out, double a, const double* x, double b, const double* y,
                      double c, int64_t n) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::AXPBY;
    op.dst = out; op.x = x; op.y = y; op.a = a; op.b = b; op.cc = c; op.n = n;
    tape_.push_back(op);
  }
  ops::axpby(out, a, x, b, y, c, n, s_);
}

void Schedule::rank1_(double* out, double a, const double* A, double b, const double* t,
                      int64_t n) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::RANK1;
    op.dst = out; op.x = A; op.y = t; op.a = a; op.b = b; op.n = n;
    tape_.push_back(op);
  }
  ops::rank1(out, a, A, b, t, n, s_);
}

void Schedule::sym_(double* R, int64_t n) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::SYMM;
    op.dst = R; op.n = n;
    tape_.push_back(op);
  }
  ops::symmetrize(R, n, s_);
}

void Schedule::copy_(double* dst, const double* src, int64_t n) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::COPY;
    op.dst = dst; op.x = src; op.n = n;
    tape_.push_back(op);
  }
  ops::d2d(dst, src, n, s_);
}

void Schedule::zero_(double* p, int64_t n) {
  if (taping_) {
    TapeOp op;
    op.kind = TapeOp::ZERO;
    op.dst = p; op.n = n;
    tape_.push_back(op);
  }
  ops::zero(p, n, s_);
}

double* Schedule::bar_of(const double* p) const {
  if (!p) return nullptr;
  for (const Region& r : regions_)
    if (p >= r.p && p < r.p + r.n) return r.bar ? r.bar + (p - r.p) : nullptr;
  return nullptr;
}

View Schedule::barv(const View& v) const {
  View w = v;
  w.p = bar_of(v.p);
  return w;
}

namespace {
View transposed(const View& v) {
  View t = v;
  std::swap(t.s_ro, t.s_co);
  std::swap(t.s_ri, t.s_ci);
  return t;
}
}  // namespace

// Adjoint of C (and C2) = alpha A B + beta C:  Abar += alpha Cbar B^T,
// Bbar += alpha A^T Cbar.  An adjoint output that every batch entry shares
// (batch strides zero) is summed over the batch by folding the batch index into
// the contraction index, or launch by launch where that is not expressible.
void Schedule::reverse_gemm(const Contraction& c) {
  if (c.M <= 0 || c.N <= 0 || c.K <= 0 || c.batch <= 0) return;
  if (c.beta != 0.0 && c.beta != 1.0)
    throw Error(ERR_UNSUPPORTED, "reverse mode: contraction with beta other than 0 or 1");
  auto run = [&](Contraction d) {
    const bool shared = d.batch > 1 && d.C.s_bo == 0 && d.C.s_bi == 0;
    if (!shared) { exec_(d); return; }
    if (d.Ki == 0 && d.Bi == 0 && d.A.s_bo == 0 && d.B.s_bo == 0) {
      // sum over the batch as part of the contraction: k' = (b, k)
      Contraction e = d;
      e.K = d.K * d.batch; e.Ki = d.K; e.batch = 1;
      e.A.s_co = d.A.s_bi; e.B.s_ro = d.B.s_bi;
      e.A.s_bi = e.B.s_bi = e.C.s_bi = 0;
      exec_(e);
      return;
    }
    const int64_t Bi = d.Bi > 0 ? d.Bi : d.batch;
    for (int64_t b = 0; b < d.batch; ++b) {
      Contraction e = d;
      e.batch = 1; e.Bi = 0;
      const int64_t bo = b / Bi, bi = b % Bi;
      e.A.p += bo * d.A.s_bo + bi * d.A.s_bi;
      e.B.p += bo * d.B.s_bo + bi * d.B.s_bi;
      e.A.s_bo = e.A.s_bi = e.B.s_bo = e.B.s_bi = e.C.s_bo = e.C.s_bi = 0;
      gemm(e, s_, scratch_);
    }
  };
  const bool hasA = bar_of(c.A.p) != nullptr, hasB = bar_of(c.B.p) != nullptr;
  const View outs[2] = {c.C, c.C2};
  for (int w = 0; w < 2; ++w) {
    const View& O = outs[w];
    if (!O.p || !bar_of(O.p)) continue;
    if (hasA) {
      Contraction d;
      d.M = c.M; d.N = c.K; d.K = c.N; d.batch = c.batch;
      d.Mi = c.Mi; d.Ni = c.Ki; d.Ki = c.Ni; d.Bi = c.Bi;
      d.A = barv(O); d.B = transposed(c.B); d.C = barv(c.A);
      d.alpha = c.alpha; d.beta = 1.0;
      run(d);
    }
    if (hasB) {
      Contraction d;
      d.M = c.K; d.N = c.N; d.K = c.M; d.batch = c.batch;
      d.Mi = c.Ki; d.Ni = c.Ni; d.Ki = c.Mi; d.Bi = c.Bi;
      d.A = transposed(c.A); d.B = barv(O); d.C = barv(c.B);
      d.alpha = c.alpha; d.beta = 1.0;
      run(d);
    }
  }
}

void Schedule::reverse(const std::vector<TapeOp>& tape) {
  for (size_t k = tape.size(); k-- > 0;) {
    const TapeOp& op = tape[k];
    switch (op.kind) {
      case TapeOp::GEMM: {
        if (op.recompute) {
          exec_(op.pre);
          for (const Contraction& q : op.pres) exec_(q);
          if (double* zb = bar_of(op.zero_p)) ops::zero(zb, op.zero_n, s_);
        }
        reverse_gemm(op.c);
        break;
      }
      case TapeOp::PERM: {  // dst = a P(src) + b dst
        double* db = bar_of(op.dst);
        if (!db) break;
        int64_t e[4];
        int inv[4];
        for (int q = 0; q < 4; ++q) e[q] = op.d[op.perm[q]];
        for (int q = 0; q < 4; ++q) inv[op.perm[q]] = q;
        if (double* sb = bar_of(op.x)) ops::permute4(sb, db, e, inv, op.a, 1.0, s_);
        const int64_t n = e[0] * e[1] * e[2] * e[3];
        if (op.b == 0.0) ops::zero(db, n, s_);
        else if (op.b != 1.0) ops::axpby(db, op.b, db, 0.0, nullptr, 0.0, n, s_);
        break;
      }
      case TapeOp::AXPBY: {  // out = a x + b y + c out
        double* ob = bar_of(op.dst);
        if (!ob) break;
        double keep = op.cc;
        if (op.x == op.dst) keep += op.a;
        else if (double* xb = bar_of(op.x)) ops::axpby(xb, 1.0, xb, op.a, ob, 0.0, op.n, s_);
        if (op.y) {
          if (op.y == op.dst) keep += op.b;
          else if (double* yb = bar_of(op.y)) ops::axpby(yb, 1.0, yb, op.b, ob, 0.0, op.n, s_);
        }
        if (keep == 0.0) ops::zero(ob, op.n, s_);
        else if (keep != 1.0) ops::axpby(ob, keep, ob, 0.0, nullptr, 0.0, op.n, s_);
        break;
      }
      case TapeOp::RANK1: {  // out = a A + b t t^T  (n x n)
        double* ob = bar_of(op.dst);
        if (!ob) break;
        const int64_t n = op.n;
        if (double* tb = bar_of(op.y)) {  // tbar += b (obar + obar^T) t
          Contraction g; g.M = n; g.N = 1; g.K = n;
          g.A = rm(ob, n); g.B = vw(cp(op.y), 0, 1, 0, 0); g.C = vw(tb, 0, 1, 0, 0);
          g.alpha = op.b; g.beta = 1.0;
          gemm(g, s_, scratch_);
          g.A = tr(ob, n);
          gemm(g, s_, scratch_);
        }
        if (op.x == op.dst) {
          if (op.a != 1.0) ops::axpby(ob, op.a, ob, 0.0, nullptr, 0.0, n * n, s_);
        } else {
          if (double* ab = bar_of(op.x)) ops::axpby(ab, 1.0, ab, op.a, ob, 0.0, n * n, s_);
          ops::zero(ob, n * n, s_);
        }
        break;
      }
      case TapeOp::SYMM: {
        if (double* rb = bar_of(op.dst)) ops::symmetrize(rb, op.n, s_);
        break;
      }
      case TapeOp::COPY: {
        double* db = bar_of(op.dst);
        if (!db) break;
        if (double* sb = bar_of(op.x)) ops::axpby(sb, 1.0, sb, 1.0, db, 0.0, op.n, s_);
        ops::zero(db, op.n, s_);
        break;
      }
      case TapeOp::ZERO: {
        if (double* db = bar_of(op.dst)) ops::zero(db, op.n, s_);
        break;
      }
    }
  }
}

void Schedule::energy_gradients(const double*, double*, double*) {
  throw Error(ERR_UNSUPPORTED, "energy gradients are provided by the CCSD/CCD schedules");
}

void Schedule::prepare_vjp(const double*) {
  throw Error(ERR_UNSUPPORTED, "reverse mode is provided by the CCSD/CCD schedules");
}

void Schedule::vjp(const double*, double*, const VertexBar*, const double*) {
  throw Error(ERR_UNSUPPORTED, "reverse mode is provided by the CCSD/CCD schedules");
}

}  // namespace cc4s_b200
