#include "schedule.h"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

namespace cc4s_b200 {

Schedule::~Schedule() { release_all(); }

void Schedule::release_all() {
  for (void* e : ev_) ops::event_destroy(e);
  ev_.clear();
  if (split_mem_) ops::release(split_mem_);
  split_mem_ = nullptr;
  split_ = SplitScratch();
  for (double* p : owned_) ops::release(p);
  owned_.clear();
}

double* Schedule::take(size_t elems) {
  double* p = ops::alloc(elems);
  owned_.push_back(p);
  bytes_ += elems * sizeof(double);
  return p;
}

void Schedule::gemm_(const Contraction& c) {
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

void Schedule::tc_(const Contraction& c) {
  if (precision_ == 0 || c.batch != 1 || c.K < 64 || c.M < 64 || c.N < 64) {
    gemm_(c);
    return;
  }
  const size_t need = gemm_split_scratch_bytes(c);
  if (need > split_.bytes) {
    ops::sync(s_);
    if (split_mem_) ops::release(split_mem_);
    split_mem_ = nullptr;
    const size_t doubles = (need + 7) / 8 + 2;
    split_mem_ = ops::alloc(doubles);
    split_.p = split_mem_ + 2;
    split_.bytes = need;
    split_.error = reinterpret_cast<int*>(split_mem_);
    ops::zero(split_mem_, 2, s_);
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
    gemm_split(c, s_, split_);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  gemm_split(c, s_, split_);
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

void Schedule::structure_factor(const double* T, double* S_dev, double* dGph_dev) {
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
  {  // W[G][(a,i)] = sum_{b,j} Gamma^hp_Gjb M[(b,j),(a,i)]
    Contraction c; c.M = G; c.N = n1; c.K = n1; c.Ki = o;
    c.A = vw(sGhp_, 0, n1, 1, v); c.B = vw(M, o * n1, n1, 0, 1); c.C = rm(adjW_, n1);
    zgemm(c, gi, mi, gi, false, false, true);
  }
  {  // S[G] = Re sum_r conj(Gamma^ph_G,r) W_G,r   (batched dot products)
    Contraction c; c.M = 1; c.N = 1; c.K = n1; c.batch = G;
    c.A = vw(sGph_, 0, 0, 0, 1, 0, n1); c.B = vw(adjW_, 0, 1, 0, 0, 0, n1);
    c.C = vw(S_dev, 0, 0, 0, 0, 0, 1);
    zgemm(c, gi, gi, 0, scplx_, false);
  }
  if (dGph_dev) {
    if (scplx_) throw Error(ERR_UNSUPPORTED, "dE/dGamma is provided on the real path only");
    Contraction c; c.M = G; c.N = n1; c.K = n1;  // dE/dGph = 2 Gph M
    c.A = rm(sGph_, n1); c.B = rm(M, n1); c.C = rm(dGph_dev, n1); c.alpha = 2.0;
    tc_(c);
  }
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

}  // namespace cc4s_b200
