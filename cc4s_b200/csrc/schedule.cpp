#include "schedule.h"

#include <cstring>

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
    ops::event_record(ev_[2 * k], s_);
    gemm_split(c, s_, split_);
    ops::event_record(ev_[2 * k + 1], s_);
    return;
  }
  gemm_split(c, s_, split_);
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
  }
  p.launches = static_cast<int>(ev_flops_.size());
  ev_flops_.clear();
  prof_ = p;
}

}  // namespace cc4s_b200
