// Test-only entry into Schedule::ein for the emulation library: one labelled
// contraction C = alpha A B + beta C on host arrays (the emulated device memory),
// so that the label fusion, the host loops over wide index groups, batch labels
// and the planar complex path can be checked against numpy's einsum.
#include <cstring>
#include <string>
#include <vector>

#include "../../cc4s_b200/csrc/schedule.h"

namespace {
using cc4s_b200::Schedule;

class EinProbe : public Schedule {
 public:
  EinProbe() : Schedule(nullptr) {}
  void residual(const double*, double*) override {}
  const double* Vd() const override { return nullptr; }
  const double* Ve() const override { return nullptr; }
  using Schedule::ein;
  using Schedule::Ten;
};

EinProbe::Ten make(const char* labels, const int64_t* dims, double* p, int64_t im, int conj) {
  EinProbe::Ten t;
  t.p = p;
  t.labels = labels;
  t.dims.assign(dims, dims + std::strlen(labels));
  t.im = im;
  t.conj = conj != 0;
  return t;
}
}  // namespace

// Returns 0 on success, else writes the error message into err (errlen bytes).
extern "C" int emu_ein(double alpha, const char* la, const int64_t* da, double* A, int64_t a_im,
                       int conjA, const char* lb, const int64_t* db, double* B, int64_t b_im,
                       int conjB, double beta, const char* lc, const int64_t* dc, double* C,
                       int64_t c_im, int64_t* launches, char* err, int errlen) {
  try {
    EinProbe e;
    const uint64_t g0 = cc4s_b200::gemm_launch_count();
    e.ein(alpha, make(la, da, A, a_im, conjA), make(lb, db, B, b_im, conjB), beta,
          make(lc, dc, C, c_im, 0));
    if (launches) *launches = static_cast<int64_t>(cc4s_b200::gemm_launch_count() - g0);
    return 0;
  } catch (const std::exception& x) {
    std::strncpy(err, x.what(), static_cast<size_t>(errlen) - 1);
    err[errlen - 1] = 0;
    return 1;
  }
}
