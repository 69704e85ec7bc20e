// Direct-ring CCD residual (cc4s Drccd::getResiduum) on one B200.
#pragma once

#include "ccsd_complex.h"
#include "ccsd_real.h"
#include "schedule.h"

namespace cc4s_b200 {

struct DrccdOptions {
  bool linearized = false;              // "linearized"
  bool adjacent_pairs_exchange = false; // "adjacentPairsExchange"
};

// Works on both integral paths: real (half-grid, planes = 1) and complex
// (planar, planes = 2).  The vertex slices are those of RealSystem /
// ComplexSystem (complex ones have their imaginary plane at +size).
class Drccd : public Schedule {
 public:
  Drccd(int64_t o, int64_t v, int64_t G, bool complex_path, double* Gph, double* Ghp,
        const DrccdOptions& opt, Stream s);

  void residual(const double* T, double* R) override;
  const double* Vd() const override { return Vd_; }
  const double* Ve() const override { return Ve_; }
  const double* Vd_im() const override { return cplx_ ? Vd_ + D2_ : nullptr; }
  const double* Ve_im() const override { return cplx_ ? Ve_ + D2_ : nullptr; }

 private:
  int64_t o_, v_, G_, D2_;
  bool cplx_;
  double *Gph_, *Ghp_;
  DrccdOptions opt_;
  double *Vd_ = nullptr, *Ve_ = nullptr, *Wq_ = nullptr, *W1_ = nullptr, *Q_ = nullptr;
};

}  // namespace cc4s_b200
