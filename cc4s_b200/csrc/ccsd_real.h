// Real-path CCSD / CCD residual (cc4s Ccsd<Real>::getResiduum) on one B200.
#pragma once

#include "ops.h"

#include <vector>

namespace cc4s_b200 {

struct RealOptions {
  bool ccd = false;         // T1 == 0, R1 dropped
  bool ppl = true;          // particle-particle ladder from vertex slabs
  int64_t slab = 0;         // PPL slab size in virtual orbitals (0: automatic)
};

// Device-resident inputs of the real path.  G counts stacked real rows: the
// reference's real integrals Re*Re + Im*Im (VertexCoulombIntegrals.cxx:87-121)
// are one real vertex whose auxiliary index runs over [Re rows; Im rows].
struct RealSystem {
  int64_t o = 0, v = 0, G = 0;
  double* eh = nullptr;   // [o]
  double* ep = nullptr;   // [v]
  double* Gpp = nullptr;  // [G][v][v]  Gamma_G,a,b
  double* Gph = nullptr;  // [G][v][o]  Gamma_G,a,i
  double* Ghh = nullptr;  // [G][o][o]  Gamma_G,k,i
  double* Ghp = nullptr;  // [G][o][v]  Gamma_G,i,a
};

class CcsdReal {
 public:
  CcsdReal(const RealSystem& sys, const RealOptions& opt, Stream s);
  ~CcsdReal();
  CcsdReal(const CcsdReal&) = delete;
  CcsdReal& operator=(const CcsdReal&) = delete;

  // R = residual(T).  T, R are amplitude vectors (ops::AmpShape, one plane);
  // T == nullptr is the first iteration (R1 = 0, R2 = V_abij).
  void residual(const double* T, double* R);

  // Pair-layout integrals used by the energy: Vd = V_abij, Ve = V_baij.
  const double* Vd() const { return Vd_; }
  const double* Ve() const { return Ve_; }

  // FP64-equivalent flops of one residual evaluation (this schedule).
  double flops_per_residual() const { return flops_; }
  size_t device_bytes() const { return bytes_; }

  // Per-launch timing of the tensor-core contractions (CUDA events around each
  // launch).  Off by default; when on, residual() synchronises at its end.
  void set_profile(bool on) { profile_ = on; }
  struct Profile {
    double gemm_seconds = 0, gemm_flops = 0;      // all contractions of the last residual
    double top_seconds = 0, top_flops = 0;        // the most expensive single launch
    int launches = 0;
  };
  const Profile& profile() const { return prof_; }

 private:
  void gemm_(const Contraction& c);
  double* take(size_t elems);
  void build_integrals();
  void ppl(const double* Xp, double* R2, const double* dGpp);

  RealSystem sys_;
  RealOptions opt_;
  Stream s_;
  GemmScratch scratch_;
  std::vector<double*> owned_;
  size_t bytes_ = 0;
  double flops_ = 0.0;
  bool count_flops_ = true;
  bool profile_ = false;
  Profile prof_;
  std::vector<void*> ev_;          // event pool: 2 per profiled launch
  std::vector<double> ev_flops_;
  void profile_finish();
  // static integrals
  double *Vd_ = nullptr, *Ve_ = nullptr, *Vp_ = nullptr, *Vtp_ = nullptr;
  double *Vhhhh_ = nullptr, *Vhhhp_ = nullptr, *Vh2_ = nullptr;
  // workspace
  double *Xd_ = nullptr, *Xp_ = nullptr, *Te_ = nullptr, *Y_ = nullptr, *W8_ = nullptr,
         *Tp_ = nullptr, *EX_ = nullptr;
  double *Kki_ = nullptr, *Kac_ = nullptr, *Lac_ = nullptr, *Lki_ = nullptr, *jG_ = nullptr;
  double *U_ = nullptr, *dGph_ = nullptr, *W_ = nullptr, *Z_ = nullptr, *W1_ = nullptr,
         *F_ = nullptr, *dGpp_ = nullptr, *dGhh_ = nullptr, *Q_ = nullptr, *Xkl1_ = nullptr,
         *Xkl2_ = nullptr, *kck_ = nullptr, *P1_ = nullptr, *P_ = nullptr, *slab_ = nullptr;
  int64_t slab_rows_ = 0;
};

}  // namespace cc4s_b200
