// Real-path CCSD / CCD residual (cc4s Ccsd<Real>::getResiduum) on one B200.
#pragma once

#include "schedule.h"

namespace cc4s_b200 {

struct RealOptions {
  bool ccd = false;         // T1 == 0, R1 dropped
  bool adjoint = false;     // reverse mode (separate buffers for every recorded value)
  bool ppl = true;          // particle-particle ladder from vertex slabs
  int64_t slab = 0;         // PPL block size in virtual orbitals (0: automatic)
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

class CcsdReal : public Schedule {
 public:
  CcsdReal(const RealSystem& sys, const RealOptions& opt, Stream s);

  void residual(const double* T, double* R) override;
  const double* Vd() const override { return Vd_; }
  // The exchange integrals V_abji are read from Vd through index views (no copy).
  const double* Ve() const override { return nullptr; }
  // dE/dT (amplitude vector g) and dE/dV_abij (pair layout Vd_bar, may be null) of
  // E = sum X (2 V_abij - V_abji), X = T2 + T1 T1, at amplitudes T.
  void energy_gradients(const double* T, double* g, double* Vd_bar) override;
  void prepare_vjp(const double* T) override;
  void vjp(const double* Rbar, double* Tbar, const VertexBar* gbar,
           const double* extra_Vd_bar) override;

 private:
  void build_integrals();
  void ppl(const double* Xd, double* R2, const double* dGpp);

  RealSystem sys_;
  RealOptions opt_;
  // static integrals: Vd is the only (vo)^2 one; its exchange and pp pairings
  // are strided views
  double *Vd_ = nullptr;
  double *Vhhhh_ = nullptr, *Vhhhp_ = nullptr, *Vh2_ = nullptr;
  // workspace: four (vo)^2 buffers.  EX also holds 2V - V^x (for Kki, Kac) at
  // the start of a residual and the ring / singles combinations (W8) between uses.
  double *Xd_ = nullptr, *Y_ = nullptr, *EX_ = nullptr;
  // roles: 2V - V^x, crossed-ring EX, ring M1, singles 2X - X^x, X'^x, dressed ring vertex
  double *Vt_ = nullptr, *EX2_ = nullptr, *W8r_ = nullptr, *W8s_ = nullptr, *Yx_ = nullptr,
         *A2_ = nullptr;
  // reverse mode: forward output of the prepared residual and its amplitudes
  double* Rf_ = nullptr;
  const double* Tprep_ = nullptr;
  double *Kki_ = nullptr, *Kac_ = nullptr, *Lac_ = nullptr, *Lki_ = nullptr, *jG_ = nullptr;
  double *U_ = nullptr, *dGph_ = nullptr, *W_ = nullptr, *Z_ = nullptr, *W1_ = nullptr,
         *F_ = nullptr, *dGpp_ = nullptr, *dGhh_ = nullptr, *Q_ = nullptr, *Xkl1_ = nullptr,
         *Xkl2_ = nullptr, *kck_ = nullptr, *P1_ = nullptr, *P_ = nullptr, *slab_ = nullptr;
  int64_t slab_rows_ = 0, slab_cols_ = 0;  // ladder block size, c-panel size
};

}  // namespace cc4s_b200
