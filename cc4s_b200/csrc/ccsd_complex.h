// Complex-path CCSD / CCD residual (cc4s Ccsd<Complex>::getResiduum) on one B200.
//
// Complex tensors are stored as two planes (real plane, then imaginary plane);
// every complex contraction runs as four real FP64 tensor-core contractions,
// with conjugation folded into the sign of the imaginary-plane terms.
#pragma once

#include "ccsd_real.h"
#include "schedule.h"

namespace cc4s_b200 {

// Device-resident inputs of the complex path (planar complex, im plane at +size).
struct ComplexSystem {
  int64_t o = 0, v = 0, G = 0;
  double* eh = nullptr;
  double* ep = nullptr;
  double* Gpp = nullptr;  // [G][v][v]
  double* Gph = nullptr;  // [G][v][o]
  double* Ghh = nullptr;  // [G][o][o]
  double* Ghp = nullptr;  // [G][o][v]
};

class CcsdComplex : public Schedule {
 public:
  CcsdComplex(const ComplexSystem& sys, const RealOptions& opt, Stream s);

  void residual(const double* T, double* R) override;
  const double* Vd() const override { return Vd_; }
  // The exchange integrals V_baij are read from Vd by block swap (no copy).
  const double* Ve() const override { return nullptr; }
  const double* Vd_im() const override { return Vd_ + D2_; }
  const double* Ve_im() const override { return nullptr; }
  // Reverse mode (schedules built with opt.adjoint), as on the real path: every
  // complex tensor is its two real planes, so the recorded real operations give
  // the adjoints with respect to the real and imaginary parts.
  void energy_gradients(const double* T, double* g, double* Vd_bar) override;
  void prepare_vjp(const double* T) override;
  void vjp(const double* Rbar, double* Tbar, const VertexBar* gbar,
           const double* extra_Vd_bar) override;

 private:
  // X = T + alpha t t^T on planar complex operands (recorded while taping)
  void zrank1_(double* Xr, double* Xi, const double* Tr, const double* Ti, const double* tr,
               const double* ti, double alpha, int64_t n);
  void zperm(double* dst, int64_t dst_im, const double* src, int64_t src_im, const int64_t d[4],
             const int p[4], double alpha, double beta, bool conj = false);
  void zaxpby(double* out, double a, const double* x, double b, const double* y, int64_t n);
  void build_integrals();

  ComplexSystem sys_;
  RealOptions opt_;
  int64_t D2_ = 0;
  // Stored (vo)^2 complex tensors: Vd, Vh4, M2, X, Y, EX.  Every other pairing
  // is a strided view; EX also holds 2 V_klcd - V_kldc at the start of a
  // residual and the ring / singles combinations (W8) between uses.
  double *Vd_ = nullptr, *Vh4_ = nullptr, *M2_ = nullptr, *Vhhhh_ = nullptr,
         *Vhhhp_ = nullptr, *Vh2_ = nullptr;
  double *Xd_ = nullptr, *Y_ = nullptr, *W8_ = nullptr, *EX_ = nullptr;
  // roles sharing EX, Y and cTdGph on the fast path, separate in reverse mode:
  // 2V - V^x (Kki, Kac, kck), crossed-ring EX, singles W8, the first Y of the
  // ring, the dressed ring vertex after its second dressing; zt: t_re + t_im
  double *Vt_ = nullptr, *EX2_ = nullptr, *W8s_ = nullptr, *Yx_ = nullptr, *cTdGph2_ = nullptr,
         *zt_ = nullptr;
  double* Rf_ = nullptr;
  const double* Tprep_ = nullptr;
  double *Kki_ = nullptr, *Kac_ = nullptr, *Lac_ = nullptr, *Lki_ = nullptr, *jG_ = nullptr,
         *U_ = nullptr, *cTdGph_ = nullptr, *W_ = nullptr, *SQ_ = nullptr, *W1_ = nullptr,
         *F_ = nullptr, *cTdGpp_ = nullptr, *dGpp_ = nullptr, *dGhh_ = nullptr,
         *Xkl1_ = nullptr, *Xkl2_ = nullptr, *kck_ = nullptr, *P1_ = nullptr, *P_ = nullptr,
         *slab_ = nullptr;
  int64_t slab_rows_ = 0, slab_cols_ = 0;  // ladder block size, c-panel size
};

}  // namespace cc4s_b200
