// Common machinery of the residual schedules: device allocations, flop
// accounting, split-K scratch and optional per-launch timing of contractions.
#pragma once

#include <array>
#include <string>
#include <vector>

#include "ops.h"
#include "split_gemm.cuh"

namespace cc4s_b200 {

inline View vw(double* p, int64_t s_ro, int64_t s_ri, int64_t s_co, int64_t s_ci,
               int64_t s_bo = 0, int64_t s_bi = 0) {
  View v;
  v.p = p; v.s_ro = s_ro; v.s_ri = s_ri; v.s_co = s_co; v.s_ci = s_ci; v.s_bo = s_bo;
  v.s_bi = s_bi;
  return v;
}
inline double* cp(const double* p) { return const_cast<double*>(p); }

class Schedule {
 public:
  explicit Schedule(Stream s) : s_(s) {}
  virtual ~Schedule();
  Schedule(const Schedule&) = delete;
  Schedule& operator=(const Schedule&) = delete;

  // R = residual(T) on amplitude vectors (ops::AmpShape layout); T == nullptr is
  // the first iteration (R1 = 0, R2 = V_abij).
  virtual void residual(const double* T, double* R) = 0;
  // Pair-layout integrals of the energy: Vd = V_abij, Ve = V_baij (imaginary
  // planes null on the real path).
  virtual const double* Vd() const = 0;
  virtual const double* Ve() const = 0;
  virtual const double* Vd_im() const { return nullptr; }
  virtual const double* Ve_im() const { return nullptr; }

  double flops_per_residual() const { return flops_; }
  size_t device_bytes() const { return bytes_; }

  void set_profile(bool on) { profile_ = on; }
  // 0: FP64 throughout; 3: the large ladder / ring / vertex contractions run as
  // three-slice split-precision products on the tcgen05 tensor cores (in adjoint
  // mode also the recorded forward pass and the large contractions of the
  // reverse sweep).
  void set_precision(int slices) { precision_ = slices; }
  // Non-zero if a bounded wait inside a tensor-core kernel expired (synchronises).
  int device_error();

  // Adjoint of the energy at frozen amplitudes T (amplitude-vector layout):
  //   S_dev[G]    = Re sum conj(G^ph_Gai) G^hp_Gjb (2 X_abij - X_abji), the transition
  //                 structure factor of FiniteSizeCorrection.cxx:113-125 (= dE/dV(G));
  //   dGph_dev    = dE/dGamma^ph_Gai = 2 sum_bj (2X - X^x)[(a,i),(b,j)] Gamma^ph_Gbj
  //                 (real path only; may be null).
  // G runs over the schedule's auxiliary rows (stacked Re/Im rows on the real path).
  void structure_factor(const double* T, double* S_dev, double* dGph_dev);
  // The plane-wave structure factor of FiniteSizeCorrection.cxx:50-133 with
  // singular vectors:  S[G] = Re sum_{F,F'} conj(Uw_GF) Q_FF' Uw_GF',
  //   Q_FF' = sum_r conj(Gamma^ph_F,r) W_F',r   (W as in structure_factor),
  // Uw = U_GF / sqrt(V(G)) planar complex [2][NGG][NF] (device), NF the caller's
  // vertex rows (the real path's stacked Re/Im rows are folded back into complex
  // rows).  Equal to Gamma_G = U Gamma_F followed by structure_factor, without
  // forming the NGG vertex rows.
  void structure_factor_pw(const double* T, const double* Uw, int64_t NGG, int64_t NF,
                           double* S_dev);
  int64_t aux_rows() const { return sG_; }

  // ---- reverse mode ---------------------------------------------------------
  // Vector-Jacobian products of the residual at fixed amplitudes, for schedules
  // built in adjoint mode.  prepare_vjp(T) evaluates the residual once (in FP64,
  // or with the large contractions in split precision when set_precision(3) was
  // given) with every device operation recorded (buffers that the fast path reuses are
  // separate allocations then, so every recorded value survives);
  // vjp(Rbar, Tbar, gbar) replays the record backwards:
  //   Tbar = Rbar^T dR/dT   (amplitude-vector layout, T2 part symmetrised),
  //   gbar->X += Rbar^T dR/dGamma_X  for the vertex blocks given (may be null),
  // where extra_Vd_bar (pair layout, may be null) is added to the adjoint of the
  // integrals V_abij before they are propagated to the vertex.
  struct VertexBar {
    double* Gpp = nullptr;  // [G][v][v]
    double* Gph = nullptr;  // [G][v][o]
    double* Ghh = nullptr;  // [G][o][o]
    double* Ghp = nullptr;  // [G][o][v]
  };
  bool adjoint_mode() const { return adjoint_; }
  // dE/dT (amplitude vector g, every plane) and dE/dV_abij (pair layout, every
  // plane; may be null) of the correlation energy at amplitudes T.
  virtual void energy_gradients(const double* T, double* g, double* Vd_bar);
  virtual void prepare_vjp(const double* T);
  virtual void vjp(const double* Rbar, double* Tbar, const VertexBar* gbar,
                   const double* extra_Vd_bar);
  struct Profile {
    double gemm_seconds = 0, gemm_flops = 0;  // all contractions of the last residual
    double top_seconds = 0, top_flops = 0;    // the most expensive single launch
    int launches = 0;
    // split-precision launches only (FP64-equivalent flops; 6 FP16 products each)
    double split_seconds = 0, split_flops = 0;
    int split_launches = 0;
  };
  const Profile& profile() const { return prof_; }

 protected:
  // One recorded device operation (forward), replayed backwards by reverse().
  struct TapeOp {
    enum Kind { GEMM, PERM, AXPBY, RANK1, SYMM, COPY, ZERO } kind = GEMM;
    Contraction c;                      // GEMM
    bool recompute = false;             // GEMM: rerun `pre` (and `pres`) forward and
    Contraction pre;                    // clear the adjoint of [zero_p, zero_p + zero_n) first
    std::vector<Contraction> pres;      // further contractions of the recomputation
    double* zero_p = nullptr;
    int64_t zero_n = 0;
    double* dst = nullptr;              // PERM / AXPBY / RANK1 / SYMM / COPY / ZERO output
    const double* x = nullptr;          // PERM / COPY source, AXPBY x, RANK1 A
    const double* y = nullptr;          // AXPBY y, RANK1 t
    int64_t d[4] = {0, 0, 0, 0};
    int perm[4] = {0, 1, 2, 3};
    double a = 0.0, b = 0.0, cc = 0.0;  // PERM alpha/beta; AXPBY a, b, c; RANK1 a, b
    int64_t n = 0;
  };
  // A forward buffer and its adjoint (same size and layout).
  struct Region { const double* p; int64_t n; double* bar; };
  void structure_factor_w(const double* T);
  double* bar_of(const double* p) const;
  View barv(const View& v) const;
  void reverse(const std::vector<TapeOp>& tape);
  void reverse_gemm(const Contraction& c);
  // Bandwidth operations that are recorded while taping.
  void perm_(double* dst, const double* src, const int64_t d[4], const int p[4], double alpha,
             double beta);
  void axpby_(double* out, double a, const double* x, double b, const double* y, double c,
              int64_t n);
  void rank1_(double* out, double a, const double* A, double b, const double* t, int64_t n);
  void sym_(double* R, int64_t n);
  void copy_(double* dst, const double* src, int64_t n);
  void zero_(double* p, int64_t n);
  bool adjoint_ = false;
  bool taping_ = false;
  std::vector<TapeOp> tape_;            // residual at the prepared amplitudes
  std::vector<TapeOp> integrals_tape_;  // iteration-independent integrals from the vertex
  std::vector<Region> regions_;
  std::vector<size_t> owned_n_;         // element counts of owned_
  std::vector<double*> bar_bufs_;       // adjoints of owned_ (adjoint mode)

  double* take(size_t elems);
  void gemm_(const Contraction& c);
  // A large contraction: split precision when enabled (batch 1), else FP64.
  // Recorded on the tape when taping, like gemm_.
  void tc_(const Contraction& c);
  bool split_ok(const Contraction& c) const;
  void split_exec(const Contraction& c);
  // Makes the split scratch hold `regular` bytes for per-contraction packing plus a
  // second region of `extra` bytes (split_extra_) that survives those calls; may
  // reallocate (synchronises).  A later split_exec that needs more than `regular`
  // reallocates with an extra region of the same size (its contents are lost).
  void split_reserve(size_t regular, size_t extra);
  // One split contraction whose B was sliced by split_pack_b (recorded like tc_).
  void tc_packed_b_(const Contraction& c, const SplitPackedB& b);
  // One split contraction with both operands sliced beforehand (split_pack_operand);
  // counted and profiled like tc_, not recorded.
  void tc_prepacked_(const Contraction& c, const SplitOperand& A, const SplitRuns& ar,
                     const SplitOperand& B, const SplitRuns& br);
  void exec_(const Contraction& c);
  // C = alpha * op(A) op(B) + beta * C on planar complex operands: the
  // imaginary plane of each operand sits at the given element offset (0: the
  // operand is real); conjA / conjB conjugate an operand.  Four real
  // contractions; `big` routes them through tc_.
  void zgemm(Contraction c, int64_t a_im, int64_t b_im, int64_t c_im, bool conjA = false,
             bool conjB = false, bool big = false);
  // A labelled operand of ein(): a dense row-major tensor whose indices are named
  // by one character each, in memory order (last fastest), with their extents;
  // `im` the element offset of the imaginary plane (0: real), `conj` conjugates it.
  struct Ten {
    double* p = nullptr;
    std::string labels;
    std::vector<int64_t> dims;
    int64_t im = 0;
    bool conj = false;
  };
  // C = alpha * A B + beta * C over labelled operands, like numpy's einsum with the
  // summed labels those of A and B absent from C (every label in exactly two of the
  // operands, or in all three as a batch label).  Labels that stay adjacent in
  // every operand are fused; groups still wider than the contraction's two levels
  // are looped over on the host.  One zgemm per launch (FP64, or tc_ when big).
  void ein(double alpha, const Ten& A, const Ten& B, double beta, const Ten& C,
           bool big = false);
  void profile_finish();
  int precision_ = 0;
  SplitScratch split_;
  double* split_mem_ = nullptr;
  void* split_extra_ = nullptr;
  size_t split_extra_bytes_ = 0;
  // vertex description for the adjoint (set by each schedule)
  int64_t so_ = 0, sv_ = 0, sG_ = 0;
  bool scplx_ = false;
  double* sGph_ = nullptr;
  double* sGhp_ = nullptr;
  double* adjX_ = nullptr;
  double* adjW_ = nullptr;
  void release_all();

  Stream s_;
  GemmScratch scratch_;
  std::vector<double*> owned_;
  size_t bytes_ = 0;
  double flops_ = 0.0;
  bool count_flops_ = true;
  bool profile_ = false;
  Profile prof_;
  std::vector<void*> ev_;
  std::vector<double> ev_flops_;
  std::vector<char> ev_split_;
  std::vector<std::array<int64_t, 4>> ev_shape_;  // M, N, K, batch of each profiled launch
};

}  // namespace cc4s_b200
