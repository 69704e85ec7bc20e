// Perturbative triples (T) energy on the device (real half-grid path and
// planar complex path).
//
// The energy of cc4s PerturbativeTriples / PerturbativeTriplesReference
// (src/main/algorithms/PerturbativeTriplesReference.cxx:107-175; the tuple
// loop of perturbative-triples/src/atrip/Atrip.cxx:447-525 with
// include/atrip/Equations.hpp), evaluated over blocks of virtual indices:
//
//   X_abcijk  = sum_d T_adij V_bcdk - sum_l T_abil V_jklc          (base term)
//   W         = sum of X over the six simultaneous permutations of (ai)(bj)(ck)
//   S         = W + T_ai V_bcjk + T_bj V_acik + T_ck V_abij
//   E_(T)     = sum_abcijk W (4/3 S_abcijk - 2 S_acbijk + 2/3 S_bcaijk) / D,
//   D         = eps_i + eps_j + eps_k - eps_a - eps_b - eps_c.
// Complex path: the hole integrals enter conjugated, and the two reference
// steps differ in one conjugation of the energy: PerturbativeTriples (atrip,
// Equations.hpp getEnergyDistinct) takes Re conj(W) Z, PerturbativeTriplesReference
// (:136-173) takes Re conj(W) conj(Z).  The energy kernel returns
// sum Re W Re Z / D and sum Im W Im Z / D, their sum and difference.
//
// For every block triple A <= B <= C the block array S[(a,i)][(b,j)][(c,k)]
// (a in A, b in B, c in C, pair layout) is formed on the device: the singles
// first, then six contractions over K = v + o, each the particle term of one
// output arrangement and the (transposed) hole term that writes the same
// elements, each writing its permutation of X straight into the pair layout
// through the strided output view.  The energy kernel then sums over
// the block; the other orderings of the three blocks are folded in through the
// symmetry of W and S under simultaneous permutations, which turns each
// ordering into a permutation of the hole indices inside the same block
// (coefficients()).  Blocks sized so that the block array stays in L2 keep the
// six read-modify-write passes of the contractions on chip.
#pragma once

#include "ccsd_complex.h"
#include "ccsd_real.h"
#include "schedule.h"

namespace cc4s_b200 {

struct TriplesOptions {
  int64_t block = 0;            // virtual indices per block (0: automatic)
  bool reference_form = false;  // complex path: PerturbativeTriplesReference's conjugation
  // The cT branch of PerturbativeTriplesReference (:92-109, :178-179): the
  // completely renormalised intermediates I_bcek, I_mcjk of ct::getCompleteTriples
  // (CompleteTriples.cxx:11-118) in place of V_bcek and V_jkmc in a second block
  // array M, and E = sum M (4/3 S - 2 S_acb + 2/3 S_bca)^* / D.
  bool complete = false;
};

struct TriplesOutcome {
  double energy = 0.0;
  double seconds = 0.0;         // device time of the block loop (integrals excluded)
  double setup_seconds = 0.0;   // device time of the integral slices
  double flops = 0.0;           // 2 o^3 v^3 (o + v), the reference's count
  double executed_flops = 0.0;  // contractions launched (whole block triples)
  int64_t block = 0, block_triples = 0;
  // cT: the denominator of the CR-(T) energy, correlation / cr_denominator
  // (ct::getDenominator, CompleteTriples.cxx:120-165); 0 otherwise
  double cr_denominator = 0.0;
  // with profiling: device time of the singles, the particle contractions, the
  // hole contractions and the energy kernel, summed over the block triples
  double phase_seconds[4] = {0.0, 0.0, 0.0, 0.0};
};

class Triples : public Schedule {
 public:
  // Real half-grid path (stacked Re/Im vertex rows) or the planar complex path
  // (cs != nullptr; rs then only gives o, v, G, eh, ep).
  Triples(const RealSystem& rs, const ComplexSystem* cs, const TriplesOptions& opt, Stream s);
  // E_(T) of amplitudes T (amplitude-vector layout: one real plane, or real and
  // imaginary planes on the complex path) on the device.
  TriplesOutcome run(const double* T);
  // Not a residual schedule.
  void residual(const double* T, double* R) override;
  const double* Vd() const override { return Vpphh_; }
  const double* Ve() const override { return nullptr; }

  // Block length whose block arrays (arrays * planes * (block * o)^3) fit the L2-sized budget.
  static int64_t auto_block(int64_t o, int64_t v, int planes);
  // Weights of the six hole permutations (012, 021, 102, 120, 201, 210) for the
  // block triple (A, B, C), A <= B <= C: every distinct ordering sigma of the
  // blocks adds 4/3 to the identity, -2 to sigma t23 sigma^-1 and 2/3 to
  // sigma c^-1 sigma^-1 (t23 swaps the last two positions, c rotates left).
  static void coefficients(int64_t A, int64_t B, int64_t C, double coef[6]);

 private:
  // S += the six permutations of X = sum_d T V^p - sum_l T V^h through the
  // K-concatenated operands Ac (rows (pair, hole)) and Bc (columns (virtual, pair)).
  void connected(const ops::TriplesBlock& b, const int64_t X[3], const int64_t n[3],
                 const double* Ac, const double* Bc, double* S);
  // The same six contractions in the split form from operands sliced once per
  // evaluation (w = 0: S from Ac_/Bc_, w = 1: M from AcM_/BcM_).
  void connected_packed(const ops::TriplesBlock& b, const int64_t X[3], const int64_t n[3],
                        int w, double* S);
  // Slices Ac (rows (pair, hole) and (hole, pair)) and Bc (rows (virtual, pair)) of
  // every plane for connected_packed.
  void pack_operands(int w, const double* Ac, const double* Bc);
  // Ac[(a,i)][j][k] = T_adij (k = d < v), -V^h_jail^* (k = v + l);
  // Bc[b][(c,k)][k'] = V^p_bcdk (k' = d < v), T_cbkl (k' = v + l); V^p in the layout of
  // Vppph_, V^h in that of Vhhhp_.
  void concat_operands(const double* T, const double* Vp, const double* Vh, double* Ac,
                       double* Bc);
  // I_bcek into Ip_ and I_mcjk into Ih_ at amplitudes T (cT branch).
  void complete_intermediates(const double* T);
  // beta C + alpha V_pqsr for the integral slice `name` (LO RO LI RI), C labelled
  // by lab = the characters of p, q, s, r.
  void vslice(const char* name, const char* lab, double alpha, double beta, const Ten& C);
  RealSystem sys_;
  const ComplexSystem* cs_ = nullptr;
  bool cplx_ = false, reference_form_ = false, complete_ = false;
  int64_t o_ = 0, v_ = 0, n1_ = 0, nb_ = 0;
  int64_t vi_pphh_ = 0, vi_ppph_ = 0, vi_hhhp_ = 0, si_ = 0;  // imaginary-plane offsets
  double* Vpphh_ = nullptr;  // V_abij, pair layout [(a,i)][(b,j)]
  double* Vppph_ = nullptr;  // V_bcdk as [b][(c,k)][d]
  double* Vhhhp_ = nullptr;  // V_jklc as [j][(c,k)][l]
  double* S_ = nullptr;      // block array (imaginary plane at S_ + si_)
  double* Ip_ = nullptr;     // cT: I_bcdk in the layout of Vppph_
  double* Ih_ = nullptr;     // cT: I_lcjk as [j][(c,k)][l], the layout of Vhhhp_
  double* Mb_ = nullptr;     // cT: block array of M (layout of S_)
  // K-concatenated operands of the block contractions (K = v + o; second pair for M)
  double* Ac_ = nullptr;
  double* Bc_ = nullptr;
  double* AcM_ = nullptr;
  double* BcM_ = nullptr;
  int64_t kc_ = 0, ai_ = 0, bi_ = 0;  // v + o; imaginary-plane offsets of Ac, Bc
  struct Sliced {
    SplitOperand A, A2, B;  // Ac rows (pair, hole), Ac rows (hole, pair), Bc rows (virtual, pair)
  };
  Sliced sl_[2][2];         // [S or M][plane]
  double* sl_mem_[2] = {nullptr, nullptr};
  double* ws_ = nullptr;     // reduction partials
  double* slots_ = nullptr;  // two energy sums of every block triple, then their totals
  double* cr_slots_ = nullptr;  // cT: the two CR-(T) sums of every block triple, then totals
  // cT: 1 + 2 sum t_ai t_ai + sum (2 T_abij - T_baij)(T_abij + t_ai t_bj), the amplitude-only
  // terms of the CR-(T) denominator (real part)
  double cr_amplitude_terms(const double* T);
  int64_t ntri_ = 0;
  double setup_seconds_ = 0.0;
};

}  // namespace cc4s_b200
