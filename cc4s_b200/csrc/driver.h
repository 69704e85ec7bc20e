// State behind one cc4s_cc_handle.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../../include/cc4s_cc.h"
#include "ccsd_complex.h"
#include "drccd.h"
#include "ccsd_real.h"
#include "ops.h"
#include "triples.h"

namespace cc4s_b200 {

struct Handle {
  explicit Handle(const cc4s_cc_options& o);
  ~Handle();

  void set_inputs(const double* eps_h, int64_t No, const double* eps_p, int64_t Nv,
                  const double* gamma, int64_t NG, bool is_complex, bool half_grid);
  void set_initial(const double* T1, const double* T2);
  int run(cc4s_cc_result* out);
  void get_amplitudes(double* T1, double* T2);
  void residual(const double* T1, const double* T2, double* R1, double* R2);
  void backward(double* S_of_G, double* dE_dGamma);

  // helpers
  double* take(size_t elems);
  void free_state();
  void allocate_state();
  void reset_mixer();
  void require_inputs() const;
  // Layout change between the caller's column-major T1/T2 and the device
  // amplitude vector, through a full-size device staging vector st (not dst/src).
  void upload_amplitudes(double* dst, const double* T1, const double* T2, double* st);
  void download_amplitudes(const double* src, double* T1, double* T2, double* st);
  void mix(double* A_new, double* dT_new, double* norm2_dev, double* out);
  std::string diis_failure(int status, int iteration, double energy, double norm);
  // reverse mode (real path)
  Schedule* adjoint_schedule();
  void scatter_vertex_bar(const Schedule::VertexBar& vb, double* out);
  void residual_vjp(const double* T1, const double* T2, const double* R1b, const double* R2b,
                    double* T1b, double* T2b, double* dGamma);
  void relaxed_gradient(int max_iterations, double convergence, double* dE_dGamma,
                        cc4s_cc_lambda_result* out);
  // finite-size correction (structure factor + interpolation) at the current amplitudes
  void finite_size_correction(const double* U, int64_t NGG, const double* V, const double* grid,
                              const double* recip, const cc4s_cc_fsc_options& o, double* S_out,
                              cc4s_cc_fsc_result* out);
  // perturbative triples at the current amplitudes
  void triples(const cc4s_cc_triples_options& o, cc4s_cc_triples_result* out);

  cc4s_cc_options opt;
  Stream stream = nullptr;
  void* ev0 = nullptr;
  void* ev1 = nullptr;
  std::string error;

  RealSystem sys;
  ComplexSystem csys;
  ops::AmpShape shape{0, 0, 1};
  bool complex_path = false;
  std::vector<double*> vertex;  // device inputs (vertex slices, energies)
  std::vector<double*> state;   // amplitudes, DIIS history, scalars
  std::unique_ptr<Schedule> solver;
  std::unique_ptr<Schedule> adj;  // reverse-mode schedule, built on first use

  double* Tcur = nullptr;   // current amplitudes (mixer output)
  double* Rbuf = nullptr;   // residual
  double* dTlast = nullptr; // linear mixer: last change
  std::vector<double*> A;   // DIIS amplitude slots
  std::vector<double*> Rs;  // DIIS change slots
  double* scal = nullptr;   // [0..3] energy, [4] norm^2, [8..] dots
  double* ws = nullptr;     // reduction partials
  double* B = nullptr;      // DIIS bordered overlap matrix
  double* coef = nullptr;   // DIIS coefficients
  int* status_dev = nullptr;
  std::vector<int> valid;
  int next_index = 0, count = 0;
  bool linear_has_last = false;
  bool have_T = false;
  // shape of the caller's vertex (for the adjoint outputs)
  int64_t in_NG = 0, in_Np = 0;
  bool in_complex = false, in_stacked = false;
};

}  // namespace cc4s_b200
