// Iteration loop (CoupledCluster::run) and the extern "C" entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "driver.h"

namespace cc4s_b200 {

int energy_noalloc(const double* T1, const double* T2, const double* V, int64_t No, int64_t Nv,
                   int is_complex, double* out, cudaStream_t stream, const char** err);

// Reference layout T1[a,i], T2[a,b,i,j] (first index fastest) -> amplitude vector.
// Complex host buffers are interleaved (re, im); device vectors are planar.
void Handle::upload_amplitudes(double* dst, const double* T1, const double* T2, double* st) {
  const int64_t o = shape.o, v = shape.v, n1 = v * o, pl = shape.plane();
  std::vector<double> h1, h2;
  for (int64_t p = 0; p < shape.planes; ++p) {
    const double* s1 = T1;
    const double* s2 = T2;
    if (shape.planes > 1) {
      h1.resize(n1);
      h2.resize(n1 * n1);
      for (int64_t k = 0; k < n1; ++k) h1[k] = T1[2 * k + p];
      for (int64_t k = 0; k < n1 * n1; ++k) h2[k] = T2[2 * k + p];
      s1 = h1.data();
      s2 = h2.data();
    }
    ops::h2d(st, s1, n1, stream);
    ops::h2d(st + n1, s2, n1 * n1, stream);
    const int64_t d1[4] = {1, 1, o, v};
    const int p1[4] = {0, 1, 3, 2};
    ops::permute4(dst + p * pl, st, d1, p1, 1.0, 0.0, stream);
    const int64_t d2[4] = {o, o, v, v};  // [j][i][b][a]
    const int p2[4] = {3, 1, 2, 0};      // -> [a][i][b][j]
    ops::permute4(dst + p * pl + n1, st + n1, d2, p2, 1.0, 0.0, stream);
    ops::sync(stream);
  }
}

void Handle::download_amplitudes(const double* src, double* T1, double* T2, double* st) {
  const int64_t o = shape.o, v = shape.v, n1 = v * o, pl = shape.plane();
  std::vector<double> h1, h2;
  for (int64_t p = 0; p < shape.planes; ++p) {
    const int64_t d1[4] = {1, 1, v, o};
    const int p1[4] = {0, 1, 3, 2};
    ops::permute4(st, src + p * pl, d1, p1, 1.0, 0.0, stream);
    const int64_t d2[4] = {v, o, v, o};  // [a][i][b][j]
    const int p2[4] = {3, 1, 2, 0};      // -> [j][i][b][a]
    ops::permute4(st + n1, src + p * pl + n1, d2, p2, 1.0, 0.0, stream);
    if (shape.planes == 1) {
      if (T1) ops::d2h(T1, st, n1, stream);
      if (T2) ops::d2h(T2, st + n1, n1 * n1, stream);
      ops::sync(stream);
    } else {
      h1.resize(n1);
      h2.resize(n1 * n1);
      ops::d2h(h1.data(), st, n1, stream);
      ops::d2h(h2.data(), st + n1, n1 * n1, stream);
      ops::sync(stream);
      if (T1) for (int64_t k = 0; k < n1; ++k) T1[2 * k + p] = h1[k];
      if (T2) for (int64_t k = 0; k < n1 * n1; ++k) T2[2 * k + p] = h2[k];
    }
  }
}

void Handle::set_initial(const double* T1, const double* T2) {
  require_inputs();
  if (!T1 || !T2) throw Error(ERR_INVALID_ARGUMENT, "null amplitudes");
  const int64_t n1 = shape.n1(), np = shape.planes;
  for (int64_t k = 0; k < n1 * np; ++k)
    if (!std::isfinite(T1[k])) throw Error(ERR_NON_FINITE, "non-finite T1");
  for (int64_t k = 0; k < n1 * n1 * np; ++k)
    if (!std::isfinite(T2[k])) throw Error(ERR_NON_FINITE, "non-finite T2");
  upload_amplitudes(Tcur, T1, T2, Rbuf);
  ops::sync(stream);
  have_T = true;
}

// Error text of a failed DIIS solve: the reason, the iteration and the bordered
// overlap matrix (DiisMixer.cxx:116-133 raises the same failure).
std::string Handle::diis_failure(int status, int iteration, double energy, double norm) {
  const int N = static_cast<int>(A.size()), M = N + 1;
  std::vector<double> b(M * M);
  ops::d2h(b.data(), B, b.size(), stream);
  ops::sync(stream);
  std::string msg = std::string("Diagonalization failed (") +
                    (status == 2 ? "non-finite entry" : "singular") +
                    " DIIS system) at iteration " + std::to_string(iteration + 1) +
                    "; previous energy " + std::to_string(energy) + ", residuum norm " +
                    std::to_string(norm) + "; B =";
  char buf[64];
  for (int r = 0; r < M; ++r) {
    msg += " [";
    for (int c = 0; c < M; ++c) {
      std::snprintf(buf, sizeof(buf), c ? " %.3e" : "%.3e", b[r * M + c]);
      msg += buf;
    }
    msg += "]";
  }
  return msg;
}

void Handle::mix(double* A_new, double* dT_new, double* norm2_dev, double* out) {
  const int64_t n = shape.total();
  if (opt.mixer == CC4S_MIXER_LINEAR) {
    const double r = opt.ratio;
    if (!linear_has_last) {
      ops::d2d(out, A_new, n, stream);
      ops::d2d(dTlast, dT_new, n, stream);
      linear_has_last = true;
    } else {
      ops::axpby(out, r, A_new, 1.0 - r, out, 0.0, n, stream);
      ops::axpby(dTlast, r, dT_new, 1.0 - r, dTlast, 0.0, n, stream);
    }
    const double* ys[1] = {dTlast};
    ops::dots(dTlast, ys, 1, n, norm2_dev, ws, stream);
    return;
  }
  const int N = static_cast<int>(A.size());
  const int next = next_index;
  valid[next] = 1;
  const double* ys[8];
  int ny = 0;
  for (int i = 0; i < N; ++i)
    if (valid[i]) ys[ny++] = Rs[i];
  ops::dots_packed(Rs[next], ys, ny, shape, scal + 8, ws, stream);
  if (count < N) ++count;
  ops::diis_solve(B, scal + 8, valid.data(), N, next, count, coef, status_dev, stream);
  const double* xs[16];
  const double* rs[16];
  for (int j = 0; j < count; ++j) {
    const int slot = (next + N - j) % N;
    xs[j] = A[slot];
    rs[j] = Rs[slot];
  }
  ops::lincomb_packed(out, xs, rs, coef, count, shape, norm2_dev, ws, stream);
  next_index = (next + 1) % N;
}

int Handle::run(cc4s_cc_result* out) {
  require_inputs();
  std::memset(out, 0, sizeof(*out));
  out->second_order = std::nan("");
  reset_mixer();
  const bool split = opt.precision != CC4S_PRECISION_FP64;
  solver->set_precision(split ? 3 : 0);
  const int maxIt = opt.max_iterations;
  const double shift = opt.level_shift;
  const int N = static_cast<int>(A.size());
  std::complex<double> e(0.0, 0.0), prev(0.0, 0.0);
  double host[8];
  double Dr = 0, Xr = 0;
  int i = 0;
  for (; i < maxIt; ++i) {
    ops::event_record(ev0, stream);
    solver->residual(have_T ? Tcur : nullptr, Rbuf);
    const int slot = opt.mixer == CC4S_MIXER_DIIS ? next_index : 0;
    if (opt.mixer == CC4S_MIXER_DIIS)
      ops::jacobi_packed(A[slot], Rs[slot], Rbuf, have_T ? Tcur : nullptr, sys.eh, sys.ep, shape,
                         shift, stream);
    else
      ops::jacobi(A[slot], Rs[slot], Rbuf, have_T ? Tcur : nullptr, sys.eh, sys.ep, shape, shift,
                  stream);
    const bool second = !have_T;
    mix(A[slot], Rs[slot], scal + 4, Tcur);
    have_T = true;
    ops::energy(Tcur, solver->Vd(), solver->Vd_im(), solver->Ve(), solver->Ve_im(), shape, scal, ws, stream);
    ops::event_record(ev1, stream);
    ops::d2h(host, scal, 5, stream);
    double st = 0.0;
    if (opt.mixer == CC4S_MIXER_DIIS) ops::d2h(&st, reinterpret_cast<double*>(status_dev), 1, stream);
    ops::sync(stream);
    const float ms = ops::event_ms(ev0, ev1);
    int status_int;
    std::memcpy(&status_int, &st, sizeof(int));
    if (opt.mixer == CC4S_MIXER_DIIS && status_int != 0)
      throw Error(ERR_DIIS_SINGULAR, diis_failure(status_int, i, prev.real(), i > 0 && i <= CC4S_MAX_HISTORY ? out->residuum_norm[i - 1] : 0.0));
    if (opt.precision != CC4S_PRECISION_FP64 && solver->device_error())
      throw Error(ERR_TIMEOUT, "a tensor-core kernel gave up a bounded wait");
    Dr = host[0]; Xr = host[1];
    e = std::complex<double>(host[0] + host[1], host[2] + host[3]);
    const double norm = std::sqrt(host[4]);
    if (!std::isfinite(e.real()) || !std::isfinite(norm))
      throw Error(ERR_NON_FINITE, "non-finite energy or residuum norm at iteration " + std::to_string(i + 1));
    if (i < CC4S_MAX_HISTORY) {
      out->energy[i] = e.real();
      out->delta_energy[i] = (e - prev).real();
      out->residuum_norm[i] = norm;
      out->seconds[i] = ms * 1e-3;
      out->history_len = i + 1;
    }
    if (second) out->second_order = e.real();
    if (std::abs(e - prev) < opt.energy_convergence && norm < opt.amplitudes_convergence) break;
    // defect correction: the split form brings the amplitudes close, FP64 finishes
    if (split && !out->refined_from && opt.precision_refinement > 0.0 &&
        norm < opt.precision_refinement) {
      solver->set_precision(0);
      out->refined_from = i + 2;
    }
    prev = e;
  }
  (void)N;
  if (maxIt == 0) {
    if (!have_T) throw Error(ERR_STATE, "maxIterations = 0 needs initial amplitudes");
    ops::energy(Tcur, solver->Vd(), solver->Vd_im(), solver->Ve(), solver->Ve_im(), shape, scal, ws, stream);
    ops::d2h(host, scal, 4, stream);
    ops::sync(stream);
    Dr = host[0]; Xr = host[1];
    e = std::complex<double>(host[0] + host[1], host[2] + host[3]);
  }
  out->correlation = e.real();
  out->correlation_imag = e.imag();
  out->direct = Dr;
  out->exchange = Xr;
  out->iterations = (i < maxIt) ? i + 1 : maxIt;
  out->converged = i < maxIt ? 1 : 0;
  out->flops_per_iteration = solver->flops_per_residual();
  return (maxIt > 0 && i == maxIt) ? ERR_NOT_CONVERGED : OK;
}

void Handle::get_amplitudes(double* T1, double* T2) {
  require_inputs();
  if (!have_T) throw Error(ERR_STATE, "no amplitudes: run first");
  download_amplitudes(Tcur, T1, T2, Rbuf);
}

void Handle::residual(const double* T1, const double* T2, double* R1, double* R2) {
  require_inputs();
  const int64_t n1 = shape.n1();
  const bool first = (T1 == nullptr && T2 == nullptr);
  if (!first && (!T1 || !T2))
    throw Error(ERR_INVALID_ARGUMENT, "give both T1 and T2, or neither");
  // The caller's amplitudes go to a temporary device vector (also the staging
  // buffer of the layout change), so the handle's current amplitudes and mixer
  // history stay as they were.
  double* Tin = ops::alloc(shape.total());
  try {
    if (!first) upload_amplitudes(Tin, T1, T2, Rbuf);
    solver->residual(first ? nullptr : Tin, Rbuf);
    download_amplitudes(Rbuf, R1, R2, Tin);
  } catch (...) {
    ops::release(Tin);
    throw;
  }
  ops::release(Tin);
  (void)n1;
}

// Adjoint of the energy at the current (frozen) amplitudes.
void Handle::backward(double* S_of_G, double* dE_dGamma) {
  require_inputs();
  if (!have_T) throw Error(ERR_STATE, "no amplitudes: run or set initial amplitudes first");
  if (!S_of_G && !dE_dGamma) return;
  if (dE_dGamma && complex_path)
    throw Error(ERR_UNSUPPORTED, "dE/dGamma is provided on the real (half-grid) path only");
  const int64_t G = solver->aux_rows(), o = shape.o, v = shape.v, n1 = o * v;
  double* Sd = ops::alloc(G);
  double* dG = nullptr;
  try {
    if (dE_dGamma) dG = ops::alloc(G * n1);
    solver->structure_factor(Tcur, Sd, dG);
    std::vector<double> S(G), g;
    ops::d2h(S.data(), Sd, G, stream);
    if (dG) {
      g.resize(G * n1);
      ops::d2h(g.data(), dG, G * n1, stream);
    }
    ops::sync(stream);
    const int64_t NG = in_NG, Np = in_Np;
    if (S_of_G)
      for (int64_t k = 0; k < NG; ++k) S_of_G[k] = S[k] + (in_stacked ? S[k + NG] : 0.0);
    if (dE_dGamma) {
      // caller layout Gamma[G, p, q] column-major, ph block p = No + a, q = i
      const int64_t es = in_complex ? 2 : 1;
      std::memset(dE_dGamma, 0, sizeof(double) * NG * Np * Np * es);
      for (int64_t part = 0; part < (in_stacked ? 2 : 1); ++part)
        for (int64_t k = 0; k < NG; ++k)
          for (int64_t a = 0; a < v; ++a)
            for (int64_t i = 0; i < o; ++i)
              dE_dGamma[(k + NG * ((o + a) + Np * i)) * es + part] =
                  g[((part * NG + k) * v + a) * o + i];
    }
  } catch (...) {
    ops::release(Sd);
    ops::release(dG);
    throw;
  }
  ops::release(Sd);
  ops::release(dG);
}

// Reverse-mode schedule, built on first use: the fast schedule reuses buffers,
// this one keeps every recorded value of a residual.  Real half-grid path
// (CcsdReal) or complex path (CcsdComplex, adjoints of both planes).
Schedule* Handle::adjoint_schedule() {
  if (opt.method == CC4S_METHOD_DRCCD)
    throw Error(ERR_UNSUPPORTED, "reverse mode is provided for Ccsd and Ccd");
  if (!adj) {
    RealOptions ro;
    ro.ccd = opt.method == CC4S_METHOD_CCD;
    ro.ppl = opt.ppl != 0;
    ro.slab = opt.integrals_slice_size;
    ro.adjoint = true;
    if (complex_path) adj.reset(new CcsdComplex(csys, ro, stream));
    else adj.reset(new CcsdReal(sys, ro, stream));
  }
  // the handle's precision: the split form runs the recorded residual and the
  // large contractions of every reverse sweep on the tensor cores
  adj->set_precision(opt.precision != CC4S_PRECISION_FP64 ? 3 : 0);
  return adj.get();
}

// Device vertex-block adjoints -> caller layout Gamma[G, p, q] (column-major,
// interleaved complex when the input was complex; stacked Re/Im auxiliary rows
// go to the two parts).  out is overwritten.
void Handle::scatter_vertex_bar(const Schedule::VertexBar& vb, double* out) {
  const int64_t o = shape.o, v = shape.v, G = sys.G, NG = in_NG, Np = in_Np;
  // planes of the device blocks: stacked Re/Im rows (real path) or the planar
  // real and imaginary parts (complex path) go to the two parts of the output
  const int64_t es = in_complex ? 2 : 1, parts = (in_stacked || complex_path) ? 2 : 1;
  const int64_t planes = complex_path ? 2 : 1;
  std::memset(out, 0, sizeof(double) * NG * Np * Np * es);
  struct Block { const double* d; int64_t row0, nx, col0, ny; };
  const Block blocks[4] = {{vb.Gpp, o, v, o, v}, {vb.Gph, o, v, 0, o}, {vb.Ghh, 0, o, 0, o},
                           {vb.Ghp, 0, o, o, v}};
  std::vector<double> h;
  for (const Block& b : blocks) {
    if (!b.d) continue;
    h.resize(planes * G * b.nx * b.ny);
    ops::d2h(h.data(), b.d, h.size(), stream);
    ops::sync(stream);
    for (int64_t part = 0; part < parts; ++part)
      for (int64_t k = 0; k < NG; ++k)
        for (int64_t x = 0; x < b.nx; ++x)
          for (int64_t y = 0; y < b.ny; ++y)
            out[(k + NG * ((b.row0 + x) + Np * (b.col0 + y))) * es + part] +=
                h[((part * NG + k) * b.nx + x) * b.ny + y];
  }
}

void Handle::residual_vjp(const double* T1, const double* T2, const double* R1b,
                          const double* R2b, double* T1b, double* T2b, double* dGamma) {
  require_inputs();
  if (!T1 || !T2 || !R1b || !R2b) throw Error(ERR_INVALID_ARGUMENT, "null amplitudes or adjoint");
  Schedule* adjs = adjoint_schedule();
  const int64_t n = shape.total(), o = shape.o, v = shape.v, G = sys.G;
  std::vector<double*> tmp;
  auto dev = [&](int64_t k) { double* p = ops::alloc(k); tmp.push_back(p); return p; };
  try {
    double* Tin = dev(n);
    double* Rb = dev(n);
    double* Tb = dev(n);
    upload_amplitudes(Tin, T1, T2, Rbuf);
    upload_amplitudes(Rb, R1b, R2b, Rbuf);
    adjs->prepare_vjp(Tin);
    Schedule::VertexBar vb;
    if (dGamma) {
      const int64_t pl = complex_path ? 2 : 1;
      vb.Gpp = dev(pl * G * v * v); vb.Gph = dev(pl * G * v * o); vb.Ghh = dev(pl * G * o * o);
      vb.Ghp = dev(pl * G * o * v);
      ops::zero(vb.Gpp, pl * G * v * v, stream); ops::zero(vb.Gph, pl * G * v * o, stream);
      ops::zero(vb.Ghh, pl * G * o * o, stream); ops::zero(vb.Ghp, pl * G * o * v, stream);
    }
    adjs->vjp(Rb, Tb, dGamma ? &vb : nullptr, nullptr);
    download_amplitudes(Tb, T1b, T2b, Rbuf);
    if (dGamma) scatter_vertex_bar(vb, dGamma);
  } catch (...) {
    for (double* p : tmp) ops::release(p);
    throw;
  }
  for (double* p : tmp) ops::release(p);
}

// Lambda equations (dR/dT + D)^T lambda = -dE/dT by the amplitude iteration's own
// Jacobi update and mixer, then dE/dGamma = dE/dGamma|_T + lambda^T dR/dGamma.
void Handle::relaxed_gradient(int max_iterations, double convergence, double* dE_dGamma,
                              cc4s_cc_lambda_result* out) {
  require_inputs();
  if (!have_T) throw Error(ERR_STATE, "no amplitudes: run first");
  if (max_iterations < 1) throw Error(ERR_INVALID_ARGUMENT, "maxIterations < 1");
  std::memset(out, 0, sizeof(*out));
  Schedule* adjs = adjoint_schedule();
  const int64_t n = shape.total(), o = shape.o, v = shape.v, G = sys.G, n1 = shape.n1();
  std::vector<double*> tmp;
  auto dev = [&](int64_t k) { double* p = ops::alloc(k); tmp.push_back(p); return p; };
  try {
    double* lam = dev(n);
    double* g = dev(n);
    double* Jt = dev(n);
    const int64_t planes = complex_path ? 2 : 1;
    double* VdB = dev(planes * n1 * n1);
    ops::event_record(ev0, stream);
    adjs->prepare_vjp(Tcur);
    adjs->energy_gradients(Tcur, g, VdB);
    ops::event_record(ev1, stream);
    out->prepare_seconds = 1e-3 * ops::event_ms(ev0, ev1);
    reset_mixer();
    ops::zero(lam, n, stream);
    const bool diis = opt.mixer == CC4S_MIXER_DIIS;
    double host[8];
    int it = 0;
    for (; it < max_iterations; ++it) {
      ops::event_record(ev0, stream);
      if (it == 0) {
        ops::d2d(Rbuf, g, n, stream);
      } else {
        adjs->vjp(lam, Jt, nullptr, nullptr);
        ops::axpby(Rbuf, 1.0, g, 1.0, Jt, 0.0, n, stream);
      }
      const int slot = diis ? next_index : 0;
      if (diis)
        ops::jacobi_packed(A[slot], Rs[slot], Rbuf, it ? lam : nullptr, sys.eh, sys.ep,
                           shape, opt.level_shift, stream);
      else
        ops::jacobi(A[slot], Rs[slot], Rbuf, it ? lam : nullptr, sys.eh, sys.ep, shape,
                    opt.level_shift, stream);
      mix(A[slot], Rs[slot], scal + 4, lam);
      ops::event_record(ev1, stream);
      ops::d2h(host, scal + 4, 1, stream);
      double st = 0.0;
      if (diis) ops::d2h(&st, reinterpret_cast<double*>(status_dev), 1, stream);
      ops::sync(stream);
      int status_int;
      std::memcpy(&status_int, &st, sizeof(int));
      if (diis && status_int != 0)
        throw Error(ERR_DIIS_SINGULAR, "Lambda equations: " + diis_failure(status_int, it, 0.0, out->residuum_norm));
      const double norm = std::sqrt(host[0]);
      if (!std::isfinite(norm)) throw Error(ERR_NON_FINITE, "non-finite Lambda update");
      const double sec = 1e-3 * ops::event_ms(ev0, ev1);
      if (it > 0) out->vjp_seconds = sec;
      out->residuum_norm = norm;
      if (norm < convergence) { ++it; out->converged = 1; break; }
    }
    out->iterations = it;
    Schedule::VertexBar vb;
    vb.Gpp = dev(planes * G * v * v); vb.Gph = dev(planes * G * v * o);
    vb.Ghh = dev(planes * G * o * o); vb.Ghp = dev(planes * G * o * v);
    ops::zero(vb.Gpp, planes * G * v * v, stream); ops::zero(vb.Gph, planes * G * v * o, stream);
    ops::zero(vb.Ghh, planes * G * o * o, stream); ops::zero(vb.Ghp, planes * G * o * v, stream);
    ops::event_record(ev0, stream);
    adjs->vjp(lam, Jt, &vb, VdB);
    ops::event_record(ev1, stream);
    out->gradient_seconds = 1e-3 * ops::event_ms(ev0, ev1);
    if (dE_dGamma) scatter_vertex_bar(vb, dE_dGamma);
  } catch (...) {
    for (double* p : tmp) ops::release(p);
    throw;
  }
  for (double* p : tmp) ops::release(p);
}

}  // namespace cc4s_b200

// ---------------------------------------------------------------------------
using cc4s_b200::Error;
using cc4s_b200::Handle;

struct cc4s_cc_handle {
  Handle* impl;
};

// Perturbative triples at the current amplitudes (triples.h).  The schedule
// and its integral slices live for this call only.
void Handle::triples(const cc4s_cc_triples_options& o, cc4s_cc_triples_result* out) {
  require_inputs();
  if (!have_T) throw Error(ERR_STATE, "no amplitudes: run the CoupledCluster step or set initial amplitudes first");
  if (o.block_size < 0) throw Error(ERR_INVALID_ARGUMENT, "block_size < 0");
  if (o.formulation != 0 && o.formulation != 1)
    throw Error(ERR_INVALID_ARGUMENT, "formulation must be 0 or 1");
  if (o.cT != 0 && o.cT != 1) throw Error(ERR_INVALID_ARGUMENT, "cT must be 0 or 1");
  TriplesOptions to;
  to.block = o.block_size;
  to.reference_form = o.formulation == 1;
  to.complete = o.cT == 1;
  Triples tr(sys, complex_path ? &csys : nullptr, to, stream);
  tr.set_precision(opt.precision == CC4S_PRECISION_SPLIT3 ? 3 : 0);
  tr.set_profile(opt.profile != 0);
  const TriplesOutcome r = tr.run(Tcur);
  if (!std::isfinite(r.energy)) throw Error(ERR_NON_FINITE, "non-finite (T) energy");
  out->correlation = r.energy;
  out->seconds = r.seconds;
  out->setup_seconds = r.setup_seconds;
  out->flops = r.flops;
  out->executed_flops = r.executed_flops;
  out->block_size = r.block;
  out->block_triples = r.block_triples;
  for (int k = 0; k < 4; ++k) out->phase_seconds[k] = r.phase_seconds[k];
  out->cr_denominator = r.cr_denominator;
  // the basis MP2 energy of the (T*) ratio (PerturbativeTriplesStar.hpp:79-99)
  ops::mp2_energy(solver->Vd(), solver->Vd_im(), sys.eh, sys.ep, shape.o, shape.v, scal, ws,
                  stream);
  double mp2[2];
  ops::d2h(mp2, scal, 2, stream);
  ops::sync(stream);
  out->mp2_energy = mp2[0] + mp2[1];
}

// Finite-size correction at the current amplitudes: the plane-wave structure
// factor S(G) on the device (Schedule::structure_factor_pw), then the lattice
// box and the two energy sums of FiniteSizeCorrection::interpolation
// (FiniteSizeCorrection.cxx:135-310).  The box geometry comes from the grid
// vectors on the host, as the reference derives it.
void Handle::finite_size_correction(const double* U, int64_t NGG, const double* V,
                                    const double* grid, const double* recip,
                                    const cc4s_cc_fsc_options& o, double* S_out,
                                    cc4s_cc_fsc_result* out) {
  require_inputs();
  if (!have_T) throw Error(ERR_STATE, "no amplitudes: run the CoupledCluster step or set initial amplitudes first");
  if (!grid || !recip) throw Error(ERR_INVALID_ARGUMENT, "null grid vectors or reciprocal basis");
  if (NGG <= 0) throw Error(ERR_BAD_SHAPE, "NGG must be positive");
  if (!U && NGG != in_NG) throw Error(ERR_BAD_SHAPE, "without singular vectors NGG must equal NG");
  if (o.interpolation_grid_size <= 0) throw Error(ERR_INVALID_ARGUMENT, "interpolationGridSize <= 0");
  const int64_t NF = in_NG;
  // geometry (host): inverse basis, cell volume, box of the lattice coordinates
  ops::FscGeometry g;
  double B[3][3], A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) B[r][c] = recip[3 * r + c];
  auto cross = [](const double* a, const double* b, double* out3) {
    out3[0] = a[1] * b[2] - a[2] * b[1];
    out3[1] = a[2] * b[0] - a[0] * b[2];
    out3[2] = a[0] * b[1] - a[1] * b[0];
  };
  double c01[3], c12[3], c20[3];
  cross(B[0], B[1], c01); cross(B[1], B[2], c12); cross(B[2], B[0], c20);
  const double omega = std::fabs(c01[0] * B[2][0] + c01[1] * B[2][1] + c01[2] * B[2][2]);
  if (!(omega > 0.0) || !std::isfinite(omega)) throw Error(ERR_INVALID_ARGUMENT, "degenerate reciprocal basis");
  for (int c = 0; c < 3; ++c) { A[0][c] = c12[c] / omega; A[1][c] = c20[c] / omega; A[2][c] = c01[c] / omega; }
  double dmin[3] = {0, 0, 0}, dmax[3] = {0, 0, 0};
  for (int64_t i = 0; i < NGG; ++i)
    for (int d = 0; d < 3; ++d) {
      const double x = A[d][0] * grid[3 * i] + A[d][1] * grid[3 * i + 1] + A[d][2] * grid[3 * i + 2];
      if (!std::isfinite(x)) throw Error(ERR_NON_FINITE, "non-finite grid vector");
      dmin[d] = std::min(dmin[d], x);
      dmax[d] = std::max(dmax[d], x);
    }
  int64_t cells = 1;
  for (int d = 0; d < 3; ++d) {
    g.dims[d] = static_cast<int64_t>(std::floor(dmax[d] - dmin[d] + 1.5));
    g.origin[d] = std::floor(dmin[d] + 0.5);
    if (g.dims[d] < 4) throw Error(ERR_BAD_SHAPE, "interpolation box needs at least 4 points per direction");
    cells *= g.dims[d];
    if (cells > (int64_t(1) << 31)) throw Error(ERR_BAD_SHAPE, "interpolation box too large");
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) { g.A[3 * r + c] = A[r][c]; g.B[3 * r + c] = B[r][c]; }
  g.NG = NGG;
  g.N = o.interpolation_grid_size;
  g.f = o.unit_factor * omega / 2.0 / M_PI / M_PI;
  std::vector<double*> tmp;
  auto tk = [&](int64_t n) { double* p = ops::alloc(n); tmp.push_back(p); return p; };
  try {
    double* Uw = tk(2 * NGG * NF);
    double* Ud = U ? tk(2 * NGG * NF) : nullptr;
    double* Vd = V ? tk(NGG) : nullptr;
    double* Sd = tk(NGG);
    double* gd = tk(3 * NGG);
    double* box = tk(cells);
    double* red = tk(2048);
    double* sums = tk(2);
    ops::event_record(ev0, stream);
    if (Ud) ops::h2d(Ud, U, 2 * NGG * NF, stream);
    if (Vd) ops::h2d(Vd, V, NGG, stream);
    ops::h2d(gd, grid, 3 * NGG, stream);
    ops::fsc_prepare_u(Uw, Uw + NGG * NF, Ud, Vd, NGG, NF, stream);
    solver->structure_factor_pw(Tcur, Uw, NGG, NF, Sd);
    ops::fsc_box(box, Sd, gd, g, stream);
    ops::fsc_sums(box, Sd, gd, g, red, sums, stream);
    double h[2];
    ops::d2h(h, sums, 2, stream);
    if (S_out) ops::d2h(S_out, Sd, NGG, stream);
    ops::event_record(ev1, stream);
    out->seconds = ops::event_ms(ev0, ev1) * 1e-3;
    ops::sync(stream);
    if (solver->device_error()) throw Error(ERR_TIMEOUT, "tensor-core kernel wait expired");
    const double N3 = double(g.N) * g.N * g.N;
    out->uncorrected = h[0];
    out->corrected = h[1] / N3 / 8.0;
    out->correction = out->corrected - out->uncorrected;
    for (int d = 0; d < 3; ++d) out->box[d] = g.dims[d];
    if (!std::isfinite(out->corrected) || !std::isfinite(out->uncorrected))
      throw Error(ERR_NON_FINITE, "non-finite finite-size correction");
  } catch (...) {
    for (double* p : tmp) ops::release(p);
    throw;
  }
  for (double* p : tmp) ops::release(p);
}

namespace {
thread_local std::string g_create_error;

template <class F>
int guarded(cc4s_cc_handle* h, F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    if (h && h->impl) h->impl->error = e.what(); else g_create_error = e.what();
    return e.status;
  } catch (const std::exception& e) {
    if (h && h->impl) h->impl->error = e.what(); else g_create_error = e.what();
    return cc4s_b200::ERR_CUDA;
  } catch (...) {
    if (h && h->impl) h->impl->error = "unknown error"; else g_create_error = "unknown error";
    return cc4s_b200::ERR_CUDA;
  }
}
}  // namespace

extern "C" {

void cc4s_cc_default_options(cc4s_cc_options* o) {
  if (!o) return;
  o->method = CC4S_METHOD_CCSD;
  o->precision = CC4S_PRECISION_FP64;
  o->mixer = CC4S_MIXER_DIIS;
  o->max_residua = 4;
  o->ratio = 1.0;
  o->max_iterations = 16;
  o->energy_convergence = 1e-7;
  o->amplitudes_convergence = 1e-6;
  o->level_shift = 0.0;
  o->integrals_slice_size = 0;
  o->ppl = 1;
  o->device = 0;
  o->profile = 0;
  o->linearized = 0;
  o->adjacent_pairs_exchange = 0;
  o->precision_refinement = 0.0;
}

int cc4s_cc_create(const cc4s_cc_options* opt, cc4s_cc_handle** h) {
  if (!opt || !h) { g_create_error = "null argument"; return CC4S_ERR_INVALID_ARGUMENT; }
  *h = nullptr;
  return guarded(nullptr, [&] {
    auto* hh = new cc4s_cc_handle{nullptr};
    try {
      hh->impl = new Handle(*opt);
    } catch (...) {
      delete hh;
      throw;
    }
    *h = hh;
    return 0;
  });
}

int cc4s_cc_set_inputs(cc4s_cc_handle* h, const double* eps_h, int64_t No, const double* eps_p,
                       int64_t Nv, const double* gamma, int64_t NG, int is_complex,
                       int half_grid) {
  if (!h || !h->impl) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] {
    h->impl->set_inputs(eps_h, No, eps_p, Nv, gamma, NG, is_complex != 0, half_grid != 0);
    return 0;
  });
}

int cc4s_cc_set_initial_amplitudes(cc4s_cc_handle* h, const double* T1, const double* T2) {
  if (!h || !h->impl) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] { h->impl->set_initial(T1, T2); return 0; });
}

int cc4s_cc_run(cc4s_cc_handle* h, cc4s_cc_result* out) {
  if (!h || !h->impl || !out) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] { return h->impl->run(out); });
}

int cc4s_cc_get_amplitudes(cc4s_cc_handle* h, double* T1, double* T2) {
  if (!h || !h->impl) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] { h->impl->get_amplitudes(T1, T2); return 0; });
}

int cc4s_cc_residual(cc4s_cc_handle* h, const double* T1, const double* T2, double* R1,
                     double* R2) {
  if (!h || !h->impl || !R1 || !R2) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] { h->impl->residual(T1, T2, R1, R2); return 0; });
}

int cc4s_cc_backward(cc4s_cc_handle* h, double* S_of_G, double* dE_dGamma) {
  if (!h || !h->impl) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] { h->impl->backward(S_of_G, dE_dGamma); return 0; });
}

int cc4s_cc_residual_vjp(cc4s_cc_handle* h, const double* T1, const double* T2,
                         const double* R1bar, const double* R2bar, double* T1bar, double* T2bar,
                         double* dGamma) {
  if (!h || !h->impl || !T1bar || !T2bar) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] {
    h->impl->residual_vjp(T1, T2, R1bar, R2bar, T1bar, T2bar, dGamma);
    return 0;
  });
}

int cc4s_cc_relaxed_gradient(cc4s_cc_handle* h, int max_iterations, double convergence,
                             double* dE_dGamma, cc4s_cc_lambda_result* out) {
  if (!h || !h->impl || !out) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] {
    h->impl->relaxed_gradient(max_iterations, convergence, dE_dGamma, out);
    return out->converged ? 0 : static_cast<int>(CC4S_WARN_NOT_CONVERGED);
  });
}

void cc4s_cc_triples_default_options(cc4s_cc_triples_options* o) {
  if (!o) return;
  o->block_size = 0;
  o->formulation = 0;
  o->cT = 0;
}

int cc4s_cc_perturbative_triples(cc4s_cc_handle* h, const cc4s_cc_triples_options* opt,
                                 cc4s_cc_triples_result* out) {
  if (!h || !h->impl || !opt || !out) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] {
    h->impl->triples(*opt, out);
    return 0;
  });
}

void cc4s_cc_fsc_default_options(cc4s_cc_fsc_options* o) {
  if (!o) return;
  o->interpolation_grid_size = 20;
  o->unit_factor = 1.0;
}

int cc4s_cc_finite_size_correction(cc4s_cc_handle* h, const double* singular_vectors,
                                   int64_t NGG, const double* coulomb_potential,
                                   const double* grid_vectors, const double* reciprocal_basis,
                                   const cc4s_cc_fsc_options* opt, double* S_of_G,
                                   cc4s_cc_fsc_result* out) {
  if (!h || !h->impl || !opt || !out) return CC4S_ERR_INVALID_ARGUMENT;
  return guarded(h, [&] {
    h->impl->finite_size_correction(singular_vectors, NGG, coulomb_potential, grid_vectors,
                                    reciprocal_basis, *opt, S_of_G, out);
    return 0;
  });
}

int cc4s_cc_get_stats(const cc4s_cc_handle* h, cc4s_cc_stats* out) {
  if (!h || !h->impl || !out) return CC4S_ERR_INVALID_ARGUMENT;
  // each split-precision contraction is two slicing launches plus the tensor-core kernel
  out->gemm_launches = cc4s_b200::gemm_launch_count() + cc4s_b200::split_launch_count() +
                       cc4s_b200::split_pack_launch_count();
  out->other_launches = cc4s_b200::ops::launch_count();
  size_t bytes = 0;
  if (h->impl->solver) bytes += h->impl->solver->device_bytes();
  out->device_bytes = bytes;
  out->flops_per_residual = h->impl->solver ? h->impl->solver->flops_per_residual() : 0.0;
  out->gemm_seconds = out->gemm_flops = out->top_seconds = out->top_flops = 0.0;
  out->gemm_profiled_launches = 0;
  out->split_seconds = out->split_flops = 0.0;
  out->split_launches = 0;
  if (h->impl->solver) {
    const auto& p = h->impl->solver->profile();
    out->gemm_seconds = p.gemm_seconds;
    out->gemm_flops = p.gemm_flops;
    out->top_seconds = p.top_seconds;
    out->top_flops = p.top_flops;
    out->gemm_profiled_launches = p.launches;
    out->split_seconds = p.split_seconds;
    out->split_flops = p.split_flops;
    out->split_launches = p.split_launches;
  }
  return 0;
}

int cc4s_cc_energy_noalloc(const double* T1, const double* T2, const double* Vpphh, int64_t No,
                           int64_t Nv, int is_complex, double* energy, void* stream) {
  const char* err = "";
  const int st = cc4s_b200::energy_noalloc(T1, T2, Vpphh, No, Nv, is_complex, energy,
                                            static_cast<cudaStream_t>(stream), &err);
  if (st) g_create_error = err;
  return st;
}

int cc4s_cc_destroy(cc4s_cc_handle* h) {
  if (!h) return CC4S_ERR_INVALID_ARGUMENT;
  int st = guarded(h, [&] { delete h->impl; h->impl = nullptr; return 0; });
  delete h;
  return st;
}

const char* cc4s_cc_last_error(const cc4s_cc_handle* h) {
  if (h && h->impl) return h->impl->error.c_str();
  return g_create_error.c_str();
}

}  // extern "C"
