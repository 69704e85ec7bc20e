// CoupledCluster iteration driver and C ABI (include/cc4s_cc.h).
//
// Host-side restatement of CoupledCluster::run (CoupledCluster.cxx:56-191) and
// of the mixers (DiisMixer.cxx:59-107, LinearMixer.cxx:44-61).  Amplitudes,
// residual, DIIS history, overlap matrix and coefficients stay on the device;
// per iteration only the energy and the residual norm (5 doubles) and the
// DIIS status come back to the host for the convergence test.
#include "driver.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace cc4s_b200 {

Handle::Handle(const cc4s_cc_options& o) : opt(o) {
  if (opt.method != CC4S_METHOD_CCSD && opt.method != CC4S_METHOD_CCD &&
      opt.method != CC4S_METHOD_DRCCD)
    throw Error(ERR_INVALID_ARGUMENT, "Unknown method");
  if (opt.mixer != CC4S_MIXER_DIIS && opt.mixer != CC4S_MIXER_LINEAR)
    throw Error(ERR_INVALID_ARGUMENT, "Unknown mixer type");
  if (opt.mixer == CC4S_MIXER_DIIS && (opt.max_residua < 1 || opt.max_residua > 8))
    throw Error(ERR_UNSUPPORTED, "maxResidua must be in [1, 8]");
  if (opt.precision != CC4S_PRECISION_FP64 && opt.precision != CC4S_PRECISION_SPLIT3)
    throw Error(ERR_UNSUPPORTED, "precision must be FP64 or the three-slice split form");
  if (opt.max_iterations < 0) throw Error(ERR_INVALID_ARGUMENT, "maxIterations < 0");
  stream = ops::stream_create(opt.device);
  ev0 = ops::event_create();
  ev1 = ops::event_create();
}

Handle::~Handle() {
  free_state();
  for (double* p : vertex) ops::release(p);
  ops::event_destroy(ev0);
  ops::event_destroy(ev1);
  ops::stream_destroy(stream);
}

double* Handle::take(size_t elems) {
  double* p = ops::alloc(elems);
  state.push_back(p);
  return p;
}

void Handle::free_state() {
  adj.reset();
  solver.reset();
  for (double* p : state) ops::release(p);
  state.clear();
  A.clear(); Rs.clear();
  Tcur = Rbuf = dTlast = scal = ws = B = coef = nullptr;
  status_dev = nullptr;
  have_T = false;
}

void Handle::set_inputs(const double* eps_h, int64_t No, const double* eps_p, int64_t Nv,
                        const double* gamma, int64_t NG, bool is_complex, bool half_grid) {
  if (!eps_h || !eps_p || !gamma) throw Error(ERR_INVALID_ARGUMENT, "null input");
  if (No <= 0 || Nv <= 0 || NG <= 0) throw Error(ERR_BAD_SHAPE, "No, Nv, NG must be positive");
  const int64_t Np = No + Nv;
  const int64_t nin = NG * Np * Np * (is_complex ? 2 : 1);
  for (int64_t k = 0; k < No; ++k)
    if (!std::isfinite(eps_h[k])) throw Error(ERR_NON_FINITE, "non-finite eps_h");
  for (int64_t k = 0; k < Nv; ++k)
    if (!std::isfinite(eps_p[k])) throw Error(ERR_NON_FINITE, "non-finite eps_p");
  free_state();
  for (double* p : vertex) ops::release(p);
  vertex.clear();
  // The vertex goes to the device once; its finiteness and whether any
  // imaginary part is non-zero are decided there (ops::scan_vertex).
  double* staging = ops::alloc(nin);
  bool has_imag = false;
  try {
    ops::h2d(staging, gamma, nin, stream);
    const int flags = ops::scan_vertex(staging, nin, is_complex, stream);
    if (flags & 1) throw Error(ERR_NON_FINITE, "non-finite Coulomb vertex");
    has_imag = (flags & 2) != 0;
    in_NG = NG;
    in_Np = Np;
    in_complex = is_complex;
    in_stacked = half_grid && has_imag;
    auto vtake = [&](size_t n) { double* p = ops::alloc(n); vertex.push_back(p); return p; };
    if (!half_grid) {
      // Complex path: planar complex slices (imaginary plane at +size, zero for real input).
      ComplexSystem cs;
      cs.o = No; cs.v = Nv; cs.G = NG;
      cs.eh = vtake(No); cs.ep = vtake(Nv);
      const int64_t spp = NG * Nv * Nv, sph = NG * Nv * No, shh = NG * No * No;
      cs.Gpp = vtake(2 * spp); cs.Gph = vtake(2 * sph); cs.Ghh = vtake(2 * shh); cs.Ghp = vtake(2 * sph);
      ops::h2d(cs.eh, eps_h, No, stream);
      ops::h2d(cs.ep, eps_p, Nv, stream);
      const int parts = is_complex ? 2 : 1;
      for (int part = 0; part < 2; ++part) {
        if (part >= parts) {
          ops::zero(cs.Gpp + spp, spp, stream); ops::zero(cs.Gph + sph, sph, stream);
          ops::zero(cs.Ghh + shh, shh, stream); ops::zero(cs.Ghp + sph, sph, stream);
          break;
        }
        ops::gather_vertex(cs.Gpp + part * spp, staging, is_complex, part, NG, Np, No, Nv, No, Nv, stream);
        ops::gather_vertex(cs.Gph + part * sph, staging, is_complex, part, NG, Np, No, Nv, 0, No, stream);
        ops::gather_vertex(cs.Ghh + part * shh, staging, is_complex, part, NG, Np, 0, No, 0, No, stream);
        ops::gather_vertex(cs.Ghp + part * sph, staging, is_complex, part, NG, Np, 0, No, No, Nv, stream);
      }
      ops::sync(stream);
      csys = cs;
      sys = RealSystem();
      sys.o = No; sys.v = Nv; sys.G = NG; sys.eh = cs.eh; sys.ep = cs.ep;
      shape = ops::AmpShape{No, Nv, 2};
      complex_path = true;
    } else {
      // Real path: stack Re and (if present) Im rows into one real auxiliary index.
      const int64_t parts = has_imag ? 2 : 1;
      const int64_t G = NG * parts;
      RealSystem rs;
      rs.o = No; rs.v = Nv; rs.G = G;
      rs.eh = vtake(No); rs.ep = vtake(Nv);
      rs.Gpp = vtake(G * Nv * Nv); rs.Gph = vtake(G * Nv * No);
      rs.Ghh = vtake(G * No * No); rs.Ghp = vtake(G * No * Nv);
      ops::h2d(rs.eh, eps_h, No, stream);
      ops::h2d(rs.ep, eps_p, Nv, stream);
      for (int64_t part = 0; part < parts; ++part) {
        const int64_t off = part * NG;
        ops::gather_vertex(rs.Gpp + off * Nv * Nv, staging, is_complex, (int)part, NG, Np, No, Nv, No, Nv, stream);
        ops::gather_vertex(rs.Gph + off * Nv * No, staging, is_complex, (int)part, NG, Np, No, Nv, 0, No, stream);
        ops::gather_vertex(rs.Ghh + off * No * No, staging, is_complex, (int)part, NG, Np, 0, No, 0, No, stream);
        ops::gather_vertex(rs.Ghp + off * No * Nv, staging, is_complex, (int)part, NG, Np, 0, No, No, Nv, stream);
      }
      ops::sync(stream);
      sys = rs;
      shape = ops::AmpShape{No, Nv, 1};
      complex_path = false;
    }
  } catch (...) {
    ops::release(staging);
    for (double* p : vertex) ops::release(p);
    vertex.clear();
    throw;
  }
  ops::release(staging);
  allocate_state();
}

void Handle::allocate_state() {
  RealOptions ro;
  ro.ccd = opt.method == CC4S_METHOD_CCD;
  ro.ppl = opt.ppl != 0;
  // integralsSliceSize sets the ladder block size.  Real path: the ladder is
  // symmetric under (a,c) <-> (b,d), so the block size only trades memory for
  // speed (0: automatic).  Complex path: blocks follow the reference's slices
  // exactly (default No).
  ro.slab = opt.integrals_slice_size;
  if (opt.method == CC4S_METHOD_DRCCD) {
    DrccdOptions dro;
    dro.linearized = opt.linearized != 0;
    dro.adjacent_pairs_exchange = opt.adjacent_pairs_exchange != 0;
    if (complex_path)
      solver.reset(new Drccd(csys.o, csys.v, csys.G, true, csys.Gph, csys.Ghp, dro, stream));
    else
      solver.reset(new Drccd(sys.o, sys.v, sys.G, false, sys.Gph, sys.Ghp, dro, stream));
  } else if (complex_path) {
    solver.reset(new CcsdComplex(csys, ro, stream));
  } else {
    solver.reset(new CcsdReal(sys, ro, stream));
  }
  solver->set_profile(opt.profile != 0);
  solver->set_precision(opt.precision == CC4S_PRECISION_SPLIT3 ? 3 : 0);
  const int64_t n = shape.total();
  Tcur = take(n);
  Rbuf = take(n);
  const int N = opt.mixer == CC4S_MIXER_DIIS ? opt.max_residua : 1;
  // DIIS history in packed form (upper triangle of the symmetric T2 part): half
  // the memory of full vectors, same overlaps and combinations.
  const int64_t slot = opt.mixer == CC4S_MIXER_DIIS ? shape.packed_total() : n;
  for (int k = 0; k < N; ++k) { A.push_back(take(slot)); Rs.push_back(take(slot)); }
  if (opt.mixer == CC4S_MIXER_LINEAR) dTlast = take(n);
  scal = take(64);
  ws = take(4096 * 8);
  B = take((N + 1) * (N + 1));
  coef = take(32);
  status_dev = reinterpret_cast<int*>(take(4));
  reset_mixer();
  ops::sync(stream);
}

void Handle::reset_mixer() {
  const int N = static_cast<int>(A.size());
  std::vector<double> b((N + 1) * (N + 1), 0.0);
  for (int i = 1; i <= N; ++i) { b[i] = -1.0; b[i * (N + 1)] = -1.0; }
  ops::h2d(B, b.data(), b.size(), stream);
  valid.assign(N, 0);
  next_index = 0;
  count = 0;
  linear_has_last = false;
}

void Handle::require_inputs() const {
  if (!solver) throw Error(ERR_STATE, "inputs not set");
}

}  // namespace cc4s_b200
