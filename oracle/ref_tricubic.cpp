// Test infrastructure, not product code: a C entry point around the reference's
// own Catmull-Rom tricubic interpolator (src/main/gte/TricubicInterpolation.hpp,
// IntpTricubic3<double> with catmullRom = true, the class FiniteSizeCorrection.cxx:254-258
// constructs), compiled from the header where it lies in the reference tree by
// oracle/build_ref.py, so that the oracle's restatement (oracle/fsc.py) is
// checked against the reference's arithmetic itself.
#include <gte/TricubicInterpolation.hpp>

extern "C" void ref_tricubic(int nx, int ny, int nz, double x0, double y0, double z0,
                             const double* F, int n, const double* points, double* out) {
  // unit spacing, as FiniteSizeCorrection.cxx:254-258 builds it on the lattice box
  gte::IntpTricubic3<double> f(nx, ny, nz, x0, 1.0, y0, 1.0, z0, 1.0, F, true);
  for (int k = 0; k < n; ++k) out[k] = f(points[3 * k], points[3 * k + 1], points[3 * k + 2]);
}
