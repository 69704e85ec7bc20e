// Bandwidth kernels of the CoupledCluster step (sm_100a).
//
// All kernels are grid-stride loops sized in multiples of the 148 SMs, with
// coalesced 64-bit accesses; transposing permutations stage 32 x 32 tiles in
// shared memory.  Reductions are two-pass and deterministic: each block writes
// a partial sum (warp shuffles + shared memory), a single block then adds the
// partials in a fixed order.
#include "ops.h"

#include <atomic>
#include <cmath>

namespace cc4s_b200 {
namespace ops {

namespace {
std::atomic<uint64_t> g_launches{0};
inline void count() { g_launches.fetch_add(1); }
constexpr int RED_BLOCKS = 148 * 4;  // partial sums per reduction
constexpr int RED_THREADS = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV values; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k][w] = v[k];
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < nw ? sh[k][lane] : 0.0;
      v[k] = warp_sum(x);
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
struct Perm4 {
  int64_t e[4];   // destination dims
  int64_t ss[4];  // source stride of destination axis k
  int64_t ds[4];  // destination strides
};

// Destination inner axis is the source inner axis: straight copy of rows.
__global__ void permute_rows_kernel(double* dst, const double* src, Perm4 p, double alpha,
                                    double beta) {
  const int64_t rows = p.e[0] * p.e[1] * p.e[2];
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int64_t i2 = r % p.e[2];
    const int64_t i1 = (r / p.e[2]) % p.e[1];
    const int64_t i0 = r / (p.e[2] * p.e[1]);
    const double* s = src + i0 * p.ss[0] + i1 * p.ss[1] + i2 * p.ss[2];
    double* d = dst + i0 * p.ds[0] + i1 * p.ds[1] + i2 * p.ds[2];
    for (int64_t x = threadIdx.x; x < p.e[3]; x += blockDim.x) {
      const double v = alpha * s[x];
      d[x] = (beta != 0.0) ? v + beta * d[x] : v;
    }
  }
}

// General permutation: tile over (destination inner axis 3, destination axis q that
// holds the source inner axis); the other two destination axes form the batch.
__global__ void permute_tiled_kernel(double* dst, const double* src, Perm4 p, int q, int b0,
                                     int b1, double alpha, double beta) {
  __shared__ double tile[32][33];
  const int64_t nx = p.e[3], ny = p.e[q];
  const int64_t tx = (nx + 31) / 32, ty = (ny + 31) / 32;
  const int64_t nb = p.e[b0] * p.e[b1];
  const int64_t total = tx * ty * nb;
  for (int64_t blk = blockIdx.x; blk < total; blk += gridDim.x) {
    const int64_t bx = blk % tx;
    const int64_t by = (blk / tx) % ty;
    const int64_t bb = blk / (tx * ty);
    const int64_t ib1 = bb % p.e[b1], ib0 = bb / p.e[b1];
    const int64_t sbase = ib0 * p.ss[b0] + ib1 * p.ss[b1];
    const int64_t dbase = ib0 * p.ds[b0] + ib1 * p.ds[b1];
    // Read: source inner axis (= destination axis q) is contiguous; lanes along y.
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t x = bx * 32 + r, y = by * 32 + threadIdx.x;
      if (x < nx && y < ny) tile[r][threadIdx.x] = src[sbase + x * p.ss[3] + y * p.ss[q]];
    }
    __syncthreads();
    // Write: destination axis 3 contiguous; lanes along x.
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t y = by * 32 + r, x = bx * 32 + threadIdx.x;
      if (x < nx && y < ny) {
        double* d = dst + dbase + y * p.ds[q] + x;
        const double v = alpha * tile[threadIdx.x][r];
        *d = (beta != 0.0) ? v + beta * *d : v;
      }
    }
    __syncthreads();
  }
}

__global__ void axpby_kernel(double* out, double a, const double* x, double b,
                             const double* y, double c, int64_t n) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v = a * x[e];
    if (y) v += b * y[e];
    if (c != 0.0) v += c * out[e];
    out[e] = v;
  }
}

__global__ void rank1_kernel(double* out, double a, const double* A, double b, const double* t,
                             int64_t n) {
  const int64_t total = n * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n, c = e - (e / n) * n;
    out[e] = a * A[e] + b * t[r] * t[c];
  }
}

__global__ void zrank1_kernel(double* ore, double* oim, const double* are, const double* aim,
                              const double* tre, const double* tim, double b, int64_t n) {
  const int64_t total = n * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n, c = e - (e / n) * n;
    const double xr = tre[r] * tre[c] - tim[r] * tim[c];
    const double xi = tre[r] * tim[c] + tim[r] * tre[c];
    ore[e] = are[e] + b * xr;
    oim[e] = aim[e] + b * xi;
  }
}

// R <- R + R^T on 32 x 32 tile pairs (I <= J).
__global__ void symmetrize_kernel(double* R, int64_t n) {
  __shared__ double t1[32][33];
  __shared__ double t2[32][33];
  const int64_t T = (n + 31) / 32;
  const int64_t pairs = T * (T + 1) / 2;
  for (int64_t blk = blockIdx.x; blk < pairs; blk += gridDim.x) {
    // Map blk -> (I, J), I <= J, row-major over the upper triangle.
    int64_t I = static_cast<int64_t>((2.0 * T + 1.0 - sqrt((2.0 * T + 1.0) * (2.0 * T + 1.0) - 8.0 * blk)) / 2.0);
    if (I < 0) I = 0;
    while (I > 0 && I * T - I * (I - 1) / 2 > blk) --I;
    while ((I + 1) * T - (I + 1) * I / 2 <= blk) ++I;
    const int64_t J = I + (blk - (I * T - I * (I - 1) / 2));
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t rr = I * 32 + r, cc = J * 32 + threadIdx.x;
      t1[r][threadIdx.x] = (rr < n && cc < n) ? R[rr * n + cc] : 0.0;
      const int64_t rr2 = J * 32 + r, cc2 = I * 32 + threadIdx.x;
      t2[r][threadIdx.x] = (rr2 < n && cc2 < n) ? R[rr2 * n + cc2] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t rr = I * 32 + r, cc = J * 32 + threadIdx.x;
      // element (rr, cc) of block (I,J) pairs with element (cc, rr) of block (J,I)
      const double s = t1[r][threadIdx.x] + t2[threadIdx.x][r];
      if (rr < n && cc < n) R[rr * n + cc] = s;
      const int64_t rr2 = J * 32 + r, cc2 = I * 32 + threadIdx.x;
      const double s2 = t2[r][threadIdx.x] + t1[threadIdx.x][r];
      if (I != J && rr2 < n && cc2 < n) R[rr2 * n + cc2] = s2;
    }
    __syncthreads();
  }
}

__global__ void gather_vertex_kernel(double* out, const double* in, int cplx, int part,
                                     int64_t NG, int64_t Np, int64_t row0, int64_t nx,
                                     int64_t col0, int64_t ny) {
  __shared__ double tile[32][33];
  const int64_t tg = (NG + 31) / 32, tyn = (ny + 31) / 32;
  const int64_t total = tg * tyn * nx;
  const int64_t es = cplx ? 2 : 1;
  for (int64_t blk = blockIdx.x; blk < total; blk += gridDim.x) {
    const int64_t bg = blk % tg;
    const int64_t by = (blk / tg) % tyn;
    const int64_t x = blk / (tg * tyn);
    const int64_t p = row0 + x;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t y = by * 32 + r, g = bg * 32 + threadIdx.x;
      if (y < ny && g < NG) {
        const int64_t q = col0 + y;
        tile[r][threadIdx.x] = in[(g + NG * (p + Np * q)) * es + part];
      }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t g = bg * 32 + r, y = by * 32 + threadIdx.x;
      if (y < ny && g < NG) out[(g * nx + x) * ny + y] = tile[threadIdx.x][r];
    }
    __syncthreads();
  }
}

__global__ void scan_vertex_kernel(const double* p, int64_t n, int cplx, int* flags) {
  int f = 0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double x = p[e];
    if (!isfinite(x)) f |= 1;
    if (cplx && (e & 1) && x != 0.0) f |= 2;
  }
  f = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

struct JacobiArgs {
  double* Tnew; double* dT; const double* R; const double* Told;
  const double* eh; const double* ep;
  int64_t o, v, plane, total;
  double shift;
};

__global__ void jacobi_kernel(JacobiArgs a) {
  const int64_t n1 = a.v * a.o;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q = e % a.plane;
    double D;
    if (q < n1) {
      const int64_t ai = q;
      D = a.ep[ai / a.o] - a.eh[ai % a.o];
    } else {
      const int64_t r = q - n1;
      const int64_t ai = r / n1, bj = r - (r / n1) * n1;
      D = a.ep[ai / a.o] - a.eh[ai % a.o] + a.ep[bj / a.o] - a.eh[bj % a.o];
    }
    double rv = a.R[e];
    const double told = a.Told ? a.Told[e] : 0.0;
    if (a.Told && a.shift != 0.0) rv -= a.shift * told;
    const double tn = rv * (-1.0 / (D + a.shift));
    a.Tnew[e] = tn;
    a.dT[e] = a.Told ? tn - told : tn;
  }
}

struct EnergyArgs {
  const double* T; const double* Vdr; const double* Vdi; const double* Ver; const double* Vei;
  int64_t o, v, plane;
  int planes;
  double* ws;
};

__global__ void energy_kernel(EnergyArgs a) {
  const int64_t n1 = a.v * a.o;
  const int64_t n2 = n1 * n1;
  const double* t1r = a.T;
  const double* t2r = a.T + n1;
  const double* t1i = a.planes > 1 ? a.T + a.plane : nullptr;
  const double* t2i = a.planes > 1 ? a.T + a.plane + n1 : nullptr;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n2;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n1, c = e - (e / n1) * n1;
    // exchange element: Ve[e] or, without Ve, V_baij = Vd[(b,i),(a,j)] (coalesced in j)
    int64_t ex = e;
    if (!a.Ver) {
      const int64_t aa = r / a.o, i = r - aa * a.o, b = c / a.o, j = c - b * a.o;
      ex = (b * a.o + i) * n1 + aa * a.o + j;
    }
    const double* Ver = a.Ver ? a.Ver : a.Vdr;
    const double* Vei = a.Ver ? a.Vei : a.Vdi;
    if (!t1i) {
      const double x = t2r[e] + t1r[r] * t1r[c];
      acc[0] += x * a.Vdr[e];
      acc[1] += x * Ver[ex];
    } else {
      // X = T2 + T1 T1 (complex);  X * conj(V)
      const double xr = t2r[e] + t1r[r] * t1r[c] - t1i[r] * t1i[c];
      const double xi = t2i[e] + t1r[r] * t1i[c] + t1i[r] * t1r[c];
      const double vdr = a.Vdr[e], vdi = a.Vdi ? a.Vdi[e] : 0.0;
      const double ver = Ver[ex], vei = Vei ? Vei[ex] : 0.0;
      acc[0] += xr * vdr + xi * vdi;
      acc[1] += xr * ver + xi * vei;
      acc[2] += xi * vdr - xr * vdi;
      acc[3] += xi * ver - xr * vei;
    }
  }
  block_sum<4>(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) a.ws[blockIdx.x * 4 + k] = acc[k];
}

struct Mp2Args {
  const double* Vr;
  const double* Vi;
  const double* eh;
  const double* ep;
  int64_t o, v;
  double* ws;
};

// Per-block partial sums of Re(conj(V_abij) V_abij) / D and Re(conj(V_abij) V_abji) / D
// over the pair layout [a][i][b][j]; V_abji = V[(a,j),(b,i)].
__global__ void mp2_energy_kernel(Mp2Args a) {
  const int64_t n1 = a.v * a.o, n2 = n1 * n1;
  double acc[2] = {0.0, 0.0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n2;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n1, c = e - r * n1;
    const int64_t aa = r / a.o, i = r - aa * a.o, b = c / a.o, j = c - b * a.o;
    const double d = a.eh[i] + a.eh[j] - a.ep[aa] - a.ep[b];
    const int64_t ex = (aa * a.o + j) * n1 + b * a.o + i;
    const double vr = a.Vr[e], xr = a.Vr[ex];
    const double vi = a.Vi ? a.Vi[e] : 0.0, xi = a.Vi ? a.Vi[ex] : 0.0;
    acc[0] += (vr * vr + vi * vi) / d;
    acc[1] += (vr * xr + vi * xi) / d;
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < 2; ++k) a.ws[blockIdx.x * 2 + k] = acc[k];
}

// Fixed-order sum of per-block partials: dst[k] = scale[k] * sum_b ws[b*nvals + k].
__global__ void finish_kernel(double* dst, const double* ws, int nparts, int nvals,
                              double s0, double s1, double s2, double s3) {
  const double sc[4] = {s0, s1, s2, s3};
  for (int k = 0; k < nvals; ++k) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) v += ws[b * nvals + k];
    double arr[1] = {v};
    block_sum<1>(arr);
    if (threadIdx.x == 0) dst[k] = (k < 4 ? sc[k] : 1.0) * arr[0];
    __syncthreads();
  }
}

struct DotArgs {
  const double* x;
  const double* y[8];
  int ny;
  int64_t n;
  double* ws;
};

__global__ void dots_kernel(DotArgs a) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double xv = a.x[e];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < a.ny) acc[k] += xv * a.y[k][e];
  }
  block_sum<8>(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < a.ny; ++k) a.ws[blockIdx.x * a.ny + k] = acc[k];
}

struct LinArgs {
  double* out;
  const double* x[16];
  const double* y[16];
  const double* coef;
  int nx;
  int64_t n;
  double* ws;
};

__global__ void lincomb_kernel(LinArgs a) {
  double c[16];
  for (int k = 0; k < 16; ++k) c[k] = k < a.nx ? a.coef[k] : 0.0;
  double nrm[1] = {0.0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v = 0.0, w = 0.0;
    for (int k = 0; k < a.nx; ++k) {
      v += c[k] * a.x[k][e];
      if (a.y[0]) w += c[k] * a.y[k][e];
    }
    a.out[e] = v;
    nrm[0] += w * w;
  }
  if (a.ws) {
    block_sum<1>(nrm);
    if (threadIdx.x == 0) a.ws[blockIdx.x] = nrm[0];
  }
}

// ---- packed amplitude vectors ----------------------------------------------
// Per plane a packed vector holds T1 (n1 values) and then, for each row r of
// the symmetric T2 pair matrix, its columns r..n1-1; row r starts at
// n1 + tri_off(r, n1).
__device__ __forceinline__ int64_t tri_off(int64_t r, int64_t n) {
  return r * n - r * (r - 1) / 2;
}

struct PackedJacobiArgs {
  double* Tnew; double* dT; const double* R; const double* Told;
  const double* eh; const double* ep;
  int64_t o, v, plane, pplane, items;  // items = planes * (n1 + 1): T1, then T2 rows
  double shift;
};

// Same arithmetic as jacobi_kernel, element by element, on the upper triangle.
__global__ void jacobi_packed_kernel(PackedJacobiArgs a) {
  const int64_t n1 = a.v * a.o;
  for (int64_t it = blockIdx.x; it < a.items; it += gridDim.x) {
    const int64_t pl = it / (n1 + 1), w = it - pl * (n1 + 1);
    const double* R = a.R + pl * a.plane;
    const double* To = a.Told ? a.Told + pl * a.plane : nullptr;
    double* Tn = a.Tnew + pl * a.pplane;
    double* dT = a.dT + pl * a.pplane;
    if (w == 0) {
      for (int64_t ai = threadIdx.x; ai < n1; ai += blockDim.x) {
        const double D = a.ep[ai / a.o] - a.eh[ai % a.o];
        double rv = R[ai];
        const double told = To ? To[ai] : 0.0;
        if (To && a.shift != 0.0) rv -= a.shift * told;
        const double tn = rv * (-1.0 / (D + a.shift));
        Tn[ai] = tn;
        dT[ai] = To ? tn - told : tn;
      }
      continue;
    }
    const int64_t r = w - 1;
    const double Dr = a.ep[r / a.o] - a.eh[r % a.o];
    const double* Rr = R + n1 + r * n1;
    const double* Tr = To ? To + n1 + r * n1 : nullptr;
    const int64_t po = n1 + tri_off(r, n1) - r;  // packed index of column c is po + c
    for (int64_t c = r + threadIdx.x; c < n1; c += blockDim.x) {
      const double D = Dr + a.ep[c / a.o] - a.eh[c % a.o];
      double rv = Rr[c];
      const double told = Tr ? Tr[c] : 0.0;
      if (Tr && a.shift != 0.0) rv -= a.shift * told;
      const double tn = rv * (-1.0 / (D + a.shift));
      Tn[po + c] = tn;
      dT[po + c] = Tr ? tn - told : tn;
    }
  }
}

struct PackedDotArgs {
  const double* x;
  const double* y[8];
  int ny;
  int64_t n1, pplane, items;  // items = planes * (n1 + 1)
  double* ws;
};

// Weighted dots: off-diagonal T2 entries stand for two elements of the full vector.
__global__ void dots_packed_kernel(PackedDotArgs a) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t it = blockIdx.x; it < a.items; it += gridDim.x) {
    const int64_t pl = it / (a.n1 + 1), w = it - pl * (a.n1 + 1);
    const int64_t b = pl * a.pplane + (w == 0 ? 0 : a.n1 + tri_off(w - 1, a.n1));
    const int64_t len = w == 0 ? a.n1 : a.n1 - (w - 1);
    for (int64_t k = threadIdx.x; k < len; k += blockDim.x) {
      const double wt = (w == 0 || k == 0) ? 1.0 : 2.0;
      const double xv = wt * a.x[b + k];
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q < a.ny) acc[q] += xv * a.y[q][b + k];
    }
  }
  block_sum<8>(acc);
  if (threadIdx.x == 0)
    for (int q = 0; q < a.ny; ++q) a.ws[blockIdx.x * a.ny + q] = acc[q];
}

struct PackedLinArgs {
  double* out;
  const double* x[16];
  const double* y[16];
  const double* coef;
  int nx;
  int64_t n1, plane, pplane, nT, items;  // nT = ceil(n1 / 32); items = planes * (1 + tiles)
  double* ws;
};

// out (full) = sum_j coef[j] x_j on 32 x 32 tiles (I, J), I <= J, of the upper
// triangle; each tile is written in place and, through shared memory, mirrored.
__global__ void lincomb_packed_kernel(PackedLinArgs a) {
  __shared__ double tile[32][33];
  double c[16];
  for (int k = 0; k < 16; ++k) c[k] = k < a.nx ? a.coef[k] : 0.0;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t n1 = a.n1, nT = a.nT;
  const int64_t per = 1 + nT * (nT + 1) / 2;
  double nrm[1] = {0.0};
  for (int64_t it = blockIdx.x; it < a.items; it += gridDim.x) {
    const int64_t pl = it / per, w = it - pl * per;
    const int64_t pb = pl * a.pplane;
    double* ob = a.out + pl * a.plane;
    if (w == 0) {
      for (int64_t e = threadIdx.x; e < n1; e += blockDim.x) {
        double v = 0.0, u = 0.0;
        for (int k = 0; k < a.nx; ++k) {
          v += c[k] * a.x[k][pb + e];
          if (a.y[0]) u += c[k] * a.y[k][pb + e];
        }
        ob[e] = v;
        nrm[0] += u * u;
      }
      continue;
    }
    // tile t -> (I, J): row I of tiles holds nT - I tiles
    const int64_t t = w - 1;
    int64_t I = static_cast<int64_t>(
        (2.0 * nT + 1.0 - sqrt((2.0 * nT + 1.0) * (2.0 * nT + 1.0) - 8.0 * t)) / 2.0);
    if (I < 0) I = 0;
    while (I > 0 && tri_off(I, nT) > t) --I;
    while (I + 1 < nT && tri_off(I + 1, nT) <= t) ++I;
    const int64_t J = I + (t - tri_off(I, nT));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t r = I * 32 + ty + 8 * q, cc = J * 32 + tx;
      double v = 0.0;
      if (r < n1 && cc < n1 && cc >= r) {
        const int64_t pidx = pb + n1 + tri_off(r, n1) + (cc - r);
        double u = 0.0;
        for (int k = 0; k < a.nx; ++k) {
          v += c[k] * a.x[k][pidx];
          if (a.y[0]) u += c[k] * a.y[k][pidx];
        }
        ob[n1 + r * n1 + cc] = v;
        nrm[0] += (cc == r ? 1.0 : 2.0) * u * u;
      }
      tile[ty + 8 * q][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // element (rr, cc) of the lower triangle = (cc, rr)
      const int64_t rr = J * 32 + ty + 8 * q, cc = I * 32 + tx;
      if (rr < n1 && cc < n1 && rr > cc) ob[n1 + rr * n1 + cc] = tile[tx][ty + 8 * q];
    }
    __syncthreads();
  }
  if (a.ws) {
    block_sum<1>(nrm);
    if (threadIdx.x == 0) a.ws[blockIdx.x] = nrm[0];
  }
}

struct DiisArgs {
  double* B;
  const double* dots;
  int valid[16];
  int N, next, count;
  double* coef;
  int* status;
};

// Single-thread bordered DIIS solve with partial-pivoting LU (dim <= 17).
__global__ void diis_solve_kernel(DiisArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int M = a.N + 1;
  int di = 0;
  for (int i = 0; i < a.N; ++i) {
    if (!a.valid[i]) continue;
    const double ov = 2.0 * a.dots[di++];
    a.B[(i + 1) * M + (a.next + 1)] = ov;
    a.B[(a.next + 1) * M + (i + 1)] = ov;
  }
  const int dim = a.count + 1;
  double m[17][17];
  double x[17];
  for (int r = 0; r < dim; ++r) {
    for (int c = 0; c < dim; ++c) m[r][c] = a.B[r * M + c];
    x[r] = r == 0 ? -1.0 : 0.0;
  }
  int singular = 0;
  for (int k = 0; k < dim; ++k) {
    int piv = k;
    double best = fabs(m[k][k]);
    for (int r = k + 1; r < dim; ++r)
      if (fabs(m[r][k]) > best) { best = fabs(m[r][k]); piv = r; }
    if (!isfinite(best)) { singular = 2; break; }
    if (best == 0.0) { singular = 1; break; }
    if (piv != k) {
      for (int c = 0; c < dim; ++c) { double t = m[k][c]; m[k][c] = m[piv][c]; m[piv][c] = t; }
      double t = x[k]; x[k] = x[piv]; x[piv] = t;
    }
    for (int r = k + 1; r < dim; ++r) {
      const double f = m[r][k] / m[k][k];
      for (int c = k; c < dim; ++c) m[r][c] -= f * m[k][c];
      x[r] -= f * x[k];
    }
  }
  if (!singular) {
    for (int k = dim - 1; k >= 0; --k) {
      double s = x[k];
      for (int c = k + 1; c < dim; ++c) s -= m[k][c] * x[c];
      x[k] = s / m[k][k];
    }
    for (int j = 0; j < a.count; ++j) {
      const int slot = (a.next + a.N - j) % a.N;
      a.coef[j] = x[slot + 1];
    }
  }
  a.status[0] = singular;
}

}  // namespace

// ---------------------------------------------------------------------------
double* alloc(size_t elems) {
  void* p = nullptr;
  if (elems == 0) elems = 1;
  cudaError_t e = cudaMalloc(&p, elems * sizeof(double));
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(elems * 8) +
                                       " bytes failed: " + cudaGetErrorString(e));
  }
  return static_cast<double*>(p);
}
void release(void* p) {
  if (p) cudaFree(p);
}
void zero(double* p, size_t elems, Stream s) {
  CC_CHECK(cudaMemsetAsync(p, 0, elems * sizeof(double), s));
}
void h2d(double* d, const double* h, size_t elems, Stream s) {
  CC_CHECK(cudaMemcpyAsync(d, h, elems * sizeof(double), cudaMemcpyHostToDevice, s));
}
void d2h(double* h, const double* d, size_t elems, Stream s) {
  CC_CHECK(cudaMemcpyAsync(h, d, elems * sizeof(double), cudaMemcpyDeviceToHost, s));
}
void d2d(double* d, const double* src, size_t elems, Stream s) {
  CC_CHECK(cudaMemcpyAsync(d, src, elems * sizeof(double), cudaMemcpyDeviceToDevice, s));
}
void sync(Stream s) { CC_CHECK(cudaStreamSynchronize(s)); }
Stream stream_create(int device) {
  CC_CHECK(cudaSetDevice(device));
  cudaStream_t s;
  CC_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}
void stream_destroy(Stream s) {
  if (s) cudaStreamDestroy(s);
}
void* event_create() {
  cudaEvent_t e;
  CC_CHECK(cudaEventCreate(&e));
  return e;
}
void event_record(void* e, Stream s) { CC_CHECK(cudaEventRecord(static_cast<cudaEvent_t>(e), s)); }
float event_ms(void* a, void* b) {
  CC_CHECK(cudaEventSynchronize(static_cast<cudaEvent_t>(b)));
  float ms = 0.f;
  CC_CHECK(cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(a), static_cast<cudaEvent_t>(b)));
  return ms;
}
void event_destroy(void* e) {
  if (e) cudaEventDestroy(static_cast<cudaEvent_t>(e));
}

uint64_t launch_count() { return g_launches.load(); }

void permute4(double* dst, const double* src, const int64_t d[4], const int perm[4],
              double alpha, double beta, Stream s) {
  int64_t sstr[4];
  sstr[3] = 1;
  for (int k = 2; k >= 0; --k) sstr[k] = sstr[k + 1] * d[k + 1];
  Perm4 p;
  for (int k = 0; k < 4; ++k) {
    p.e[k] = d[perm[k]];
    p.ss[k] = sstr[perm[k]];
  }
  p.ds[3] = 1;
  for (int k = 2; k >= 0; --k) p.ds[k] = p.ds[k + 1] * p.e[k + 1];
  const int64_t total = p.e[0] * p.e[1] * p.e[2] * p.e[3];
  if (total == 0) return;
  if (perm[3] == 3) {
    const int64_t rows = p.e[0] * p.e[1] * p.e[2];
    int threads = p.e[3] >= 256 ? 256 : (p.e[3] >= 128 ? 128 : (p.e[3] >= 64 ? 64 : 32));
    permute_rows_kernel<<<grid_for(rows, 1, 148 * 64), threads, 0, s>>>(dst, src, p, alpha, beta);
  } else {
    int q = 0;
    for (int k = 0; k < 4; ++k)
      if (perm[k] == 3) q = k;
    int b[2], nb = 0;
    for (int k = 0; k < 3; ++k)
      if (k != q) b[nb++] = k;
    const int64_t tiles = ((p.e[3] + 31) / 32) * ((p.e[q] + 31) / 32) * p.e[b[0]] * p.e[b[1]];
    permute_tiled_kernel<<<grid_for(tiles, 1, 148 * 64), dim3(32, 8), 0, s>>>(
        dst, src, p, q, b[0], b[1], alpha, beta);
  }
  CC_LAUNCH_CHECK();
  count();
}

void copy4(double* dst, const int64_t ds[4], const double* src, const int64_t ss[4],
           const int64_t e[4], double alpha, double beta, Stream s) {
  if (ds[3] != 1) throw Error(ERR_STATE, "copy4: the destination's inner stride must be 1");
  Perm4 p;
  for (int k = 0; k < 4; ++k) { p.e[k] = e[k]; p.ss[k] = ss[k]; p.ds[k] = ds[k]; }
  const int64_t total = e[0] * e[1] * e[2] * e[3];
  if (total == 0) return;
  if (ss[3] == 1) {
    const int64_t rows = e[0] * e[1] * e[2];
    int threads = e[3] >= 256 ? 256 : (e[3] >= 128 ? 128 : (e[3] >= 64 ? 64 : 32));
    permute_rows_kernel<<<grid_for(rows, 1, 148 * 64), threads, 0, s>>>(dst, src, p, alpha, beta);
  } else {
    int q = 0;  // the destination axis with the smallest source stride
    for (int k = 1; k < 3; ++k)
      if (ss[k] < ss[q]) q = k;
    int b[2], nb = 0;
    for (int k = 0; k < 3; ++k)
      if (k != q) b[nb++] = k;
    const int64_t tiles = ((e[3] + 31) / 32) * ((e[q] + 31) / 32) * e[b[0]] * e[b[1]];
    permute_tiled_kernel<<<grid_for(tiles, 1, 148 * 64), dim3(32, 8), 0, s>>>(
        dst, src, p, q, b[0], b[1], alpha, beta);
  }
  CC_LAUNCH_CHECK();
  count();
}

void axpby(double* out, double a, const double* x, double b, const double* y, double c,
           int64_t n, Stream s) {
  if (n <= 0) return;
  axpby_kernel<<<grid_for(n, 256), 256, 0, s>>>(out, a, x, b, y, c, n);
  CC_LAUNCH_CHECK();
  count();
}

void rank1(double* out, double a, const double* A, double b, const double* t, int64_t n,
           Stream s) {
  if (n <= 0) return;
  rank1_kernel<<<grid_for(n * n, 256), 256, 0, s>>>(out, a, A, b, t, n);
  CC_LAUNCH_CHECK();
  count();
}

void zrank1(double* out_re, double* out_im, const double* A_re, const double* A_im,
            const double* t_re, const double* t_im, double b, int64_t n, Stream s) {
  if (n <= 0) return;
  zrank1_kernel<<<grid_for(n * n, 256), 256, 0, s>>>(out_re, out_im, A_re, A_im, t_re, t_im, b, n);
  CC_LAUNCH_CHECK();
  count();
}

void symmetrize(double* R, int64_t n, Stream s) {
  if (n <= 0) return;
  const int64_t T = (n + 31) / 32;
  symmetrize_kernel<<<grid_for(T * (T + 1) / 2, 1, 148 * 64), dim3(32, 8), 0, s>>>(R, n);
  CC_LAUNCH_CHECK();
  count();
}

void gather_vertex(double* out, const double* in, bool in_complex, int part, int64_t NG,
                   int64_t Np, int64_t row0, int64_t nx, int64_t col0, int64_t ny, Stream s) {
  if (NG <= 0 || nx <= 0 || ny <= 0) return;
  const int64_t tiles = ((NG + 31) / 32) * ((ny + 31) / 32) * nx;
  gather_vertex_kernel<<<grid_for(tiles, 1, 148 * 64), dim3(32, 8), 0, s>>>(
      out, in, in_complex ? 1 : 0, part, NG, Np, row0, nx, col0, ny);
  CC_LAUNCH_CHECK();
  count();
}

void jacobi(double* Tnew, double* dT, const double* R, const double* Told, const double* eh,
            const double* ep, const AmpShape& sh, double shift, Stream s) {
  JacobiArgs a{Tnew, dT, R, Told, eh, ep, sh.o, sh.v, sh.plane(), sh.total(), shift};
  jacobi_kernel<<<grid_for(sh.total(), 256), 256, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
}

int scan_vertex(const double* p, int64_t n, bool complex_values, Stream s) {
  int* flags = reinterpret_cast<int*>(alloc(1));
  int h = 0;
  try {
    CC_CHECK(cudaMemsetAsync(flags, 0, sizeof(int), s));
    scan_vertex_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n, complex_values ? 1 : 0, flags);
    CC_LAUNCH_CHECK();
    count();
    CC_CHECK(cudaMemcpyAsync(&h, flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    CC_CHECK(cudaStreamSynchronize(s));
  } catch (...) {
    release(flags);
    throw;
  }
  release(flags);
  return h;
}

void sum_partials_to(double* dst_dev, const double* ws, int nparts, int nvals, Stream s) {
  finish_kernel<<<1, 256, 0, s>>>(dst_dev, ws, nparts, nvals, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
}

void jacobi_packed(double* Tnew_p, double* dT_p, const double* R, const double* Told,
                   const double* eh, const double* ep, const AmpShape& sh, double shift,
                   Stream s) {
  PackedJacobiArgs a{Tnew_p, dT_p, R, Told, eh, ep, sh.o, sh.v, sh.plane(), sh.packed_plane(),
                     sh.planes * (sh.n1() + 1), shift};
  jacobi_packed_kernel<<<grid_for(a.items, 1, 148 * 16), 256, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
}

void dots_packed(const double* x, const double* const* ys, int ny, const AmpShape& sh,
                 double* out_dev, double* ws, Stream s) {
  if (ny <= 0) return;
  if (ny > 8) throw Error(ERR_UNSUPPORTED, "dots: at most 8 vectors");
  PackedDotArgs a{};
  a.x = x; a.ny = ny; a.n1 = sh.n1(); a.pplane = sh.packed_plane();
  a.items = sh.planes * (sh.n1() + 1); a.ws = ws;
  for (int k = 0; k < ny; ++k) a.y[k] = ys[k];
  dots_packed_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, ny, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
  count();
}

void lincomb_packed(double* out, const double* const* xs, const double* const* ys,
                    const double* coef_dev, int nx, const AmpShape& sh, double* norm2_dev,
                    double* ws, Stream s) {
  if (nx > 16) throw Error(ERR_UNSUPPORTED, "lincomb: at most 16 vectors");
  PackedLinArgs a{};
  a.out = out; a.coef = coef_dev; a.nx = nx;
  a.n1 = sh.n1(); a.plane = sh.plane(); a.pplane = sh.packed_plane();
  a.nT = (sh.n1() + 31) / 32;
  a.items = sh.planes * (1 + a.nT * (a.nT + 1) / 2);
  a.ws = (ys && norm2_dev) ? ws : nullptr;
  for (int k = 0; k < nx; ++k) {
    a.x[k] = xs[k];
    a.y[k] = ys ? ys[k] : nullptr;
  }
  lincomb_packed_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
  if (a.ws) {
    finish_kernel<<<1, 256, 0, s>>>(norm2_dev, ws, RED_BLOCKS, 1, 1.0, 1.0, 1.0, 1.0);
    CC_LAUNCH_CHECK();
    count();
  }
}

void energy(const double* T, const double* Vd_re, const double* Vd_im, const double* Ve_re,
            const double* Ve_im, const AmpShape& sh, double* out_dev, double* ws, Stream s) {
  EnergyArgs a{T, Vd_re, Vd_im, Ve_re, Ve_im, sh.o, sh.v, sh.plane(), (int)sh.planes, ws};
  energy_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  // direct = 2 * sum X V_ijab, exchange = -sum X V_ijba  (CoupledCluster.cxx:223-232)
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, 4, 2.0, -1.0, 2.0, -1.0);
  CC_LAUNCH_CHECK();
  count();
  count();
}

void mp2_energy(const double* Vd_re, const double* Vd_im, const double* eh, const double* ep,
                int64_t o, int64_t v, double* out_dev, double* ws, Stream s) {
  Mp2Args a{Vd_re, Vd_im, eh, ep, o, v, ws};
  mp2_energy_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, 2, 2.0, -1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
  count();
}

void dots(const double* x, const double* const* ys, int ny, int64_t n, double* out_dev,
          double* ws, Stream s) {
  if (ny <= 0) return;
  if (ny > 8) throw Error(ERR_UNSUPPORTED, "dots: at most 8 vectors");
  DotArgs a{};
  a.x = x; a.ny = ny; a.n = n; a.ws = ws;
  for (int k = 0; k < ny; ++k) a.y[k] = ys[k];
  dots_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, ny, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
  count();
}

void diis_solve(double* B, const double* dots_dev, const int* valid_host, int N, int next,
                int count_, double* coef_dev, int* status_dev, Stream s) {
  if (N > 16) throw Error(ERR_UNSUPPORTED, "DIIS: at most 16 residua");
  DiisArgs a{};
  a.B = B; a.dots = dots_dev; a.N = N; a.next = next; a.count = count_;
  a.coef = coef_dev; a.status = status_dev;
  for (int i = 0; i < N; ++i) a.valid[i] = valid_host[i];
  diis_solve_kernel<<<1, 32, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
}

void lincomb(double* out, const double* const* xs, const double* const* ys,
             const double* coef_dev, int nx, int64_t n, double* norm2_dev, double* ws,
             Stream s) {
  if (nx > 16) throw Error(ERR_UNSUPPORTED, "lincomb: at most 16 vectors");
  LinArgs a{};
  a.out = out; a.coef = coef_dev; a.nx = nx; a.n = n;
  a.ws = (ys && norm2_dev) ? ws : nullptr;
  for (int k = 0; k < nx; ++k) {
    a.x[k] = xs[k];
    a.y[k] = ys ? ys[k] : nullptr;
  }
  lincomb_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
  if (a.ws) {
    finish_kernel<<<1, 256, 0, s>>>(norm2_dev, ws, RED_BLOCKS, 1, 1.0, 1.0, 1.0, 1.0);
    CC_LAUNCH_CHECK();
    count();
  }
}


// ---------------------------------------------------------------------------
// Finite-size correction: planar singular vectors, the stacked-to-complex fold
// of the real path, the lattice box of S(G) and the two energy sums.
__global__ void fsc_prepare_u_kernel(double* ore, double* oim, const double* U, const double* V,
                                     int64_t NGG, int64_t NF) {
  const int64_t total = NGG * NF;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t F = e / NGG, G = e - F * NGG;  // reads along the caller's G-fastest layout
    double re, im;
    if (U) {
      re = U[2 * e];
      im = U[2 * e + 1];
    } else {
      re = G == F ? 1.0 : 0.0;
      im = 0.0;
    }
    const double sc = V ? 1.0 / sqrt(V[G]) : 1.0;
    ore[G * NF + F] = re * sc;
    oim[G * NF + F] = im * sc;
  }
}

__global__ void fsc_stacked_kernel(double* Qr, double* Qi, const double* Qs, int64_t NF,
                                   int parts) {
  const int64_t total = NF * NF, S2 = parts * NF;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t F = e / NF, Fp = e - F * NF;
    if (parts == 2) {
      Qr[e] = Qs[F * S2 + Fp] + Qs[(F + NF) * S2 + Fp + NF];
      Qi[e] = Qs[F * S2 + Fp + NF] - Qs[(F + NF) * S2 + Fp];
    } else {
      Qr[e] = Qs[e];
      Qi[e] = 0.0;
    }
  }
}

__device__ __forceinline__ void fsc_direct(const FscGeometry& g, const double v[3], double x[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) x[d] = g.A[3 * d] * v[0] + g.A[3 * d + 1] * v[1] + g.A[3 * d + 2] * v[2];
}

__global__ void fsc_box_kernel(double* box, const double* S, const double* grid, FscGeometry g) {
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < g.NG;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v[3] = {grid[3 * e], grid[3 * e + 1], grid[3 * e + 2]};
    double x[3];
    fsc_direct(g, v, x);
    int64_t i[3];
    bool in = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      i[d] = static_cast<int64_t>(floor(x[d] + 0.5) - g.origin[d]);
      in = in && i[d] >= 0 && i[d] < g.dims[d];  // the box was sized on the host: never write outside
    }
    if (in) box[i[0] + g.dims[0] * (i[1] + g.dims[1] * i[2])] = S[e];
  }
}

// Catmull-Rom tricubic value of the box at direct coordinates x (unit spacing):
// index truncated toward zero and clamped, 4 x 4 x 4 neighbourhood from one
// below it with clamped indices, weights BLEND (1, t, t^2, t^3).
__device__ double fsc_tricubic(const double* box, const FscGeometry& g, const double x[3]) {
  const double BLEND[4][4] = {{0.0, -0.5, 1.0, -0.5},
                              {1.0, 0.0, -2.5, 1.5},
                              {0.0, 0.5, 2.0, -1.5},
                              {0.0, 0.0, -0.5, 0.5}};
  double w[3][4];
  int64_t base[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double t = x[d] - g.origin[d];
    int64_t i = static_cast<int64_t>(t);
    i = i < 0 ? 0 : (i >= g.dims[d] ? g.dims[d] - 1 : i);
    const double u = t - static_cast<double>(i);
    const double pw[4] = {1.0, u, u * u, u * u * u};
#pragma unroll
    for (int r = 0; r < 4; ++r)
      w[d][r] = BLEND[r][0] * pw[0] + BLEND[r][1] * pw[1] + BLEND[r][2] * pw[2] + BLEND[r][3] * pw[3];
    base[d] = i - 1;
  }
  double total = 0.0;
  for (int sl = 0; sl < 4; ++sl) {
    int64_t z = base[2] + sl;
    z = z < 0 ? 0 : (z > g.dims[2] - 1 ? g.dims[2] - 1 : z);
    for (int r = 0; r < 4; ++r) {
      int64_t y = base[1] + r;
      y = y < 0 ? 0 : (y > g.dims[1] - 1 ? g.dims[1] - 1 : y);
      const double* row = box + g.dims[0] * (y + g.dims[1] * z);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        int64_t xx = base[0] + c;
        xx = xx < 0 ? 0 : (xx > g.dims[0] - 1 ? g.dims[0] - 1 : xx);
        total += w[0][c] * w[1][r] * w[2][sl] * row[xx];
      }
    }
  }
  return total;
}

__global__ void fsc_sums_kernel(const double* box, const double* S, const double* grid,
                                FscGeometry g, double* ws) {
  double acc[2] = {0.0, 0.0};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  for (int64_t e = first; e < g.NG; e += stride) {
    const double v0 = grid[3 * e], v1 = grid[3 * e + 1], v2 = grid[3 * e + 2];
    const double n2 = v0 * v0 + v1 * v1 + v2 * v2;
    if (sqrt(n2) >= 1e-8) acc[0] += g.f / n2 * S[e];
  }
  const int64_t n2N = 2 * static_cast<int64_t>(g.N);
  const int64_t total = n2N * n2N * n2N * g.NG;
  const double inv2N = 1.0 / static_cast<double>(n2N);
  for (int64_t e = first; e < total; e += stride) {
    const int64_t i = e % g.NG, abc = e / g.NG;
    const int64_t c = abc % n2N - g.N, b = (abc / n2N) % n2N - g.N, a = abc / (n2N * n2N) - g.N;
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double ga = g.B[d] * inv2N * static_cast<double>(a);
      const double gb = g.B[3 + d] * inv2N * static_cast<double>(b);
      const double gc = g.B[6 + d] * inv2N * static_cast<double>(c);
      v[d] = ga + gb + gc + grid[3 * i + d];
    }
    const double n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (sqrt(n2) < 1e-8) continue;
    double x[3];
    fsc_direct(g, v, x);
    acc[1] += g.f * fsc_tricubic(box, g, x) / n2;
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0) {
    ws[2 * blockIdx.x] = acc[0];
    ws[2 * blockIdx.x + 1] = acc[1];
  }
}

void fsc_prepare_u(double* out_re, double* out_im, const double* U, const double* V,
                   int64_t NGG, int64_t NF, Stream s) {
  fsc_prepare_u_kernel<<<grid_for(NGG * NF, 256, 148 * 16), 256, 0, s>>>(out_re, out_im, U, V, NGG,
                                                                          NF);
  CC_LAUNCH_CHECK();
  count();
}

void fsc_stacked_to_complex(double* Q_re, double* Q_im, const double* Qs, int64_t NF, int parts,
                            Stream s) {
  fsc_stacked_kernel<<<grid_for(NF * NF, 256, 148 * 16), 256, 0, s>>>(Q_re, Q_im, Qs, NF, parts);
  CC_LAUNCH_CHECK();
  count();
}

void fsc_box(double* box, const double* S, const double* grid, const FscGeometry& g, Stream s) {
  zero(box, static_cast<size_t>(g.dims[0] * g.dims[1] * g.dims[2]), s);
  fsc_box_kernel<<<grid_for(g.NG, 256, 148 * 4), 256, 0, s>>>(box, S, grid, g);
  CC_LAUNCH_CHECK();
  count();
}

void fsc_sums(const double* box, const double* S, const double* grid, const FscGeometry& g,
              double* ws, double* out_dev, Stream s) {
  fsc_sums_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(box, S, grid, g, ws);
  CC_LAUNCH_CHECK();
  count();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, 2, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
}

// ---------------------------------------------------------------------------
// Perturbative triples: the disconnected part of one block and the block's
// energy.  Elements run with q3 fastest, so the block array and the rows of
// the pair-layout integrals are read along their contiguous index; the hole
// permutations of the energy gather from the same (a, b, c) cube of the block.
struct TriplesArgs {
  const double* S;
  const double* Si;
  double* Sw;
  double* Swi;
  const double* t1;
  const double* t1i;
  const double* V;
  const double* Vi;
  const double* eh;
  const double* ep;
  int64_t o, n1, P1, P2, P3, L2, L3, total;
  double coef[6];
  double* ws;
  const double* M;   // cT branch: block array used in place of W = S - singles
  const double* Mi;
};

struct Cplx { double re, im; };

template <bool CPLX>
__device__ __forceinline__ Cplx triples_singles_at(const TriplesArgs& a, int64_t p1, int64_t p2,
                                                   int64_t p3) {
  const int64_t v23 = p2 * a.n1 + p3, v13 = p1 * a.n1 + p3, v12 = p1 * a.n1 + p2;
  if (!CPLX) {
    return {a.t1[p1] * a.V[v23] + a.t1[p2] * a.V[v13] + a.t1[p3] * a.V[v12], 0.0};
  }
  const double t1r = a.t1[p1], t1m = a.t1i[p1], t2r = a.t1[p2], t2m = a.t1i[p2];
  const double t3r = a.t1[p3], t3m = a.t1i[p3];
  const double v23r = a.V[v23], v23m = a.Vi[v23], v13r = a.V[v13], v13m = a.Vi[v13];
  const double v12r = a.V[v12], v12m = a.Vi[v12];
  return {t1r * v23r - t1m * v23m + t2r * v13r - t2m * v13m + t3r * v12r - t3m * v12m,
          t1r * v23m + t1m * v23r + t2r * v13m + t2m * v13r + t3r * v12m + t3m * v12r};
}

template <bool CPLX>
__global__ void triples_singles_kernel(TriplesArgs a) {
  const int64_t L23 = a.L2 * a.L3;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q1 = e / L23, r = e - q1 * L23, q2 = r / a.L3, q3 = r - q2 * a.L3;
    const Cplx x = triples_singles_at<CPLX>(a, a.P1 + q1, a.P2 + q2, a.P3 + q3);
    a.Sw[e] = x.re;
    if (CPLX) a.Swi[e] = x.im;
  }
}

template <bool CPLX>
__global__ void triples_energy_kernel(TriplesArgs a) {
  const int64_t L23 = a.L2 * a.L3, o = a.o;
  const int64_t X1 = a.P1 / o, X2 = a.P2 / o, X3 = a.P3 / o;
  double acc[2] = {0.0, 0.0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q1 = e / L23, r = e - q1 * L23, q2 = r / a.L3, q3 = r - q2 * a.L3;
    const int64_t x1 = q1 / o, x2 = q2 / o, x3 = q3 / o;
    const int64_t y0 = q1 - x1 * o, y1 = q2 - x2 * o, y2 = q3 - x3 * o;
    const Cplx sg = triples_singles_at<CPLX>(a, a.P1 + q1, a.P2 + q2, a.P3 + q3);
    const double d = a.eh[y0] + a.eh[y1] + a.eh[y2] - a.ep[X1 + x1] - a.ep[X2 + x2] -
                     a.ep[X3 + x3];
    const int64_t b1 = x1 * o * L23, b2 = x2 * o * a.L3, b3 = x3 * o;
    // the hole permutations 012, 021, 102, 120, 201, 210 of the pair (a, b, c)
    const int64_t idx[6] = {e,
                            b1 + y0 * L23 + b2 + y2 * a.L3 + b3 + y1,
                            b1 + y1 * L23 + b2 + y0 * a.L3 + b3 + y2,
                            b1 + y1 * L23 + b2 + y2 * a.L3 + b3 + y0,
                            b1 + y2 * L23 + b2 + y0 * a.L3 + b3 + y1,
                            b1 + y2 * L23 + b2 + y1 * a.L3 + b3 + y0};
    double yr = 0.0, yi = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (a.coef[k] == 0.0) continue;
      yr += a.coef[k] * a.S[idx[k]];
      if (CPLX) yi += a.coef[k] * a.Si[idx[k]];
    }
    const double inv = 1.0 / d;
    const double wr = a.M ? a.M[e] : a.S[e] - sg.re;
    acc[0] += wr * yr * inv;
    if (CPLX) acc[1] += (a.M ? a.Mi[e] : a.Si[e] - sg.im) * yi * inv;
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0) {
    a.ws[2 * blockIdx.x] = acc[0];
    a.ws[2 * blockIdx.x + 1] = acc[1];
  }
}

// The CR-(T) sums of one block triple: the element loop of triples_energy_kernel with
// y (amplitudes only) in place of W; `b2` is `a` with the pair-layout T2 in place of V.
template <bool CPLX>
__global__ void triples_cr_kernel(TriplesArgs a, TriplesArgs b2) {
  const int64_t L23 = a.L2 * a.L3, o = a.o;
  const int64_t X1 = a.P1 / o, X2 = a.P2 / o, X3 = a.P3 / o;
  double acc[2] = {0.0, 0.0};
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < a.total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t q1 = e / L23, r = e - q1 * L23, q2 = r / a.L3, q3 = r - q2 * a.L3;
    const int64_t x1 = q1 / o, x2 = q2 / o, x3 = q3 / o;
    const int64_t y0 = q1 - x1 * o, y1 = q2 - x2 * o, y2 = q3 - x3 * o;
    const int64_t p1 = a.P1 + q1, p2 = a.P2 + q2, p3 = a.P3 + q3;
    const Cplx ts = triples_singles_at<CPLX>(b2, p1, p2, p3);
    // t_ai t_bj t_ck
    const double r1 = a.t1[p1], r2 = a.t1[p2], r3 = a.t1[p3];
    const double i1 = CPLX ? a.t1i[p1] : 0.0, i2 = CPLX ? a.t1i[p2] : 0.0,
                 i3 = CPLX ? a.t1i[p3] : 0.0;
    const double pr = r1 * r2 - i1 * i2, pi = r1 * i2 + i1 * r2;
    const double yre = ts.re + pr * r3 - pi * i3, yim = ts.im + pr * i3 + pi * r3;
    const double d = a.eh[y0] + a.eh[y1] + a.eh[y2] - a.ep[X1 + x1] - a.ep[X2 + x2] -
                     a.ep[X3 + x3];
    const int64_t b1 = x1 * o * L23, bb2 = x2 * o * a.L3, b3 = x3 * o;
    const int64_t idx[6] = {e,
                            b1 + y0 * L23 + bb2 + y2 * a.L3 + b3 + y1,
                            b1 + y1 * L23 + bb2 + y0 * a.L3 + b3 + y2,
                            b1 + y1 * L23 + bb2 + y2 * a.L3 + b3 + y0,
                            b1 + y2 * L23 + bb2 + y0 * a.L3 + b3 + y1,
                            b1 + y2 * L23 + bb2 + y1 * a.L3 + b3 + y0};
    double zr = 0.0, zi = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (a.coef[k] == 0.0) continue;
      zr += a.coef[k] * a.S[idx[k]];
      if (CPLX) zi += a.coef[k] * a.Si[idx[k]];
    }
    const double inv = 1.0 / d;
    acc[0] += yre * zr * inv;
    if (CPLX) acc[1] += yim * zi * inv;
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0) {
    a.ws[2 * blockIdx.x] = acc[0];
    a.ws[2 * blockIdx.x + 1] = acc[1];
  }
}

TriplesArgs triples_args(const double* t1, const double* t1i, const double* V, const double* Vi,
                         const TriplesBlock& b) {
  TriplesArgs a{};
  a.t1 = t1; a.t1i = t1i; a.V = V; a.Vi = Vi; a.o = b.o; a.n1 = b.n1;
  a.P1 = b.P[0]; a.P2 = b.P[1]; a.P3 = b.P[2];
  a.L2 = b.L[1]; a.L3 = b.L[2];
  a.total = b.L[0] * b.L[1] * b.L[2];
  return a;
}

void triples_singles(double* S, double* S_im, const double* t1, const double* t1_im,
                     const double* V, const double* V_im, const TriplesBlock& b, Stream s) {
  TriplesArgs a = triples_args(t1, t1_im, V, V_im, b);
  a.Sw = S; a.Swi = S_im;
  if (a.total <= 0) return;
  const unsigned grid = grid_for(a.total, 256, 148 * 16);
  if (S_im)
    triples_singles_kernel<true><<<grid, 256, 0, s>>>(a);
  else
    triples_singles_kernel<false><<<grid, 256, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
}

void triples_energy(const double* S, const double* S_im, const double* t1, const double* t1_im,
                    const double* V, const double* V_im, const double* eps_h,
                    const double* eps_p, const TriplesBlock& b, const double coef[6],
                    double* ws, double* out_dev, Stream s, const double* M,
                    const double* M_im) {
  TriplesArgs a = triples_args(t1, t1_im, V, V_im, b);
  a.S = S; a.Si = S_im; a.eh = eps_h; a.ep = eps_p; a.ws = ws;
  a.M = M; a.Mi = M_im;
  for (int k = 0; k < 6; ++k) a.coef[k] = coef[k];
  if (S_im)
    triples_energy_kernel<true><<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  else
    triples_energy_kernel<false><<<RED_BLOCKS, RED_THREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  count();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, 2, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
}

void triples_cr_sums(const double* S, const double* S_im, const double* t1, const double* t1_im,
                     const double* T2, const double* T2_im, const double* eps_h,
                     const double* eps_p, const TriplesBlock& b, const double coef[6],
                     double* ws, double* out_dev, Stream s) {
  TriplesArgs a = triples_args(t1, t1_im, nullptr, nullptr, b);
  a.S = S; a.Si = S_im; a.eh = eps_h; a.ep = eps_p; a.ws = ws;
  for (int k = 0; k < 6; ++k) a.coef[k] = coef[k];
  TriplesArgs b2 = triples_args(t1, t1_im, T2, T2_im, b);
  if (S_im)
    triples_cr_kernel<true><<<RED_BLOCKS, RED_THREADS, 0, s>>>(a, b2);
  else
    triples_cr_kernel<false><<<RED_BLOCKS, RED_THREADS, 0, s>>>(a, b2);
  CC_LAUNCH_CHECK();
  count();
  finish_kernel<<<1, 256, 0, s>>>(out_dev, ws, RED_BLOCKS, 2, 1.0, 1.0, 1.0, 1.0);
  CC_LAUNCH_CHECK();
  count();
}

}  // namespace ops
}  // namespace cc4s_b200
