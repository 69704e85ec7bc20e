// Correlation energy of caller-supplied device amplitudes, without any device
// allocation (cc4s_cc_energy_noalloc in include/cc4s_cc.h).
//
// Some callers cannot allocate device memory at the point where they need an
// energy: host programs whose device memory is fully owned by their own pool
// (for example a framework allocator holding every byte it may use) and that
// must not see a hidden cudaMalloc, and loops that must not pay for the device
// synchronisation a cudaFree implies.  For them this entry point takes only
// device pointers the caller already owns and keeps its own temporary data in
// a file-scope device array of fixed size.
//
// The reduction is two-pass and deterministic: one partial sum per (i, j)
// pair of occupied orbitals (the array holds kMaxPairs of them, so No is at
// most 256), then one block adds the partials in a fixed order.  Nothing has
// to start at zero: the first kernel writes every partial sum the second one
// reads, and the second one writes all four outputs.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace cc4s_b200 {

namespace {

constexpr int64_t kMaxPairs = 65536;        // No * No <= 65536, i.e. No <= 256
constexpr int kVals = 4;                    // Re/Im of direct and exchange
// Partial sums of the reduction: 65536 * 4 doubles = 2 MiB, resident on every
// device that loads the library until the process exits.
__device__ __align__(256) double g_energy_scratch[kMaxPairs * kVals];

// Per-device address of g_energy_scratch.  It is looked up again on every call
// made outside stream capture (the lookup allocates nothing), so a device reset
// or another context on the same device never leaves a stale address here;
// calls made while the stream is being captured use the address of the last
// call outside capture on that device.
double* g_scratch_addr[64] = {nullptr};
std::mutex g_scratch_mutex;

// One block per (i, j): sums over a, b of X_abij (2 conj V_abij - ...) in the
// reference's column-major layout, X_abij = T2_abij + T1_ai T1_bj.
__global__ void energy_pairs_kernel(const double* T1, const double* T2, const double* V,
                                    int64_t o, int64_t v, int cplx, double* partial) {
  const int64_t ij = blockIdx.x;
  const int64_t i = ij % o, j = ij / o;
  double acc[kVals] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t ab = threadIdx.x; ab < v * v; ab += blockDim.x) {
    const int64_t a = ab % v, b = ab / v;
    const int64_t e = a + v * (b + v * (i + o * j));          // (a,b,i,j)
    const int64_t ex = b + v * (a + v * (i + o * j));         // (b,a,i,j)
    const int64_t ai = a + v * i, bj = b + v * j;
    if (!cplx) {
      const double x = T2[e] + T1[ai] * T1[bj];
      acc[0] += x * V[e];
      acc[1] += x * V[ex];
    } else {
      const double t1ar = T1[2 * ai], t1ai = T1[2 * ai + 1];
      const double t1br = T1[2 * bj], t1bi = T1[2 * bj + 1];
      const double xr = T2[2 * e] + t1ar * t1br - t1ai * t1bi;
      const double xi = T2[2 * e + 1] + t1ar * t1bi + t1ai * t1br;
      const double vdr = V[2 * e], vdi = V[2 * e + 1], ver = V[2 * ex], vei = V[2 * ex + 1];
      acc[0] += xr * vdr + xi * vdi;   // Re(X conj(V_abij))
      acc[1] += xr * ver + xi * vei;   // Re(X conj(V_baij))
      acc[2] += xi * vdr - xr * vdi;
      acc[3] += xi * ver - xr * vei;
    }
  }
  __shared__ double sh[kVals][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kVals; ++k) {
    double x = acc[k];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < kVals; ++k) {
      double x = threadIdx.x < nw ? sh[k][threadIdx.x] : 0.0;
      for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
      if (threadIdx.x == 0) partial[ij * kVals + k] = x;
    }
  }
}

// direct = 2 sum X conj(V_abij), exchange = -sum X conj(V_baij) (CoupledCluster.cxx:223-232)
__global__ void energy_finish_kernel(const double* partial, int64_t npairs, double* out) {
  __shared__ double sh[kVals][32];
  double acc[kVals] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t p = threadIdx.x; p < npairs; p += blockDim.x)
#pragma unroll
    for (int k = 0; k < kVals; ++k) acc[k] += partial[p * kVals + k];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kVals; ++k) {
    double x = acc[k];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) sh[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    double s[kVals] = {0.0, 0.0, 0.0, 0.0};
    for (int ww = 0; ww < nw; ++ww)
      for (int k = 0; k < kVals; ++k) s[k] += sh[k][ww];
    out[0] = 2.0 * s[0];
    out[1] = -s[1];
    out[2] = 2.0 * s[2];
    out[3] = -s[3];
  }
}

}  // namespace

// Returns 0 or a status code; message in *err.
int energy_noalloc(const double* T1, const double* T2, const double* V, int64_t No, int64_t Nv,
                   int is_complex, double* out, cudaStream_t stream, const char** err) {
  if (!T1 || !T2 || !V || !out) { *err = "null pointer"; return ERR_INVALID_ARGUMENT; }
  if (No <= 0 || Nv <= 0) { *err = "No and Nv must be positive"; return ERR_BAD_SHAPE; }
  if (No * No > kMaxPairs) {
    *err = "No * No exceeds the 65536 occupied pairs of the fixed scratch array (No <= 256)";
    return ERR_BAD_SHAPE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    *err = "no current CUDA device";
    return ERR_CUDA;
  }
  // An error left pending by the caller's earlier work is reported as such and
  // left in place for the caller; nothing is launched then.
  if (cudaPeekAtLastError() != cudaSuccess) {
    *err = "a CUDA error from earlier work is pending on this thread; nothing was launched";
    return ERR_CUDA;
  }
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess) {
    *err = "cudaStreamIsCapturing failed";
    return ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (capture == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_energy_scratch);
      if (e != cudaSuccess || !p) {
        *err = "cudaGetSymbolAddress of the energy scratch array failed";
        return ERR_CUDA;
      }
      g_scratch_addr[dev] = static_cast<double*>(p);
    } else if (!g_scratch_addr[dev]) {
      *err = "the first call on a device must come before any stream capture";
      return ERR_STATE;
    }
    scratch = g_scratch_addr[dev];
  }
  energy_pairs_kernel<<<static_cast<unsigned>(No * No), 256, 0, stream>>>(
      T1, T2, V, No, Nv, is_complex ? 1 : 0, scratch);
  energy_finish_kernel<<<1, 256, 0, stream>>>(scratch, No * No, out);
  // no error was pending before the launches, so this one is theirs
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return ERR_CUDA;
  }
  return OK;
}

}  // namespace cc4s_b200
