// Common helpers for the cc4s B200 CoupledCluster library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace cc4s_b200 {

// Status codes of the C ABI (mirrored in include/cc4s_cc.h).
enum Status : int {
  OK = 0,
  ERR_INVALID_ARGUMENT = 1,
  ERR_BAD_SHAPE = 2,
  ERR_OUT_OF_MEMORY = 3,
  ERR_NOT_CONVERGED = 4,   // a warning: results are valid
  ERR_DIIS_SINGULAR = 5,
  ERR_CUDA = 6,
  ERR_TIMEOUT = 7,
  ERR_STATE = 8,
  ERR_NON_FINITE = 9,
  ERR_UNSUPPORTED = 10,
};

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    int st = (e == cudaErrorMemoryAllocation) ? ERR_OUT_OF_MEMORY : ERR_CUDA;
    throw Error(st, std::string(what) + ": " + cudaGetErrorString(e) + " at " + file + ":" +
                        std::to_string(line));
  }
}

#define CC_CHECK(x) ::cc4s_b200::cuda_check((x), #x, __FILE__, __LINE__)
#define CC_LAUNCH_CHECK() ::cc4s_b200::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

inline unsigned grid_for(int64_t n, int threads, int64_t cap = 148 * 32) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return static_cast<unsigned>(b);
}

}  // namespace cc4s_b200
