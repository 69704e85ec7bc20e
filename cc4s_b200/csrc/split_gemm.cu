// Split-precision FP64 contraction: FP16 integer slices on tcgen05 tensor cores.
//
// Kernel layout (one 128 x 128 output tile per CTA, 320 threads):
//   warp 0      TMA producer: per k-block of 32, three A-slice and three
//               B-slice tiles (128 x 32 FP16, 64-byte swizzle) into a 4-stage
//               shared-memory ring, completion tracked by mbarriers;
//   warp 1      allocates 512 TMEM columns; one thread issues tcgen05.mma
//               (M=128, N=128, K=16) for the six slice products into three
//               FP32 accumulators (TMEM columns 0, 128, 256) and commits to
//               mbarriers that release smem stages and publish K chunks;
//   warps 2..9  epilogue: after each K chunk, tcgen05.ld the three groups and
//               add them into FP64 register accumulators (two warps per TMEM
//               lane quadrant, 64 columns each); after the last chunk, scale,
//               stage the tile in the idle stage buffers and store C once,
//               coalesced along the output's contiguous index.
// Every mbarrier wait is bounded; on expiry the kernel records an error flag
// and every role leaves its loop, so the kernel always terminates.
#include "split_gemm.cuh"

#include <cuda.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace cc4s_b200 {

namespace {

// Stage geometry.  Wide stages: k-blocks of 64 (128-byte rows, 128-byte swizzle),
// two 96 KB stages, half as many TMA row requests per byte as the narrow form
// (k-blocks of 32, 64-byte rows and swizzle, four 48 KB stages).
#ifndef CC4S_SPLIT_WIDE_STAGES
#define CC4S_SPLIT_WIDE_STAGES 0
#endif
#if CC4S_SPLIT_WIDE_STAGES
constexpr int TK = 64, NST = 2;
constexpr uint32_t ROW_BYTES = 128;               // smem row of one k-block (bytes)
#else
constexpr int TK = 32, NST = 4;
constexpr uint32_t ROW_BYTES = 64;
#endif
constexpr int TM = 128, TN = 128, NSLICE = 3;
constexpr int KCHUNK = 4096;                      // exact FP32 span of the leading group
constexpr int TILE_BYTES = TM * TK * 2;           // one slice tile: 8 KB (narrow), 16 KB (wide)
constexpr int STAGE_BYTES = 2 * NSLICE * TILE_BYTES;
constexpr int SMEM_BYTES = NST * STAGE_BYTES + 1024 + 256;
constexpr uint32_t WAIT_LIMIT = 1u << 28;         // bounded mbarrier waits
constexpr int64_t RASTER_M = 8;                  // tile rows per raster group

std::atomic<uint64_t> g_split_launches{0};
std::atomic<uint64_t> g_pack_launches{0};

struct Ax {
  uint32_t inner;
  int64_t s_o, s_i;
  __host__ __device__ __forceinline__ int64_t off(uint32_t x) const {
    const uint32_t o = x / inner;
    return static_cast<int64_t>(o) * s_o + static_cast<int64_t>(x - o * inner) * s_i;
  }
};
Ax mkax(int64_t inner, int64_t s_o, int64_t s_i) {
  Ax a; a.inner = static_cast<uint32_t>(inner > 0 ? inner : 1); a.s_o = s_o; a.s_i = s_i; return a;
}

// ---------------------------------------------------------------------------
// Packing: operand element (r, k) -> three FP16 integer slices P[q][r][k]
// (row-padded to Rp, k-padded to Kp) and a per-row exponent.
struct PackArgs {
  const double* src;
  Ax ar, ak;              // two-level index maps of the row and k indices
  int64_t R, K, Rp, Kp;
  unsigned long long* rmax;  // per-row max |x| as IEEE bits (non-negative doubles)
  int* rexp;              // per-row exponent
  __half* dst;            // [3][Rp][Kp]
  int r_contig;           // 1: the row index is the contiguous one in memory
};

// Packing works on tiles of 64 rows x 64 k staged in shared memory.  The row and
// k offsets of a tile are computed once per tile (two-level index maps need an
// integer division each), every thread keeps 16 loads in flight, and the FP16
// slices leave as 16-byte vector stores along k.
constexpr int PR = 64, PKT = 64, PTHREADS = 256, PSTRIP = 16;  // strip: k tiles per row max

struct PackTile {
  double v[PR][PKT + 1];
  int64_t roff[PR];
  int64_t koff[PKT];
};

// Loads the tile (r0, k0) of the operand into t.v (zero outside R x K).
__device__ __forceinline__ void pack_load_tile(const PackArgs& a, int64_t r0, int64_t k0,
                                               PackTile& t) {
  for (int q = threadIdx.x; q < PR + PKT; q += PTHREADS) {
    if (q < PR) {
      const int64_t r = r0 + q;
      t.roff[q] = r < a.R ? a.ar.off(static_cast<uint32_t>(r)) : -1;
    } else {
      const int64_t k = k0 + (q - PR);
      t.koff[q - PR] = k < a.K ? a.ak.off(static_cast<uint32_t>(k)) : -1;
    }
  }
  __syncthreads();
  const int lo = threadIdx.x & 63, hi = threadIdx.x >> 6;  // lanes along the contiguous index
  double x[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int rr = a.r_contig ? lo : hi + 4 * j;
    const int kk = a.r_contig ? hi + 4 * j : lo;
    const int64_t ro = t.roff[rr], ko = t.koff[kk];
    x[j] = (ro >= 0 && ko >= 0) ? a.src[ro + ko] : 0.0;
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int rr = a.r_contig ? lo : hi + 4 * j;
    const int kk = a.r_contig ? hi + 4 * j : lo;
    t.v[rr][kk] = x[j];
  }
  __syncthreads();
}

// Row maxima |x| over all k, as IEEE bits of non-negative doubles: each block
// walks PSTRIP k tiles of one row strip, one atomicMax per row and strip.
__global__ void __launch_bounds__(PTHREADS) pack_max_kernel(PackArgs a) {
  __shared__ PackTile t;
  const int64_t nr = a.Rp / PR, nks = (a.Kp + PKT * PSTRIP - 1) / (PKT * PSTRIP);
  const int row = threadIdx.x >> 2, part = threadIdx.x & 3;  // 4 threads per row, 16 k each
  for (int64_t w = blockIdx.x; w < nr * nks; w += gridDim.x) {
    const int64_t r0 = (w / nks) * PR, kbeg = (w % nks) * PKT * PSTRIP;
    double m = 0.0;
    for (int64_t k0 = kbeg; k0 < kbeg + PKT * PSTRIP && k0 < a.Kp; k0 += PKT) {
      pack_load_tile(a, r0, k0, t);
#pragma unroll
      for (int j = 0; j < 16; ++j) m = fmax(m, fabs(t.v[row][16 * part + j]));
      __syncthreads();
    }
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
    const int64_t r = r0 + row;
    if (part == 0 && r < a.R && m > 0.0)
      atomicMax(&a.rmax[r], static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// Three FP16 integer slices of every element (row-padded to Rp, k-padded to Kp)
// and the per-row exponent.
__global__ void __launch_bounds__(PTHREADS) pack_slices_kernel(PackArgs a) {
  __shared__ PackTile t;
  __shared__ int rexp_s[PR];
  const int64_t nr = a.Rp / PR, nk = (a.Kp + PKT - 1) / PKT;
  const int row = threadIdx.x >> 2, part = threadIdx.x & 3;
  const int64_t pl = a.Rp * a.Kp;
  for (int64_t w = blockIdx.x; w < nr * nk; w += gridDim.x) {
    const int64_t r0 = (w / nk) * PR, k0 = (w % nk) * PKT;
    if (threadIdx.x < PR) {
      const int64_t r = r0 + threadIdx.x;
      int e = 0;
      if (r < a.R) {
        const double m = __longlong_as_double(static_cast<long long>(a.rmax[r]));
        if (m > 0.0) frexp(m, &e);
        if (k0 == 0) a.rexp[r] = e;
      }
      rexp_s[threadIdx.x] = e;
    }
    pack_load_tile(a, r0, k0, t);   // its first barrier also publishes rexp_s
    const int64_t r = r0 + row, kb = k0 + 16 * part;
    if (kb < a.Kp) {
      const int e = rexp_s[row];
      __align__(16) __half h[3][16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        double x = ldexp(t.v[row][16 * part + j], -e) * 64.0;   // |x| <= 64
        const double s1 = rint(x);
        double u = (x - s1) * 2048.0;                            // |u| <= 1024
        const double s2 = rint(u);
        u = (u - s2) * 2048.0;
        const double s3 = rint(u);
        // integers of at most 11 bits: exact in FP32 and FP16
        h[0][j] = __float2half_rn(static_cast<float>(s1));
        h[1][j] = __float2half_rn(static_cast<float>(s2));
        h[2][j] = __float2half_rn(static_cast<float>(s3));
      }
      const int64_t o = r * a.Kp + kb;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        uint4* d = reinterpret_cast<uint4*>(a.dst + q * pl + o);
        const uint4* src = reinterpret_cast<const uint4*>(h[q]);
        d[0] = src[0];
        d[1] = src[1];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Device helpers (inline PTX for sm_100a).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar));
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}
// Bounded wait for the phase with the given parity: gives up after
// WAIT_LIMIT polls or 2 seconds, whichever comes first; returns false then.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    if (ok) return true;
    if ((it & 1023) == 1023 && global_ns() - t0 > 2000000000ull) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];\n"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}
// Shared-memory matrix descriptor: K-major, swizzled rows of ROW_BYTES (64 or 128),
// 8-row groups 8 * ROW_BYTES apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFF);        // start address
  d |= static_cast<uint64_t>(1) << 16;                       // leading byte offset (16 B)
  d |= static_cast<uint64_t>((8 * ROW_BYTES) >> 4) << 32;    // stride byte offset
  d |= static_cast<uint64_t>(1) << 46;                       // descriptor version (sm100)
  d |= static_cast<uint64_t>(ROW_BYTES == 128 ? 2 : 4) << 61;  // SWIZZLE_128B / SWIZZLE_64B
  return d;
}
// Instruction descriptors: D = F32, A = B = F16, both K-major, M = 128, N = 128 or 256.
constexpr uint32_t IDESC128 = (1u << 4) | ((TN >> 3) << 17) | ((TM >> 4) << 24);
constexpr uint32_t IDESC256 = (1u << 4) | (((2 * TN) >> 3) << 17) | ((TM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                     uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
               ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// 2^e as an exact double: built from its exponent bits in the normal range.
__device__ __forceinline__ double pow2i(int e) {
  if (e >= -1022 && e <= 1023) return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
  return ldexp(1.0, e);
}
// Accumulating store of NB output elements: every old value is loaded before the
// first store, so the NB reads are in flight together (a store followed by a load
// through another pointer would otherwise serialise them: the two may alias).
template <int NB>
__device__ __forceinline__ void rmw_store(double* const (&ptr)[NB], const double (&v)[NB],
                                          double beta) {
  if (beta != 0.0) {
    double old[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) old[j] = ptr[j] ? *ptr[j] : 0.0;
#pragma unroll
    for (int j = 0; j < NB; ++j)
      if (ptr[j]) *ptr[j] = v[j] + beta * old[j];
  } else {
#pragma unroll
    for (int j = 0; j < NB; ++j)
      if (ptr[j]) *ptr[j] = v[j];
  }
}

struct SplitParams {
  int64_t M, N, K;                 // logical extents
  int64_t Mp, Np;                  // padded row counts of the packed operands (slice strides)
  int nkb;                         // k-blocks of TK
  Ax Cm, Cn, C2m, C2n;
  double* C; double* C2;
  double alpha, beta;
  const int* ea; const int* eb;    // exponents of the packed rows of A and of B
  int* error;
  // Packed rows (persistent kernel): logical row m of A is packed row
  //   a_base + (m / a_run) * a_stride + m % a_run,
  // and tiles never straddle a run (a_tiles tiles per run, nMt tile rows in all);
  // likewise n for B.  One run over the whole extent is the plain case.
  int64_t a_run, a_stride, a_base, a_tiles, nMt;
  int64_t b_run, b_stride, b_base, b_tiles, nNt;
};

__global__ void __launch_bounds__(320)
split_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
             SplitParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers, then barriers
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NST * STAGE_BYTES);
  // bars[0..NST): full, [NST..2NST): empty, [2NST]: acc_full, [2NST+1]: acc_empty
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NST + 2);
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Tile order: groups of RASTER_M tile rows sweep the tile columns together, so
  // the CTAs resident at one time share a few A row tiles and reuse each B tile
  // RASTER_M times from L2 instead of streaming B from DRAM once per tile row.
  int64_t m0, n0;
  {
    const int64_t nM = p.Mp / TM, nN = p.Np / TN, b = blockIdx.x;
    const int64_t per_group = RASTER_M * nN, group = b / per_group;
    const int64_t first = group * RASTER_M;
    const int64_t rows = nM - first < RASTER_M ? nM - first : RASTER_M;
    const int64_t in = b - group * per_group;
    m0 = (first + in % rows) * TM;
    n0 = (in / rows) * TN;
  }
  const int nchunks = (p.nkb * TK + KCHUNK - 1) / KCHUNK;
  constexpr int KB_PER_CHUNK = KCHUNK / TK;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < NST; ++s) {
      mbar_init(smem_u32(&bars[s]), 1);
      mbar_init(smem_u32(&bars[NST + s]), 1);
    }
    mbar_init(smem_u32(&bars[2 * NST]), 1);
    mbar_init(smem_u32(&bars[2 * NST + 1]), 256);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_u32(tmem_slot)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    for (int kb = 0; kb < p.nkb; ++kb) {
      const int s = kb % NST;
      if (kb >= NST && !mbar_wait(smem_u32(&bars[NST + s]), ((kb / NST) - 1) & 1)) {
        atomicExch(&abort_flag, 1);
        break;
      }
      if (abort_flag) break;
      const uint32_t full = smem_u32(&bars[s]);
      mbar_expect_tx(full, STAGE_BYTES);
      unsigned char* st = base + s * STAGE_BYTES;
      for (int q = 0; q < NSLICE; ++q) {
        tma_load_2d(smem_u32(st + q * TILE_BYTES), &tmA, full, kb * TK, static_cast<int>(q * p.Mp + m0));
        tma_load_2d(smem_u32(st + (NSLICE + q) * TILE_BYTES), &tmB, full, kb * TK,
                    static_cast<int>(q * p.Np + n0));
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    int kb = 0;
    for (int c = 0; c < nchunks && !abort_flag; ++c) {
      if (c > 0 && !mbar_wait(smem_u32(&bars[2 * NST + 1]), (c - 1) & 1)) {
        atomicExch(&abort_flag, 1);
        break;
      }
      tc_fence_after();
      const int kb_end = min(p.nkb, (c + 1) * KB_PER_CHUNK);
      bool first = true;
      for (; kb < kb_end; ++kb) {
        const int s = kb % NST;
        if (!mbar_wait(smem_u32(&bars[s]), (kb / NST) & 1)) { atomicExch(&abort_flag, 1); break; }
        tc_fence_after();
        const uint32_t st = smem_u32(base + s * STAGE_BYTES);
#pragma unroll
        for (int kk = 0; kk < TK / 16; ++kk) {
          // 32 bytes per 16-element K step inside the swizzled rows
          const uint32_t koff = kk * 32;
          // Groups of equal weight live at TMEM columns 0 (S1S1), 128 (S1S2 + S2S1)
          // and 256 (S1S3 + S2S2 + S3S1).  B slices 1 and 2 are adjacent in shared
          // memory, so A_p x [B1 | B2] is one N = 256 MMA into groups p and p+1.
          const uint32_t init = (first && kk == 0) ? 0u : 1u;
          const uint64_t a1 = sdesc(st + 0 * TILE_BYTES + koff);
          const uint64_t a2 = sdesc(st + 1 * TILE_BYTES + koff);
          const uint64_t a3 = sdesc(st + 2 * TILE_BYTES + koff);
          const uint64_t b12 = sdesc(st + (NSLICE + 0) * TILE_BYTES + koff);
          const uint64_t b1 = b12;
          const uint64_t b3 = sdesc(st + (NSLICE + 2) * TILE_BYTES + koff);
          umma(tmem + 0 * TN, a1, b12, IDESC256, init);  // S1 x [S1|S2] -> groups 0, 1
          umma(tmem + 2 * TN, a1, b3, IDESC128, init);   // S1 x S3      -> group 2
          umma(tmem + 1 * TN, a2, b12, IDESC256, 1u);    // S2 x [S1|S2] -> groups 1, 2
          umma(tmem + 2 * TN, a3, b1, IDESC128, 1u);     // S3 x S1      -> group 2
        }
        umma_commit(smem_u32(&bars[NST + s]));  // stage free once these MMAs retire
        first = false;
      }
      umma_commit(smem_u32(&bars[2 * NST]));    // chunk accumulators ready
    }
  } else if (warp >= 2) {
    // ---- epilogue: TMEM -> FP64 accumulators (all K chunks) -> one store of C ----
    // Two warps per TMEM lane quadrant (warp % 4): each thread owns one row and
    // 64 of the 128 columns, summing the three groups of every chunk in FP64.
    const int quad = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = quad * 32 + lane;
    double acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    for (int c = 0; c < nchunks; ++c) {
      if (!mbar_wait(smem_u32(&bars[2 * NST]), c & 1)) { atomicExch(&abort_flag, 1); break; }
      tc_fence_after();
#pragma unroll
      for (int cb = 0; cb < 64; cb += 16) {
        const uint32_t taddr = tmem + (static_cast<uint32_t>(quad * 32) << 16) +
                               static_cast<uint32_t>(64 * half + cb);
        uint32_t g[16];
        tmem_ld16(taddr, g);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-12;
        tmem_ld16(taddr + TN, g);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-23;
        tmem_ld16(taddr + 2 * TN, g);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-34;
      }
      tc_fence_before();
      mbar_arrive(smem_u32(&bars[2 * NST + 1]));
    }
    // After the last chunk every MMA has retired and every TMA load has been
    // consumed, so the stage buffers hold the scaled tile T[128][129] for a
    // store along whichever index of the output is contiguous.
    double* T = reinterpret_cast<double*>(base);
    constexpr int LDT = TN + 1;
    const int64_t m = m0 + row;
    const double sa = m < p.M ? ldexp(p.alpha, p.ea[m]) : 0.0;
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      const int64_t n = n0 + 64 * half + j;
      T[row * LDT + 64 * half + j] = n < p.N ? acc[j] * sa * ldexp(1.0, p.eb[n]) : 0.0;
    }
    asm volatile("bar.sync 1, 256;\n" ::: "memory");
    if (!abort_flag) {
      const int ew = warp - 2;  // 0..7
      for (int out = 0; out < 2; ++out) {
        double* O = out == 0 ? p.C : p.C2;
        if (!O) continue;
        const Ax& Om = out == 0 ? p.Cm : p.C2m;
        const Ax& On = out == 0 ? p.Cn : p.C2n;
        const bool n_contig = On.s_i == 1 && On.inner > 1;
        for (int q = 0; q < 16; ++q) {
          double* ptr[4];
          double val[4];
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            // n-contiguous: warp row r, lanes along columns; otherwise warp column, lanes along rows
            const int r = n_contig ? ew + 8 * q : 32 * b + lane;
            const int cc = n_contig ? 32 * b + lane : ew + 8 * q;
            const int64_t mm = m0 + r, nn = n0 + cc;
            const bool in = mm < p.M && nn < p.N;
            ptr[b] = in ? O + Om.off(static_cast<uint32_t>(mm)) + On.off(static_cast<uint32_t>(nn))
                        : nullptr;
            val[b] = T[r * LDT + cc];
          }
          rmw_store<4>(ptr, val, p.beta);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicExch(p.error, 1);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
  }
}

// ---------------------------------------------------------------------------
// Persistent variant: one CTA per SM walks the tiles (same raster order), so
// barrier set-up and TMEM allocation happen once, and the producer and the MMA
// issuer run ahead into the next tile while the epilogue warps store the last
// one.  TMEM is handed back after each chunk's drain as before; the stores use
// warp-private transposes (32 rows x 16 columns, XOR-swizzled), so no barrier
// spans warps and every warp leaves on an abort by a warp-uniform decision.
constexpr int WBUF_DOUBLES = 32 * 16;
constexpr int SMEM_BYTES_P = NST * STAGE_BYTES + 8 * WBUF_DOUBLES * 8 + 1024 + 256;

// Tile t in the grouped raster order: logical origins (m0, n0), packed-row origins
// (pa, pb) and the valid extents (mlim, nlim) of the tile.
struct TileAt {
  int64_t m0, n0, pa, pb;
  int mlim, nlim;
};
__device__ __forceinline__ TileAt tile_at(const SplitParams& p, int64_t t) {
  const int64_t nM = p.nMt, nN = p.nNt;
  const int64_t per_group = RASTER_M * nN, group = t / per_group;
  const int64_t first = group * RASTER_M;
  const int64_t rows = nM - first < RASTER_M ? nM - first : RASTER_M;
  const int64_t in = t - group * per_group;
  const int64_t tm = first + in % rows, tn = in / rows;
  TileAt a;
  const int64_t rm = tm / p.a_tiles, om = (tm - rm * p.a_tiles) * TM;
  const int64_t rn = tn / p.b_tiles, on = (tn - rn * p.b_tiles) * TN;
  a.m0 = rm * p.a_run + om;
  a.n0 = rn * p.b_run + on;
  a.pa = p.a_base + rm * p.a_stride + om;
  a.pb = p.b_base + rn * p.b_stride + on;
  const int64_t ml = min(p.a_run - om, p.M - a.m0), nl = min(p.b_run - on, p.N - a.n0);
  a.mlim = static_cast<int>(ml < 0 ? 0 : (ml > TM ? TM : ml));
  a.nlim = static_cast<int>(nl < 0 ? 0 : (nl > TN ? TN : nl));
  return a;
}

__global__ void __launch_bounds__(320)
split_kernel_persistent(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, SplitParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  double* wbufs = reinterpret_cast<double*>(base + NST * STAGE_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + NST * STAGE_BYTES + 8 * WBUF_DOUBLES * 8);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NST + 2);
  __shared__ int abort_flag;
  volatile int* abort_v = &abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ntiles = p.nMt * p.nNt;
  const int nchunks = (p.nkb * TK + KCHUNK - 1) / KCHUNK;
  constexpr int KB_PER_CHUNK = KCHUNK / TK;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < NST; ++s) {
      mbar_init(smem_u32(&bars[s]), 1);
      mbar_init(smem_u32(&bars[NST + s]), 1);
    }
    mbar_init(smem_u32(&bars[2 * NST]), 1);
    mbar_init(smem_u32(&bars[2 * NST + 1]), 256);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(smem_u32(tmem_slot)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: every k-block of every tile of this CTA ----
    uint32_t it = 0;
    for (int64_t t = blockIdx.x; t < ntiles && !*abort_v; t += gridDim.x) {
      const TileAt ta = tile_at(p, t);
      for (int kb = 0; kb < p.nkb; ++kb, ++it) {
        const int s = it % NST;
        if (it >= NST && !mbar_wait(smem_u32(&bars[NST + s]), ((it / NST) - 1) & 1)) {
          atomicExch(&abort_flag, 1);
          break;
        }
        if (*abort_v) break;
        const uint32_t full = smem_u32(&bars[s]);
        mbar_expect_tx(full, STAGE_BYTES);
        unsigned char* st = base + s * STAGE_BYTES;
        for (int q = 0; q < NSLICE; ++q) {
          tma_load_2d(smem_u32(st + q * TILE_BYTES), &tmA, full, kb * TK,
                      static_cast<int>(q * p.Mp + ta.pa));
          tma_load_2d(smem_u32(st + (NSLICE + q) * TILE_BYTES), &tmB, full, kb * TK,
                      static_cast<int>(q * p.Np + ta.pb));
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: chunks of all tiles, global stage and chunk counters ----
    uint32_t it = 0, q = 0;
    for (int64_t t = blockIdx.x; t < ntiles && !*abort_v; t += gridDim.x) {
      int kb = 0;
      for (int c = 0; c < nchunks && !*abort_v; ++c, ++q) {
        if (q > 0 && !mbar_wait(smem_u32(&bars[2 * NST + 1]), (q - 1) & 1)) {
          atomicExch(&abort_flag, 1);
          break;
        }
        tc_fence_after();
        const int kb_end = min(p.nkb, (c + 1) * KB_PER_CHUNK);
        bool first = true;
        for (; kb < kb_end; ++kb, ++it) {
          const int s = it % NST;
          if (!mbar_wait(smem_u32(&bars[s]), (it / NST) & 1)) { atomicExch(&abort_flag, 1); break; }
          tc_fence_after();
          const uint32_t st = smem_u32(base + s * STAGE_BYTES);
#pragma unroll
          for (int kk = 0; kk < TK / 16; ++kk) {
            const uint32_t koff = kk * 32;
            const uint32_t init = (first && kk == 0) ? 0u : 1u;
            const uint64_t a1 = sdesc(st + 0 * TILE_BYTES + koff);
            const uint64_t a2 = sdesc(st + 1 * TILE_BYTES + koff);
            const uint64_t a3 = sdesc(st + 2 * TILE_BYTES + koff);
            const uint64_t b12 = sdesc(st + (NSLICE + 0) * TILE_BYTES + koff);
            const uint64_t b3 = sdesc(st + (NSLICE + 2) * TILE_BYTES + koff);
            umma(tmem + 0 * TN, a1, b12, IDESC256, init);  // S1 x [S1|S2] -> groups 0, 1
            umma(tmem + 2 * TN, a1, b3, IDESC128, init);   // S1 x S3      -> group 2
            umma(tmem + 1 * TN, a2, b12, IDESC256, 1u);    // S2 x [S1|S2] -> groups 1, 2
            umma(tmem + 2 * TN, a3, b12, IDESC128, 1u);    // S3 x S1      -> group 2
          }
          umma_commit(smem_u32(&bars[NST + s]));
          first = false;
        }
        umma_commit(smem_u32(&bars[2 * NST]));
      }
    }
  } else if (warp >= 2) {
    // ---- epilogue: per tile, FP64 accumulation of every chunk, then the store ----
    const int quad = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = quad * 32 + lane;
    double* wb = wbufs + (warp - 2) * WBUF_DOUBLES;
    const bool m_major = p.Cm.s_i == 1 && p.Cm.inner > 1;  // output contiguous along rows
    uint32_t q = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      if (__any_sync(0xffffffffu, *abort_v != 0)) break;
      const TileAt ta = tile_at(p, t);
      const int64_t m0 = ta.m0, n0 = ta.n0;
      double acc[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) acc[j] = 0.0;
      bool ok = true;
      for (int c = 0; c < nchunks; ++c, ++q) {
        const bool got = mbar_wait(smem_u32(&bars[2 * NST]), q & 1);
        if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
        tc_fence_after();
#pragma unroll
        for (int cb = 0; cb < 64; cb += 16) {
          const uint32_t taddr = tmem + (static_cast<uint32_t>(quad * 32) << 16) +
                                 static_cast<uint32_t>(64 * half + cb);
          uint32_t g[16];
          tmem_ld16(taddr, g);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-12;
          tmem_ld16(taddr + TN, g);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-23;
          tmem_ld16(taddr + 2 * TN, g);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[cb + j] += static_cast<double>(__uint_as_float(g[j])) * 0x1p-34;
        }
        tc_fence_before();
        mbar_arrive(smem_u32(&bars[2 * NST + 1]));  // TMEM free: the next chunk may start
      }
      if (!ok) { atomicExch(&abort_flag, 1); break; }
      // store this warp's 32 rows x 64 columns (the MMA issuer is already on the next tile).
      // The offset of a row belongs to the lane of that row; the offset and the
      // power-of-two scale of a column are computed by one lane per group of 32 (or 16)
      // columns; both reach the lanes that store an element through warp shuffles
      // (offset -1: outside the output).
      const int64_t m = m0 + row;
      const bool mv = row < ta.mlim;
      const double sa = mv ? ldexp(p.alpha, p.ea[ta.pa + row]) : 0.0;
      const int64_t rowoff = mv ? p.Cm.off(static_cast<uint32_t>(m)) : -1;
      const int64_t rowoff2 = (mv && p.C2) ? p.C2m.off(static_cast<uint32_t>(m)) : -1;
      if (m_major && !p.C2 && p.beta != 0.0) {
        // Accumulating store, lanes on consecutive rows, software-pipelined: the old
        // values of the next group of four columns are loaded before the current group
        // is written (the elements of one output tile are distinct, so the loads may
        // pass the stores), keeping two groups of loads in flight per lane.
        int64_t colL[2];
        double scL[2];
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const int jl = 64 * half + 32 * h2 + lane;
          colL[h2] = jl < ta.nlim ? p.Cn.off(static_cast<uint32_t>(n0 + jl)) : -1;
          scL[h2] = jl < ta.nlim ? pow2i(p.eb[ta.pb + jl]) : 0.0;
        }
        auto fetch = [&](int g, double* (&ptr)[4], double (&val)[4], double (&old)[4]) {
          const int h2 = g >> 3, j0 = (g & 7) * 4;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int64_t col = __shfl_sync(0xffffffffu, colL[h2], j0 + j);
            const double sc = __shfl_sync(0xffffffffu, scL[h2], j0 + j);
            val[j] = acc[32 * h2 + j0 + j] * sa * sc;
            ptr[j] = (rowoff >= 0 && col >= 0) ? p.C + rowoff + col : nullptr;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) old[j] = ptr[j] ? *ptr[j] : 0.0;
        };
        double* pc[4];
        double vc[4], oc[4];
        fetch(0, pc, vc, oc);
#pragma unroll
        for (int g = 0; g < 16; ++g) {
          double* pn[4];
          double vn[4], on[4];
          if (g + 1 < 16) fetch(g + 1, pn, vn, on);
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (pc[j]) *pc[j] = vc[j] + p.beta * oc[j];
          if (g + 1 < 16) {
#pragma unroll
            for (int j = 0; j < 4; ++j) { pc[j] = pn[j]; vc[j] = vn[j]; oc[j] = on[j]; }
          }
        }
      } else if (m_major) {
        // lanes are consecutive rows: store column by column straight from registers
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const int jl = 64 * half + 32 * h2 + lane;  // this lane's column of the group
          const int64_t colL = jl < ta.nlim ? p.Cn.off(static_cast<uint32_t>(n0 + jl)) : -1;
          const double scL = jl < ta.nlim ? pow2i(p.eb[ta.pb + jl]) : 0.0;
#pragma unroll
          for (int j0 = 0; j0 < 32; j0 += 4) {
            double* ptr[4];
            double val[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int64_t col = __shfl_sync(0xffffffffu, colL, j0 + j);
              const double sc = __shfl_sync(0xffffffffu, scL, j0 + j);
              val[j] = acc[32 * h2 + j0 + j] * sa * sc;
              ptr[j] = (rowoff >= 0 && col >= 0) ? p.C + rowoff + col : nullptr;
            }
            rmw_store<4>(ptr, val, p.beta);
            if (p.C2) {
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const int jc = 64 * half + 32 * h2 + j0 + j;
                ptr[j] = (rowoff2 >= 0 && jc < ta.nlim)
                             ? p.C2 + rowoff2 + p.C2n.off(static_cast<uint32_t>(n0 + jc)) : nullptr;
              }
              rmw_store<4>(ptr, val, p.beta);
            }
          }
        }
      } else if (!p.C2 && p.beta != 0.0) {
        // Accumulating store, lanes along columns (16-column pieces through the warp's
        // buffer), pipelined like the row-major case: the old values of the next four
        // rows are loaded before the current four are written.
#pragma unroll
        for (int piece = 0; piece < 4; ++piece) {
          const int cc = lane & 15;
          const int jn = 64 * half + 16 * piece + cc;
          const int64_t nn = n0 + jn;
          const int64_t cn = jn < ta.nlim ? p.Cn.off(static_cast<uint32_t>(nn)) : -1;
          const double scL = jn < ta.nlim ? pow2i(p.eb[ta.pb + jn]) : 0.0;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const double sc = __shfl_sync(0xffffffffu, scL, j);
            wb[lane * 16 + (j ^ (lane & 15))] = acc[16 * piece + j] * sa * sc;
          }
          __syncwarp();
          auto fetch = [&](int k0, double* (&ptr)[4], double (&val)[4], double (&old)[4]) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int r = 2 * (k0 + k) + (lane >> 4);
              const int64_t ro = __shfl_sync(0xffffffffu, rowoff, r);
              val[k] = wb[r * 16 + (cc ^ (r & 15))];
              ptr[k] = (ro >= 0 && cn >= 0) ? p.C + ro + cn : nullptr;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) old[k] = ptr[k] ? *ptr[k] : 0.0;
          };
          double* pc[4];
          double vc[4], oc[4];
          fetch(0, pc, vc, oc);
#pragma unroll
          for (int k0 = 0; k0 < 16; k0 += 4) {
            double* pn[4];
            double vn[4], on[4];
            if (k0 + 4 < 16) fetch(k0 + 4, pn, vn, on);
#pragma unroll
            for (int k = 0; k < 4; ++k)
              if (pc[k]) *pc[k] = vc[k] + p.beta * oc[k];
            if (k0 + 4 < 16) {
#pragma unroll
              for (int k = 0; k < 4; ++k) { pc[k] = pn[k]; vc[k] = vn[k]; oc[k] = on[k]; }
            }
          }
          __syncwarp();
        }
      } else {
        // 16-column pieces through the warp's buffer; lanes then run along columns
#pragma unroll
        for (int piece = 0; piece < 4; ++piece) {
          const int cc = lane & 15;  // this lane's column within the piece
          const int jn = 64 * half + 16 * piece + cc;
          const int64_t nn = n0 + jn;
          const int64_t cn = jn < ta.nlim ? p.Cn.off(static_cast<uint32_t>(nn)) : -1;
          const double scL = jn < ta.nlim ? pow2i(p.eb[ta.pb + jn]) : 0.0;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const double sc = __shfl_sync(0xffffffffu, scL, j);
            wb[lane * 16 + (j ^ (lane & 15))] = acc[16 * piece + j] * sa * sc;
          }
          __syncwarp();
#pragma unroll 1
          for (int k0 = 0; k0 < 16; k0 += 4) {
            double* ptr[4];
            double val[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int r = 2 * (k0 + k) + (lane >> 4);  // row within the warp
              const int64_t ro = __shfl_sync(0xffffffffu, rowoff, r);
              val[k] = wb[r * 16 + (cc ^ (r & 15))];
              ptr[k] = (ro >= 0 && cn >= 0) ? p.C + ro + cn : nullptr;
            }
            rmw_store<4>(ptr, val, p.beta);
            if (p.C2) {
              const int64_t cn2 = jn < ta.nlim ? p.C2n.off(static_cast<uint32_t>(nn)) : -1;
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const int r = 2 * (k0 + k) + (lane >> 4);
                const int64_t r2 = __shfl_sync(0xffffffffu, rowoff2, r);
                ptr[k] = (r2 >= 0 && cn2 >= 0) ? p.C2 + r2 + cn2 : nullptr;
              }
              rmw_store<4>(ptr, val, p.beta);
            }
          }
          __syncwarp();
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicExch(p.error, 1);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
  }
}

// ---------------------------------------------------------------------------
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  });
  if (!fn) throw Error(ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  return fn;
}

// 2-D map over packed slices [3*Rp][Kp] FP16, box TK (k) x 128 (rows), rows of
// ROW_BYTES swizzled like the MMA descriptors expect.
CUtensorMap make_map(void* base, int64_t rows, int64_t Kp) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(Kp), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(Kp * 2)};
  const cuuint32_t box[2] = {TK, 128};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, base, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE,
                           ROW_BYTES == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return m;
}

inline int64_t rup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

struct Layout2 {
  int64_t Mp, Np, Kp;
  size_t a_bytes, b_bytes, meta_bytes;
};
Layout2 layout_of(const Contraction& g) {
  Layout2 L;
  L.Mp = rup(g.M, TM);
  L.Np = rup(g.N, TN);
  L.Kp = rup(std::max<int64_t>(g.K, 1), TK);
  L.a_bytes = rup(static_cast<int64_t>(NSLICE * L.Mp * L.Kp * 2), 1024);
  L.b_bytes = rup(static_cast<int64_t>(NSLICE * L.Np * L.Kp * 2), 1024);
  L.meta_bytes = rup((L.Mp + L.Np) * (8 + 4), 1024);
  return L;
}

void pack(const View& v, bool rows_are_m, const Contraction& g, int64_t R, int64_t Rp,
          int64_t Kp, __half* dst, unsigned long long* rmax, int* rexp, cudaStream_t s) {
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  const int64_t Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1);
  PackArgs a;
  a.src = v.p;
  if (rows_are_m) {  // A(m, k): rows = m (s_ro, s_ri), k = cols (s_co, s_ci)
    a.ar = mkax(Mi, v.s_ro, v.s_ri);
    a.ak = mkax(Ki, v.s_co, v.s_ci);
    a.r_contig = (v.s_ri == 1 && v.s_ci != 1) ? 1 : 0;
  } else {           // B(k, n): rows of the packed operand = n (s_co, s_ci), k = (s_ro, s_ri)
    a.ar = mkax(Ni, v.s_co, v.s_ci);
    a.ak = mkax(Ki, v.s_ro, v.s_ri);
    a.r_contig = (v.s_ci == 1 && v.s_ri != 1) ? 1 : 0;
  }
  a.R = R; a.K = g.K; a.Rp = Rp; a.Kp = Kp;
  a.rmax = rmax; a.rexp = rexp; a.dst = dst;
  if (Rp % PR || Kp % 16) throw Error(ERR_BAD_SHAPE, "gemm_split: packed extents not tiled");
  CC_CHECK(cudaMemsetAsync(rmax, 0, R * sizeof(unsigned long long), s));
  const int64_t strips = (Rp / PR) * ((Kp + PKT * PSTRIP - 1) / (PKT * PSTRIP));
  const int64_t tiles = (Rp / PR) * ((Kp + PKT - 1) / PKT);
  pack_max_kernel<<<static_cast<unsigned>(std::min<int64_t>(strips, 148 * 8)), PTHREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  pack_slices_kernel<<<static_cast<unsigned>(std::min<int64_t>(tiles, 148 * 8)), PTHREADS, 0, s>>>(a);
  CC_LAUNCH_CHECK();
  g_pack_launches.fetch_add(2);
}

// Packed slices of both operands are limited to this many bytes: a longer K is
// cut into panels (multiples of KCHUNK where possible), each packed and
// multiplied in turn and accumulated into C in FP64.
constexpr size_t kPanelBytes = size_t(3) << 30;  // 3 GiB: one panel for the ladder contractions

// CC4S_SPLIT_PANEL_BYTES (at least 1 MiB) overrides the limit, e.g. to trade
// scratch memory for fewer, longer panels.
size_t panel_bytes() {
  if (const char* e = std::getenv("CC4S_SPLIT_PANEL_BYTES")) {
    const long long v = std::atoll(e);
    if (v >= (1ll << 20)) return static_cast<size_t>(v);
  }
  return kPanelBytes;
}

int64_t panel_len(const Contraction& g) {
  const int64_t per_k = 2 * NSLICE * (rup(g.M, TM) + rup(g.N, TN));  // bytes per k
  int64_t P = static_cast<int64_t>(panel_bytes()) / per_k;
  if (P >= KCHUNK) P = P / KCHUNK * KCHUNK;
  else P = std::max<int64_t>(TK, P / TK * TK);
  return P;
}

struct Panel { int64_t k0, kl, ki, a_off, b_off; };

// K panels of length <= P.  A two-level K index (inner extent Ki) is cut either
// into groups of whole inner runs (Ki <= P) or inside each run (Ki > P); the
// operand views are shifted to the panel start.
std::vector<Panel> panels_of(const Contraction& g, int64_t P) {
  std::vector<Panel> out;
  const int64_t K = g.K, Ki = g.Ki > 0 ? g.Ki : K;
  if (K <= P) {
    out.push_back({0, K, g.Ki, 0, 0});
  } else if (Ki >= K) {
    for (int64_t k0 = 0; k0 < K; k0 += P)
      out.push_back({k0, std::min(P, K - k0), 0, k0 * g.A.s_ci, k0 * g.B.s_ri});
  } else if (Ki <= P) {
    const int64_t runs = P / Ki;
    for (int64_t q0 = 0; q0 * Ki < K; q0 += runs)
      out.push_back({q0 * Ki, std::min(runs * Ki, K - q0 * Ki), Ki, q0 * g.A.s_co, q0 * g.B.s_ro});
  } else {
    for (int64_t q = 0; q * Ki < K; ++q)
      for (int64_t r0 = 0; r0 < Ki && q * Ki + r0 < K; r0 += P)
        out.push_back({q * Ki + r0, std::min(std::min(P, Ki - r0), K - q * Ki - r0), 0,
                       q * g.A.s_co + r0 * g.A.s_ci, q * g.B.s_ro + r0 * g.B.s_ri});
  }
  return out;
}

void split_panel(const Contraction& g, cudaStream_t s, SplitScratch& ws,
                 const SplitPackedB* pb = nullptr);

}  // namespace

uint64_t split_launch_count() { return g_split_launches.load(); }
uint64_t split_pack_launch_count() { return g_pack_launches.load(); }

size_t gemm_split_scratch_bytes(const Contraction& g) {
  Contraction h = g;
  h.K = std::min(g.K, panel_len(g));
  const Layout2 L = layout_of(h);
  return L.a_bytes + L.b_bytes + L.meta_bytes;
}

size_t split_packed_b_bytes(const Contraction& g) {
  const Layout2 L = layout_of(g);
  return L.b_bytes + rup(L.Np * 8, 1024) + rup(L.Np * 4, 1024);
}

size_t split_scratch_bytes_packed_b(const Contraction& g) {
  const Layout2 L = layout_of(g);
  return L.a_bytes + L.meta_bytes;
}

bool split_single_panel(const Contraction& g) { return g.K <= panel_len(g) && g.batch == 1; }

SplitPackedB split_pack_b(const Contraction& g, void* dst, cudaStream_t s) {
  if (!split_single_panel(g)) throw Error(ERR_UNSUPPORTED, "split_pack_b: K beyond one panel");
  const Layout2 L = layout_of(g);
  unsigned char* p = static_cast<unsigned char*>(dst);
  SplitPackedB b;
  b.slices = p;
  auto* bmax = reinterpret_cast<unsigned long long*>(p + L.b_bytes);
  b.exps = reinterpret_cast<int*>(p + L.b_bytes + rup(L.Np * 8, 1024));
  b.N = g.N; b.K = g.K; b.Np = L.Np; b.Kp = L.Kp;
  pack(g.B, false, g, g.N, L.Np, L.Kp, static_cast<__half*>(b.slices), bmax, b.exps, s);
  return b;
}

void gemm_split_packed_b(const Contraction& g, const SplitPackedB& b, cudaStream_t s,
                         SplitScratch& ws) {
  if (g.M <= 0 || g.N <= 0) return;
  if (!split_single_panel(g)) throw Error(ERR_UNSUPPORTED, "gemm_split_packed_b: K beyond one panel");
  split_panel(g, s, ws, &b);
}

void gemm_split(const Contraction& g, cudaStream_t s, SplitScratch& ws) {
  if (g.M <= 0 || g.N <= 0) return;
  if (g.batch != 1) throw Error(ERR_UNSUPPORTED, "gemm_split: batched contraction");
  if (g.K <= 0) throw Error(ERR_UNSUPPORTED, "gemm_split: empty K");
  const std::vector<Panel> ps = panels_of(g, panel_len(g));
  for (size_t i = 0; i < ps.size(); ++i) {
    Contraction h = g;
    h.K = ps[i].kl;
    h.Ki = ps[i].ki;
    h.A.p = g.A.p + ps[i].a_off;
    h.B.p = g.B.p + ps[i].b_off;
    if (i > 0) h.beta = 1.0;
    split_panel(h, s, ws);
  }
}

namespace {

// Persistent tile loop by default; CC4S_SPLIT_PERSISTENT=0 selects one tile per CTA.
bool persistent_mode() {
  static const bool persistent = [] {
    const char* e = std::getenv("CC4S_SPLIT_PERSISTENT");
    return !(e && e[0] == '0');
  }();
  return persistent;
}

void launch_persistent(const CUtensorMap& ta, const CUtensorMap& tb, const SplitParams& sp,
                       int64_t tiles, cudaStream_t s) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    CC_CHECK(cudaGetDevice(&dev));
    CC_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CC_CHECK(cudaFuncSetAttribute(split_kernel_persistent,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES_P));
  }
  dim3 grid(static_cast<unsigned>(std::min<int64_t>(tiles, sms)));
  split_kernel_persistent<<<grid, 320, SMEM_BYTES_P, s>>>(ta, tb, sp);
}

void split_panel(const Contraction& g, cudaStream_t s, SplitScratch& ws, const SplitPackedB* pb) {
  const Layout2 L = layout_of(g);
  // with a pre-packed B the scratch holds A and the metadata only
  const size_t need = L.a_bytes + (pb ? 0 : L.b_bytes) + L.meta_bytes;
  if (need > ws.bytes) throw Error(ERR_OUT_OF_MEMORY, "gemm_split: scratch too small");
  if (L.Mp * NSLICE >= (int64_t(1) << 31) || L.Np * NSLICE >= (int64_t(1) << 31) || L.Kp >= (int64_t(1) << 31))
    throw Error(ERR_BAD_SHAPE, "gemm_split: extent too large");
  unsigned char* p = static_cast<unsigned char*>(ws.p);
  __half* Apk = reinterpret_cast<__half*>(p);
  __half* Bpk = reinterpret_cast<__half*>(p + L.a_bytes);
  unsigned char* meta = p + L.a_bytes + (pb ? 0 : L.b_bytes);
  auto* amax = reinterpret_cast<unsigned long long*>(meta);
  auto* bmax = amax + L.Mp;
  int* aexp = reinterpret_cast<int*>(bmax + L.Np);
  int* bexp = aexp + L.Mp;
  pack(g.A, true, g, g.M, L.Mp, L.Kp, Apk, amax, aexp, s);
  if (pb) {   // B sliced before, by split_pack_b, for this N, K and padding
    if (pb->N != g.N || pb->K != g.K || pb->Np != L.Np || pb->Kp != L.Kp)
      throw Error(ERR_INVALID_ARGUMENT, "gemm_split: pre-packed B of another shape");
    Bpk = static_cast<__half*>(pb->slices);
    bexp = pb->exps;
  } else {
    pack(g.B, false, g, g.N, L.Np, L.Kp, Bpk, bmax, bexp, s);
  }
  const CUtensorMap ta = make_map(Apk, NSLICE * L.Mp, L.Kp);
  const CUtensorMap tb = make_map(Bpk, NSLICE * L.Np, L.Kp);
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  SplitParams sp;
  sp.M = g.M; sp.N = g.N; sp.K = g.K; sp.Mp = L.Mp; sp.Np = L.Np;
  sp.nkb = static_cast<int>(L.Kp / TK);
  sp.Cm = mkax(Mi, g.C.s_ro, g.C.s_ri);
  sp.Cn = mkax(Ni, g.C.s_co, g.C.s_ci);
  sp.C2m = mkax(Mi, g.C2.s_ro, g.C2.s_ri);
  sp.C2n = mkax(Ni, g.C2.s_co, g.C2.s_ci);
  sp.C = g.C.p; sp.C2 = g.C2.p;
  sp.alpha = g.alpha; sp.beta = g.beta;
  sp.ea = aexp; sp.eb = bexp;
  sp.error = ws.error;
  sp.a_run = g.M; sp.a_stride = 0; sp.a_base = 0; sp.a_tiles = L.Mp / TM; sp.nMt = L.Mp / TM;
  sp.b_run = g.N; sp.b_stride = 0; sp.b_base = 0; sp.b_tiles = L.Np / TN; sp.nNt = L.Np / TN;
  const int64_t tiles = (L.Np / TN) * (L.Mp / TM);
  if (tiles >= (int64_t(1) << 31)) throw Error(ERR_BAD_SHAPE, "gemm_split: too many tiles");
  if (persistent_mode()) {
    launch_persistent(ta, tb, sp, tiles, s);
  } else {
    static bool configured = false;
    if (!configured) {
      CC_CHECK(cudaFuncSetAttribute(split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
      configured = true;
    }
    dim3 grid(static_cast<unsigned>(tiles));
    split_kernel<<<grid, 320, SMEM_BYTES, s>>>(ta, tb, sp);
  }
  CC_LAUNCH_CHECK();
  g_split_launches.fetch_add(1);
}

}  // namespace
size_t split_operand_bytes(int64_t R, int64_t K) {
  const int64_t Rp = rup(std::max<int64_t>(R, 1), TM), Kp = rup(std::max<int64_t>(K, 1), TK);
  return static_cast<size_t>(rup(NSLICE * Rp * Kp * 2, 1024) + rup(Rp * 8, 1024) +
                             rup(Rp * 4, 1024));
}

SplitOperand split_pack_operand(const double* src, int64_t R, int64_t Ri, int64_t s_ro,
                                int64_t s_ri, int64_t K, int64_t s_k, void* dst, cudaStream_t s) {
  if (R <= 0 || K <= 0) throw Error(ERR_BAD_SHAPE, "split_pack_operand: empty operand");
  SplitOperand o;
  o.R = R; o.K = K;
  o.Rp = rup(R, TM);
  o.Kp = rup(K, TK);
  if (o.Rp * NSLICE >= (int64_t(1) << 31) || o.Kp >= (int64_t(1) << 31))
    throw Error(ERR_BAD_SHAPE, "split_pack_operand: extent too large");
  unsigned char* p = static_cast<unsigned char*>(dst);
  const int64_t sb = rup(NSLICE * o.Rp * o.Kp * 2, 1024);
  o.slices = p;
  auto* rmax = reinterpret_cast<unsigned long long*>(p + sb);
  o.exps = reinterpret_cast<int*>(p + sb + rup(o.Rp * 8, 1024));
  Contraction g;
  g.M = R; g.Mi = Ri; g.K = K;
  g.A.p = const_cast<double*>(src);
  g.A.s_ro = s_ro; g.A.s_ri = s_ri; g.A.s_co = 0; g.A.s_ci = s_k;
  pack(g.A, true, g, R, o.Rp, o.Kp, static_cast<__half*>(o.slices), rmax, o.exps, s);
  return o;
}

void gemm_split_prepacked(const Contraction& g, const SplitOperand& A, const SplitRuns& ar,
                          const SplitOperand& B, const SplitRuns& br, cudaStream_t s,
                          SplitScratch& ws) {
  if (g.M <= 0 || g.N <= 0) return;
  if (!persistent_mode())
    throw Error(ERR_UNSUPPORTED, "gemm_split_prepacked: needs the persistent kernel");
  if (A.K != g.K || B.K != g.K || A.Kp != B.Kp)
    throw Error(ERR_INVALID_ARGUMENT, "gemm_split_prepacked: operands of another K");
  // every packed row that a valid logical row reads lies inside the operand
  auto check = [](const SplitRuns& r, int64_t X, int64_t R, const char* what) {
    if (r.run <= 0 || r.base < 0 || r.stride < 0)
      throw Error(ERR_INVALID_ARGUMENT, std::string("gemm_split_prepacked: bad runs of ") + what);
    const int64_t nr = (X + r.run - 1) / r.run;
    const int64_t last = r.base + (nr - 1) * r.stride + std::min(r.run, X - (nr - 1) * r.run) - 1;
    const int64_t full_last = nr > 1 ? r.base + (nr - 2) * r.stride + r.run - 1 : -1;
    if (last >= R || full_last >= R)
      throw Error(ERR_INVALID_ARGUMENT, std::string("gemm_split_prepacked: runs of ") + what +
                                            " leave the operand");
    return nr;
  };
  const int64_t nra = check(ar, g.M, A.R, "A"), nrb = check(br, g.N, B.R, "B");
  const CUtensorMap ta = make_map(A.slices, NSLICE * A.Rp, A.Kp);
  const CUtensorMap tb = make_map(B.slices, NSLICE * B.Rp, B.Kp);
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M, Ni = g.Ni > 0 ? g.Ni : g.N;
  SplitParams sp;
  sp.M = g.M; sp.N = g.N; sp.K = g.K; sp.Mp = A.Rp; sp.Np = B.Rp;
  sp.nkb = static_cast<int>(A.Kp / TK);
  sp.Cm = mkax(Mi, g.C.s_ro, g.C.s_ri);
  sp.Cn = mkax(Ni, g.C.s_co, g.C.s_ci);
  sp.C2m = mkax(Mi, g.C2.s_ro, g.C2.s_ri);
  sp.C2n = mkax(Ni, g.C2.s_co, g.C2.s_ci);
  sp.C = g.C.p; sp.C2 = g.C2.p;
  sp.alpha = g.alpha; sp.beta = g.beta;
  sp.ea = A.exps; sp.eb = B.exps;
  sp.error = ws.error;
  sp.a_run = ar.run; sp.a_stride = ar.stride; sp.a_base = ar.base;
  sp.a_tiles = (ar.run + TM - 1) / TM; sp.nMt = nra * sp.a_tiles;
  sp.b_run = br.run; sp.b_stride = br.stride; sp.b_base = br.base;
  sp.b_tiles = (br.run + TN - 1) / TN; sp.nNt = nrb * sp.b_tiles;
  const int64_t tiles = sp.nMt * sp.nNt;
  if (tiles >= (int64_t(1) << 31)) throw Error(ERR_BAD_SHAPE, "gemm_split_prepacked: too many tiles");
  launch_persistent(ta, tb, sp, tiles, s);
  CC_LAUNCH_CHECK();
  g_split_launches.fetch_add(1);
}

}  // namespace cc4s_b200
