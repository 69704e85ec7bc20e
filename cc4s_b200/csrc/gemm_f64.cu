// FP64 DMMA contraction kernel (mma.sync.m16n8k16.f64) with cp.async staging.
//
// Tile 128 (m) x 128 (n) x 32 (k), 256 threads = 8 warps in a 2 x 4 grid,
// each warp owns a 64 x 32 sub-tile = 4 x 4 MMA tiles of 16 x 8.  Operand
// tiles are staged through a 3-stage cp.async ring in shared memory (212 KB).
// Shared-memory rows are padded by 4 doubles so that the fragment reads of
// both storage orders ([m][k] and [k][m]) are free of bank conflicts.
// Address arithmetic is kept off the critical path: offsets of the m / n
// tile rows are computed once per tile, k offsets with 32-bit division once
// per thread and k-tile, then stepped incrementally.
#include "gemm_f64.cuh"

#include <algorithm>
#include <atomic>

namespace cc4s_b200 {

namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int64_t RASTER_M = 8;  // tile rows per raster group

static std::atomic<uint64_t> g_launches{0};

// One index of an operand, split as x = (x / inner) * s_o + (x % inner) * s_i.
struct Axis {
  uint32_t inner;
  int64_t s_o, s_i;
  __device__ __forceinline__ int64_t off(uint32_t x) const {
    const uint32_t o = x / inner;
    return static_cast<int64_t>(o) * s_o + static_cast<int64_t>(x - o * inner) * s_i;
  }
};

struct KParams {
  int64_t M, N, K, batch, ksplit_len;
  int nsplit;
  Axis Am, Ak, Bk, Bn, Cm, Cn, C2m, C2n, Ab, Bb, Cb, C2b;
  double* A; double* B; double* C; double* C2;
  double alpha, beta;
  double* partial;  // split-K partials [nsplit][batch][M][N] or nullptr
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int n = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Loader of one operand tile stored S[u][w] (w contiguous in shared memory,
// row length W + 4).  One of (u, w) is the k index, the other is m or n.
// KU: the strided tile axis u is k; otherwise w is k.
template <int U, int W, int V, bool KU>
struct Loader {
  static constexpr int LD = W + 4;
  static constexpr int WCH = W / V;               // chunks per smem row
  static constexpr int RP = THREADS / WCH;        // rows per pass
  static constexpr int PER = U / RP;              // passes
  static_assert((U * W / V) % THREADS == 0 && THREADS % WCH == 0, "tile split");
  // fixed part (the m / n index)
  int64_t fix[KU ? 1 : PER];
  bool fok[KU ? 1 : PER];
  int wl, ul0;

  __device__ __forceinline__ void init(int tid, int64_t f0, int64_t fext, const Axis& af) {
    wl = (tid % WCH) * V;
    ul0 = tid / WCH;
    if (KU) {
      const int64_t x = f0 + wl;
      fok[0] = x < fext;
      fix[0] = fok[0] ? af.off(static_cast<uint32_t>(x)) : 0;
    } else {
#pragma unroll
      for (int r = 0; r < PER; ++r) {
        const int64_t x = f0 + ul0 + r * RP;
        fok[r] = x < fext;
        fix[r] = fok[r] ? af.off(static_cast<uint32_t>(x)) : 0;
      }
    }
  }

  __device__ __forceinline__ void load(double* S, const double* base, int64_t k0, int64_t kend,
                                       const Axis& ak) const {
    if (KU) {
      // u = k varies with r: step (ko, ki) incrementally by RP
      uint32_t k = static_cast<uint32_t>(k0 + ul0);
      uint32_t ko = k / ak.inner, ki = k - ko * ak.inner;
#pragma unroll
      for (int r = 0; r < PER; ++r) {
        const bool ok = fok[0] && (static_cast<int64_t>(k) < kend);
        const double* g = ok ? base + static_cast<int64_t>(ko) * ak.s_o +
                                   static_cast<int64_t>(ki) * ak.s_i + fix[0]
                             : base;
        double* sp = S + (ul0 + r * RP) * LD + wl;
        if (V == 2) cp_async16(sp, g, ok); else cp_async8(sp, g, ok);
        k += RP;
        ki += RP;
        while (ki >= ak.inner) { ki -= ak.inner; ++ko; }
      }
    } else {
      const int64_t k = k0 + wl;
      const bool kok = k < kend;
      const int64_t koff = kok ? ak.off(static_cast<uint32_t>(k)) : 0;
#pragma unroll
      for (int r = 0; r < PER; ++r) {
        const bool ok = kok && fok[r];
        const double* g = ok ? base + fix[r] + koff : base;
        double* sp = S + (ul0 + r * RP) * LD + wl;
        if (V == 2) cp_async16(sp, g, ok); else cp_async8(sp, g, ok);
      }
    }
  }
};

__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// A_KC: A tile stored [m][k]; otherwise [k][m].  B_NC: B tile stored [k][n]; otherwise [n][k].
template <bool A_KC, bool B_NC, int VA, int VB>
__global__ void __launch_bounds__(THREADS, 1) gemm_f64_kernel(KParams p) {
  extern __shared__ __align__(16) double smem[];
  using LA = Loader<A_KC ? BM : BK, A_KC ? BK : BM, VA, !A_KC>;
  using LB = Loader<B_NC ? BK : BN, B_NC ? BN : BK, VB, B_NC>;
  constexpr int A_SIZE = (A_KC ? BM : BK) * LA::LD;
  constexpr int B_SIZE = (B_NC ? BK : BN) * LB::LD;
  constexpr int STAGE = A_SIZE + B_SIZE;
  constexpr int ALD = LA::LD, BLD = LB::LD;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;

  // Grouped tile order: the blocks launched together cover RASTER_M tile rows
  // and sweep the tile columns, so each B column tile is read from DRAM once per
  // group of RASTER_M tile rows (and served from L2 for the others) instead of
  // once per tile row.
  int64_t m0, n0;
  {
    const int64_t nN = gridDim.x, nM = gridDim.y;
    const int64_t lin = static_cast<int64_t>(blockIdx.y) * nN + blockIdx.x;
    const int64_t per_group = RASTER_M * nN, group = lin / per_group;
    const int64_t first = group * RASTER_M;
    const int64_t rows = nM - first < RASTER_M ? nM - first : RASTER_M;
    const int64_t in = lin - group * per_group;
    m0 = (first + in % rows) * BM;
    n0 = (in / rows) * BN;
  }
  const int64_t z = blockIdx.z;
  const int64_t b = z % p.batch;
  const int split = static_cast<int>(z / p.batch);
  const int64_t kbeg = split * p.ksplit_len;
  const int64_t kend = min(p.K, kbeg + p.ksplit_len);

  const double* Ab = p.A + p.Ab.off(static_cast<uint32_t>(b));
  const double* Bb = p.B + p.Bb.off(static_cast<uint32_t>(b));

  LA la;
  LB lb;
  la.init(tid, m0, p.M, p.Am);
  lb.init(tid, n0, p.N, p.Bn);

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  const int64_t ntiles = (kend > kbeg) ? (kend - kbeg + BK - 1) / BK : 0;

  auto load_stage = [&](int64_t kt, int stage) {
    double* As = smem + stage * STAGE;
    double* Bs = As + A_SIZE;
    const int64_t k0 = kbeg + kt * BK;
    la.load(As, Ab, k0, kend, p.Ak);
    lb.load(Bs, Bb, k0, kend, p.Bk);
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ntiles) load_stage(s, s);
    cp_commit();
  }

  for (int64_t kt = 0; kt < ntiles; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    {
      const int64_t nk = kt + STAGES - 1;
      if (nk < ntiles) load_stage(nk, static_cast<int>(nk % STAGES));
      cp_commit();
    }
    const double* As = smem + (kt % STAGES) * STAGE;
    const double* Bs = As + A_SIZE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      double a[4][8], bf[4][4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int mr = wm + mt * 16 + g + ((q & 1) << 3);
          const int kc = kk + t + (q >> 1) * 4;
          a[mt][q] = A_KC ? As[mr * ALD + kc] : As[kc * ALD + mr];
        }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int nc = wn + nt * 8 + g;
          const int kc = kk + t + q * 4;
          bf[nt][q] = B_NC ? Bs[kc * BLD + nc] : Bs[nc * BLD + kc];
        }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma16(acc[mt][nt], a[mt], bf[nt]);
    }
  }
  cp_wait<0>();

  // Epilogue.
  if (p.partial) {
    double* P = p.partial + (static_cast<int64_t>(split) * p.batch + b) * p.M * p.N;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int64_t m = m0 + wm + mt * 16 + g + ((q >> 1) << 3);
          const int64_t n = n0 + wn + nt * 8 + 2 * t + (q & 1);
          if (m < p.M && n < p.N) P[m * p.N + n] = acc[mt][nt][q];
        }
    return;
  }
  double* Cb = p.C + p.Cb.off(static_cast<uint32_t>(b));
  double* C2b = p.C2 ? p.C2 + p.C2b.off(static_cast<uint32_t>(b)) : nullptr;
  int64_t co[8], co2[8];
#pragma unroll
  for (int h = 0; h < 8; ++h) {  // column offsets: nt = h >> 1, parity h & 1
    const int64_t n = n0 + wn + (h >> 1) * 8 + 2 * t + (h & 1);
    co[h] = n < p.N ? p.Cn.off(static_cast<uint32_t>(n)) : 0;
    co2[h] = (C2b && n < p.N) ? p.C2n.off(static_cast<uint32_t>(n)) : 0;
  }
  // Accumulating stores: the eight old values of a fragment row are loaded before
  // any of them is stored, so the reads are in flight together (a store followed
  // by a load through another pointer would serialise them: the two may alias).
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int64_t m = m0 + wm + mt * 16 + g + hh * 8;
      if (m >= p.M) continue;
      const int64_t ro = p.Cm.off(static_cast<uint32_t>(m));
      const int64_t ro2 = C2b ? p.C2m.off(static_cast<uint32_t>(m)) : 0;
      double val[8], old[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const int64_t n = n0 + wn + (h >> 1) * 8 + 2 * t + (h & 1);
        val[h] = p.alpha * acc[mt][h >> 1][hh * 2 + (h & 1)];
        old[h] = (p.beta != 0.0 && n < p.N) ? Cb[ro + co[h]] : 0.0;
      }
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const int64_t n = n0 + wn + (h >> 1) * 8 + 2 * t + (h & 1);
        if (n < p.N) Cb[ro + co[h]] = val[h] + p.beta * old[h];
      }
      if (C2b) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int64_t n = n0 + wn + (h >> 1) * 8 + 2 * t + (h & 1);
          old[h] = (p.beta != 0.0 && n < p.N) ? C2b[ro2 + co2[h]] : 0.0;
        }
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int64_t n = n0 + wn + (h >> 1) * 8 + 2 * t + (h & 1);
          if (n < p.N) C2b[ro2 + co2[h]] = val[h] + p.beta * old[h];
        }
      }
    }
}

// Fixed-order reduction of split-K partials, then the alpha/beta epilogue.
__global__ void splitk_reduce_kernel(KParams p) {
  const int64_t total = p.batch * p.M * p.N;
  const int64_t slab = total;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < p.nsplit; ++q) s += p.partial[q * slab + e];
    const int64_t b = e / (p.M * p.N);
    const int64_t r = e - b * p.M * p.N;
    const int64_t m = r / p.N, n = r - (r / p.N) * p.N;
    const double v = p.alpha * s;
    double* c = p.C + p.Cb.off(static_cast<uint32_t>(b)) + p.Cm.off(static_cast<uint32_t>(m)) +
                p.Cn.off(static_cast<uint32_t>(n));
    *c = (p.beta != 0.0) ? v + p.beta * *c : v;
    if (p.C2) {
      double* c2 = p.C2 + p.C2b.off(static_cast<uint32_t>(b)) +
                   p.C2m.off(static_cast<uint32_t>(m)) + p.C2n.off(static_cast<uint32_t>(n));
      *c2 = (p.beta != 0.0) ? v + p.beta * *c2 : v;
    }
  }
}

inline Axis axis(int64_t inner, int64_t s_o, int64_t s_i) {
  Axis a;
  a.inner = static_cast<uint32_t>(inner > 0 ? inner : 1);
  a.s_o = s_o;
  a.s_i = s_i;
  return a;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <bool AK, bool BN_, int VA, int VB>
void launch(const KParams& p, dim3 grid, cudaStream_t s) {
  constexpr int A_SIZE = AK ? BM * (BK + 4) : BK * (BM + 4);
  constexpr int B_SIZE = BN_ ? BK * (BN + 4) : BN * (BK + 4);
  constexpr size_t smem = static_cast<size_t>(STAGES) * (A_SIZE + B_SIZE) * sizeof(double);
  static bool configured = false;
  if (!configured) {
    CC_CHECK(cudaFuncSetAttribute(gemm_f64_kernel<AK, BN_, VA, VB>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  gemm_f64_kernel<AK, BN_, VA, VB><<<grid, THREADS, smem, s>>>(p);
  CC_LAUNCH_CHECK();
}

}  // namespace

uint64_t gemm_launch_count() { return g_launches.load(); }

void gemm(const Contraction& g0, cudaStream_t s, const GemmScratch& ws) {
  Contraction g = g0;
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  if (g.K < 0) throw Error(ERR_INVALID_ARGUMENT, "gemm: negative K");
  const int64_t lim = int64_t(1) << 31;
  if (g.M >= lim || g.N >= lim || g.K >= lim || g.batch >= lim)
    throw Error(ERR_BAD_SHAPE, "gemm: extent beyond 2^31");
  const int64_t Mi = g.Mi > 0 ? g.Mi : g.M;
  const int64_t Ni = g.Ni > 0 ? g.Ni : g.N;
  const int64_t Ki = g.Ki > 0 ? g.Ki : std::max<int64_t>(g.K, 1);
  const int64_t Bi = g.Bi > 0 ? g.Bi : g.batch;

  KParams p{};
  p.M = g.M; p.N = g.N; p.K = g.K; p.batch = g.batch;
  p.Am = axis(Mi, g.A.s_ro, g.A.s_ri);
  p.Ak = axis(Ki, g.A.s_co, g.A.s_ci);
  p.Bk = axis(Ki, g.B.s_ro, g.B.s_ri);
  p.Bn = axis(Ni, g.B.s_co, g.B.s_ci);
  p.Cm = axis(Mi, g.C.s_ro, g.C.s_ri);
  p.Cn = axis(Ni, g.C.s_co, g.C.s_ci);
  p.C2m = axis(Mi, g.C2.s_ro, g.C2.s_ri);
  p.C2n = axis(Ni, g.C2.s_co, g.C2.s_ci);
  p.Ab = axis(Bi, g.A.s_bo, g.A.s_bi);
  p.Bb = axis(Bi, g.B.s_bo, g.B.s_bi);
  p.Cb = axis(Bi, g.C.s_bo, g.C.s_bi);
  p.C2b = axis(Bi, g.C2.s_bo, g.C2.s_bi);
  p.A = g.A.p; p.B = g.B.p; p.C = g.C.p; p.C2 = g.C2.p;
  p.alpha = g.alpha; p.beta = g.beta;
  if (!p.C || (g.K > 0 && (!p.A || !p.B)))
    throw Error(ERR_INVALID_ARGUMENT, "gemm: null operand");

  // Storage order of the staged tiles: prefer the contiguous axis.
  const bool a_kc = (g.A.s_ci == 1) || (g.A.s_ri != 1);
  const bool b_nc = (g.B.s_ci == 1) || (g.B.s_ri != 1);
  auto even = [](int64_t x) { return (x & 1) == 0; };
  // 16-byte chunks need the contiguous axis to pair up and every other stride even.
  bool va2, vb2;
  if (a_kc)
    va2 = g.A.s_ci == 1 && even(Ki) && even(g.K) && even(g.A.s_co) && even(g.A.s_ro) &&
          even(g.A.s_ri) && even(g.A.s_bo) && even(g.A.s_bi) && aligned16(g.A.p);
  else
    va2 = g.A.s_ri == 1 && even(Mi) && even(g.M) && even(g.A.s_ro) && even(g.A.s_co) &&
          even(g.A.s_ci) && even(g.A.s_bo) && even(g.A.s_bi) && aligned16(g.A.p);
  if (b_nc)
    vb2 = g.B.s_ci == 1 && even(Ni) && even(g.N) && even(g.B.s_co) && even(g.B.s_ro) &&
          even(g.B.s_ri) && even(g.B.s_bo) && even(g.B.s_bi) && aligned16(g.B.p);
  else
    vb2 = g.B.s_ri == 1 && even(Ki) && even(g.K) && even(g.B.s_ro) && even(g.B.s_co) &&
          even(g.B.s_ci) && even(g.B.s_bo) && even(g.B.s_bi) && aligned16(g.B.p);

  const int64_t mt = (g.M + BM - 1) / BM, nt = (g.N + BN - 1) / BN;
  const int64_t tiles = mt * nt * g.batch;
  // Split K when the output has too few tiles to fill 148 SMs.
  int nsplit = 1;
  const int64_t target = 2 * 148;
  if (tiles < target && g.K >= 8 * BK && ws.p) {
    int64_t want = (target + tiles - 1) / tiles;
    want = std::min<int64_t>(want, g.K / (4 * BK));
    want = std::min<int64_t>(want, 64);
    while (want > 1 && static_cast<size_t>(want * g.batch * g.M * g.N) > ws.elems) --want;
    if (want > 1) nsplit = static_cast<int>(want);
  }
  int64_t klen = g.K;
  if (nsplit > 1) {
    klen = (g.K + nsplit - 1) / nsplit;
    klen = ((klen + BK - 1) / BK) * BK;
    nsplit = static_cast<int>((g.K + klen - 1) / klen);
  }
  p.nsplit = nsplit;
  p.ksplit_len = std::max<int64_t>(klen, 1);
  p.partial = nsplit > 1 ? ws.p : nullptr;
  if (mt > 65535) throw Error(ERR_BAD_SHAPE, "gemm: M too large");
  if (g.batch * nsplit > 65535) throw Error(ERR_BAD_SHAPE, "gemm: batch too large");
  dim3 grid(static_cast<unsigned>(nt), static_cast<unsigned>(mt),
            static_cast<unsigned>(g.batch * nsplit));

#define CC_GEMM_DISPATCH(AK, BNC)                                   \
  if (va2 && vb2) launch<AK, BNC, 2, 2>(p, grid, s);                \
  else if (va2) launch<AK, BNC, 2, 1>(p, grid, s);                  \
  else if (vb2) launch<AK, BNC, 1, 2>(p, grid, s);                  \
  else launch<AK, BNC, 1, 1>(p, grid, s);
  if (a_kc && b_nc) { CC_GEMM_DISPATCH(true, true) }
  else if (a_kc) { CC_GEMM_DISPATCH(true, false) }
  else if (b_nc) { CC_GEMM_DISPATCH(false, true) }
  else { CC_GEMM_DISPATCH(false, false) }
#undef CC_GEMM_DISPATCH
  g_launches.fetch_add(1);
  if (nsplit > 1) {
    splitk_reduce_kernel<<<grid_for(g.batch * g.M * g.N, 256), 256, 0, s>>>(p);
    CC_LAUNCH_CHECK();
    g_launches.fetch_add(1);
  }
}

}  // namespace cc4s_b200
