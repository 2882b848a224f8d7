// Complex FP64 GEMM on the FP64 tensor pipe (DMMA, mma.sync m8n8k4 f64).
//
// C = alpha * op(A) * op(B) + beta * Cin, batched over blockIdx.z, with
// op in {N, C (conjugate transpose), T}.  This is the contraction engine of
// every dense step on the hot path: the two GEMMs of the effective
// Hamiltonian matvec L.W.R.A (src/wrapper/multipliers/TensorMultiplier.cpp:61-93
// does them with zgemm plus explicit permutes; here the permutes are folded
// into the storage layout and the op flags), the environment updates
// (src/core/cpp/Operator.cpp:273-387), the block-reflector updates of the
// Householder QR and the absorption of R/L factors into neighbouring sites.
//
// Tiles: BM x BN complex per CTA, BK = 16 complex per stage, a WMW x WNW grid
// of warps, each warp a (BM/WMW) x (BN/WNW) tile of 8x8 DMMA fragments.
// Complex products are four real MMAs accumulated in four independent FP64
// register sets (re*re, -im*im, re*im, im*re), summed in the epilogue, so that
// consecutive MMAs of a warp do not wait on each other's accumulators.
// Operands are staged through shared memory as separate real/imaginary planes
// (padded rows: conflict-free fragment loads); the next K-slab is prefetched
// into registers while the current one is consumed.  Large-K, small-MN
// problems are split over K into a workspace and reduced by a second kernel
// that also applies the epilogue (deterministic order).  A grouped variant
// runs the tiles of many independent GEMMs (different shapes) in one
// persistent launch.
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int BK = 16;
constexpr int PAD = 4;

template <int OP>
__device__ __forceinline__ cplx load_op(const cplx* __restrict__ p, long long idx) {
  cplx v = p[idx];
  if (OP == OP_C) v.y = -v.y;
  return v;
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int BM, int BN>
struct TileSmem {
  double A_re[BK][BM + PAD], A_im[BK][BM + PAD];
  double B_re[BK][BN + PAD], B_im[BK][BN + PAD];
};

// One BM x BN output tile of op(A) op(B) over k in [kbeg, kend); result in
// the caller's accumulators acc[i][j][set][h] (set: 0 re*re, 1 -im*im,
// 2 re*im, 3 im*re).
template <int BM, int BN, int WMW, int WNW, int OPA, int OPB>
__device__ __forceinline__ void gemm_tile(const cplx* __restrict__ A, long long lda, const cplx* __restrict__ B,
                                          long long ldb, int M, int N, int m0, int n0, int kbeg, int kend,
                                          TileSmem<BM, BN>& sm,
                                          double (&acc)[BM / WMW / 8][BN / WNW / 8][4][2]) {
  constexpr int NT_ = WMW * WNW * 32;
  constexpr int WM = BM / WMW, WN = BN / WNW;
  constexpr int MT = WM / 8, NT = WN / 8;
  constexpr int AE = BM * BK / NT_;
  constexpr int BE = BN * BK / NT_;
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % WMW) * WM, wn0 = (warp / WMW) * WN;
#pragma unroll
  for (int i = 0; i < MT; i++)
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int s = 0; s < 4; s++) acc[i][j][s][0] = acc[i][j][s][1] = 0.0;

  cplx ra[AE], rb[BE];
  auto load_slab = [&](int k0) {
#pragma unroll
    for (int e = 0; e < AE; e++) {
      const int idx = tid + e * NT_;
      int m, k;
      if (OPA == OP_N) { m = idx % BM; k = idx / BM; }
      else { k = idx % BK; m = idx / BK; }
      const int gm = m0 + m, gk = k0 + k;
      cplx v = make_double2(0.0, 0.0);
      if (gm < M && gk < kend) {
        const long long off = (OPA == OP_N) ? (gm + (long long)gk * lda) : (gk + (long long)gm * lda);
        v = load_op<OPA>(A, off);
      }
      ra[e] = v;
    }
#pragma unroll
    for (int e = 0; e < BE; e++) {
      const int idx = tid + e * NT_;
      int n, k;
      if (OPB == OP_N) { k = idx % BK; n = idx / BK; }
      else { n = idx % BN; k = idx / BN; }
      const int gn = n0 + n, gk = k0 + k;
      cplx v = make_double2(0.0, 0.0);
      if (gn < N && gk < kend) {
        const long long off = (OPB == OP_N) ? (gk + (long long)gn * ldb) : (gn + (long long)gk * ldb);
        v = load_op<OPB>(B, off);
      }
      rb[e] = v;
    }
  };
  auto store_slab = [&]() {
#pragma unroll
    for (int e = 0; e < AE; e++) {
      const int idx = tid + e * NT_;
      int m, k;
      if (OPA == OP_N) { m = idx % BM; k = idx / BM; }
      else { k = idx % BK; m = idx / BK; }
      sm.A_re[k][m] = ra[e].x;
      sm.A_im[k][m] = ra[e].y;
    }
#pragma unroll
    for (int e = 0; e < BE; e++) {
      const int idx = tid + e * NT_;
      int n, k;
      if (OPB == OP_N) { k = idx % BK; n = idx / BK; }
      else { n = idx % BN; k = idx / BN; }
      sm.B_re[k][n] = rb[e].x;
      sm.B_im[k][n] = rb[e].y;
    }
  };

  const int fr = lane >> 2, fc = lane & 3;
  if (kbeg < kend) load_slab(kbeg);
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    __syncthreads();
    store_slab();
    __syncthreads();
    if (k0 + BK < kend) load_slab(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double are[MT], aim[MT], naim[MT], bre[NT], bim[NT];
#pragma unroll
      for (int i = 0; i < MT; i++) {
        are[i] = sm.A_re[kk + fc][wm0 + i * 8 + fr];
        aim[i] = sm.A_im[kk + fc][wm0 + i * 8 + fr];
        naim[i] = -aim[i];
      }
#pragma unroll
      for (int j = 0; j < NT; j++) {
        bre[j] = sm.B_re[kk + fc][wn0 + j * 8 + fr];
        bim[j] = sm.B_im[kk + fc][wn0 + j * 8 + fr];
      }
#pragma unroll
      for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++) {
          dmma(acc[i][j][0][0], acc[i][j][0][1], are[i], bre[j]);
          dmma(acc[i][j][1][0], acc[i][j][1][1], naim[i], bim[j]);
          dmma(acc[i][j][2][0], acc[i][j][2][1], are[i], bim[j]);
          dmma(acc[i][j][3][0], acc[i][j][3][1], aim[i], bre[j]);
        }
    }
  }
}

// Epilogue for accumulator element (r, c) of fragment (i, j):
// r = i*8 + lane/4, c = j*8 + 2*(lane%4) + h.
template <int BM, int BN, int WMW, int WNW>
__device__ __forceinline__ void tile_store(const double (&acc)[BM / WMW / 8][BN / WNW / 8][4][2], int M, int N,
                                           int m0, int n0, cplx alpha, const cplx* Cin, long long ldcin,
                                           cplx beta, cplx* C, long long ldc, bool raw) {
  constexpr int WM = BM / WMW, WN = BN / WNW;
  constexpr int MT = WM / 8, NT = WN / 8;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp % WMW) * WM, wn0 = (warp / WMW) * WN;
  const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
  for (int i = 0; i < MT; i++)
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int gm = m0 + wm0 + i * 8 + fr;
        const int gn = n0 + wn0 + j * 8 + 2 * fc + h;
        if (gm < M && gn < N) {
          const cplx v = make_double2(acc[i][j][0][h] + acc[i][j][1][h], acc[i][j][2][h] + acc[i][j][3][h]);
          if (raw) {
            C[gm + (long long)gn * ldc] = v;
          } else {
            cplx out = cmul(alpha, v);
            if (Cin) out = cadd(out, cmul(beta, Cin[gm + (long long)gn * ldcin]));
            C[gm + (long long)gn * ldc] = out;
          }
        }
      }
}

template <int BM, int BN, int WMW, int WNW, int OPA, int OPB>
__global__ void __launch_bounds__(WMW* WNW * 32)
zgemm_dmma_kernel(GemmArgs g, int splits, int kchunk, cplx* __restrict__ partial) {
  __shared__ TileSmem<BM, BN> sm;
  double acc[BM / WMW / 8][BN / WNW / 8][4][2];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int zb = blockIdx.z / splits, zs = blockIdx.z % splits;
  const int kbeg = zs * kchunk;
  const int kend = min(g.K, kbeg + kchunk);
  gemm_tile<BM, BN, WMW, WNW, OPA, OPB>(g.A + (long long)zb * g.strideA, g.lda, g.B + (long long)zb * g.strideB,
                                        g.ldb, g.M, g.N, m0, n0, kbeg, kend, sm, acc);
  if (splits == 1) {
    tile_store<BM, BN, WMW, WNW>(acc, g.M, g.N, m0, n0, g.alpha,
                                 g.Cin ? g.Cin + (long long)zb * g.strideCin : nullptr, g.ldcin, g.beta,
                                 g.C + (long long)zb * g.strideC, g.ldc, false);
  } else {
    cplx* P = partial + ((long long)zs * g.batch + zb) * (long long)g.M * g.N;
    tile_store<BM, BN, WMW, WNW>(acc, g.M, g.N, m0, n0, g.alpha, nullptr, 0, g.beta, P, g.M, true);
  }
}

// Grouped GEMMs (op N, N): descriptor d covers tiles [tile_begin(d), tile_begin(d+1)).
template <int BM, int BN, int WMW, int WNW>
__global__ void __launch_bounds__(WMW* WNW * 32)
zgemm_grouped_kernel(const GroupedGemm* __restrict__ descs, int ndesc, long long total_tiles) {
  __shared__ TileSmem<BM, BN> sm;
  double acc[BM / WMW / 8][BN / WNW / 8][4][2];
  for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    // binary search for the descriptor owning tile t
    int lo = 0, hi = ndesc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (descs[mid].tile_begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const GroupedGemm& d = descs[lo];
    const long long local = t - d.tile_begin;
    const int tm = (int)(local % d.tiles_m), tn = (int)(local / d.tiles_m);
    const int m0 = tm * BM, n0 = tn * BN;
    gemm_tile<BM, BN, WMW, WNW, OP_N, OP_N>(d.A, d.lda, d.B, d.ldb, d.M, d.N, m0, n0, 0, d.K, sm, acc);
    tile_store<BM, BN, WMW, WNW>(acc, d.M, d.N, m0, n0, make_double2(1.0, 0.0), nullptr, 0,
                                 make_double2(0.0, 0.0), d.C, d.ldc, false);
    __syncthreads();
  }
}

__global__ void splitk_reduce_kernel(GemmArgs g, int splits, const cplx* __restrict__ partial) {
  long long mn = (long long)g.M * g.N;
  long long total = mn * g.batch;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int zb = (int)(t / mn);
    long long e = t % mn;
    int m = (int)(e % g.M), n = (int)(e / g.M);
    cplx s = make_double2(0.0, 0.0);
    for (int z = 0; z < splits; z++) s = cadd(s, partial[((long long)z * g.batch + zb) * mn + e]);
    cplx out = cmul(g.alpha, s);
    if (g.Cin) out = cadd(out, cmul(g.beta, g.Cin[(long long)zb * g.strideCin + m + (long long)n * g.ldcin]));
    g.C[(long long)zb * g.strideC + m + (long long)n * g.ldc] = out;
  }
}

template <int BM, int BN, int WMW, int WNW>
void launch_tiles(const Stream& st, const GemmArgs& g, int splits, int kchunk, cplx* partial) {
  dim3 grid(ceil_div(g.M, BM), ceil_div(g.N, BN), g.batch * splits);
  const int threads = WMW * WNW * 32;
#define MPSGPU_GEMM_CASE(oa, ob)                                                                    \
  if (g.opA == oa && g.opB == ob) {                                                                 \
    zgemm_dmma_kernel<BM, BN, WMW, WNW, oa, ob><<<grid, threads, 0, st.s>>>(g, splits, kchunk, partial); \
    after_launch(st);                                                                               \
    return;                                                                                         \
  }
  MPSGPU_GEMM_CASE(OP_N, OP_N)
  MPSGPU_GEMM_CASE(OP_N, OP_T)
  MPSGPU_GEMM_CASE(OP_N, OP_C)
  MPSGPU_GEMM_CASE(OP_C, OP_N)
  MPSGPU_GEMM_CASE(OP_T, OP_N)
  MPSGPU_GEMM_CASE(OP_C, OP_C)
#undef MPSGPU_GEMM_CASE
  throw Error(MPSGPU_INVALID, "zgemm: unsupported op combination");
}

}  // namespace

namespace {

// Launch configuration of one GEMM: tile edge (32: 4 warps, 64: 8 warps) and
// the number of K slices.
struct GemmCfg {
  int tile = 32;
  int splits = 1;
};

// Default when no measurement is available: 64x64 tiles when they already
// fill the GPU, otherwise 32x32 plus a split over K.
GemmCfg heuristic_cfg(const GemmArgs& g) {
  const long long target = 2 * 148;
  const long long ctas64 = (long long)ceil_div(g.M, 64) * ceil_div(g.N, 64) * g.batch;
  GemmCfg c;
  c.tile = ctas64 >= target ? 64 : 32;
  const long long ctas = (long long)ceil_div(g.M, c.tile) * ceil_div(g.N, c.tile) * g.batch;
  while (c.splits < 8 && ctas * c.splits * 2 <= target && g.K / (c.splits * 2) >= 4 * BK) c.splits *= 2;
  return c;
}

void run_cfg(const Stream& st, const GemmArgs& g, GemmCfg c, Scratch& scratch) {
  int splits = c.splits;
  const int kchunk = splits > 1 ? ceil_div(ceil_div(g.K, splits), BK) * BK : g.K;
  if (splits > 1) splits = ceil_div(g.K, kchunk);
  cplx* partial = nullptr;
  if (splits > 1) partial = (cplx*)scratch.get((size_t)splits * g.batch * (size_t)g.M * g.N * sizeof(cplx));
  if (c.tile == 64) launch_tiles<64, 64, 2, 4>(st, g, splits, kchunk, partial);
  else launch_tiles<32, 32, 2, 2>(st, g, splits, kchunk, partial);
  if (splits > 1) {
    const long long total = (long long)g.M * g.N * g.batch;
    splitk_reduce_kernel<<<std::min<long long>(ceil_div(total, 256), 4096), 256, 0, st.s>>>(g, splits, partial);
    after_launch(st);
  }
}

// ---- autotuner ----------------------------------------------------------
// The first GEMM of every shape (device, M, N, K, batch, ops, epilogue) times the
// candidate configurations on its own operands, writing to a scratch output
// (C is never written twice, so aliasing of C with Cin is harmless), and the
// fastest is kept in a process-wide table that every later GEMM of that shape
// uses.  Skipped while the stream is being captured into a graph.
struct TuneKey {
  int dev, M, N, K, batch, opA, opB, cin;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, M, N, K, batch, opA, opB, cin) <
           std::tie(o.dev, o.M, o.N, o.K, o.batch, o.opA, o.opB, o.cin);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, GemmCfg> g_tune;
std::atomic<int> g_tune_mode{-1};  // -1: not read yet, 0: off, 1: on

bool autotune_enabled() {
  int m = g_tune_mode.load();
  if (m < 0) {
    const char* e = std::getenv("MPSGPU_AUTOTUNE");
    m = (e && e[0] == '0') ? 0 : 1;
    g_tune_mode.store(m);
  }
  return m == 1;
}

GemmCfg tune(const Stream& st, const GemmArgs& g, Scratch& scratch) {
  std::vector<GemmCfg> cands;
  for (int tile : {32, 64})
    for (int sp : {1, 2, 4, 8, 16}) {
      if (sp > 1 && g.K / sp < 2 * BK) continue;
      cands.push_back(GemmCfg{tile, sp});
    }
  GemmArgs t = g;
  const long long nel = (long long)(g.batch - 1) * g.strideC + g.ldc * (long long)g.N;
  cplx* tmp = nullptr;
  MPSGPU_CUDA(cudaMallocAsync((void**)&tmp, std::max<long long>(nel, 1) * sizeof(cplx), st.s));
  t.C = tmp;
  Stream quiet = st;
  quiet.prof = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  GemmCfg best = heuristic_cfg(g);
  float best_ms = 1e30f;
  try {
    MPSGPU_CUDA(cudaEventCreate(&e0));
    MPSGPU_CUDA(cudaEventCreate(&e1));
    for (const GemmCfg& c : cands) {
      run_cfg(quiet, t, c, scratch);  // warm (instruction cache, scratch size)
      MPSGPU_CUDA(cudaEventRecord(e0, st.s));
      for (int r = 0; r < 3; r++) run_cfg(quiet, t, c, scratch);
      MPSGPU_CUDA(cudaEventRecord(e1, st.s));
      MPSGPU_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      MPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFreeAsync(tmp, st.s);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MPSGPU_CUDA(cudaFreeAsync(tmp, st.s));
  return best;
}

GemmCfg choose_cfg(const Stream& st, const GemmArgs& g, Scratch& scratch) {
  if (!autotune_enabled()) return heuristic_cfg(g);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  const TuneKey key{dev, g.M, g.N, g.K, g.batch, g.opA, g.opB, g.Cin != nullptr ? 1 : 0};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st.s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return heuristic_cfg(g);
  const GemmCfg c = tune(st, g, scratch);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = c;
  return c;
}

}  // namespace

void set_gemm_autotune(int on) { g_tune_mode.store(on ? 1 : 0); }

bool gemm_autotune_on() { return autotune_enabled(); }

long long gemm_autotune_entries() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return (long long)g_tune.size();
}

void zgemm(const Stream& st, const GemmArgs& g0, Scratch& scratch) {
  GemmArgs g = g0;
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  if (g.K <= 0) {
    // C = beta * Cin (or zero)
    GemmArgs z = g;
    z.K = 0;
    long long total = (long long)g.M * g.N * g.batch;
    splitk_reduce_kernel<<<std::min<long long>(ceil_div(total, 256), 4096), 256, 0, st.s>>>(z, 0, nullptr);
    after_launch(st);
    return;
  }
  const GemmCfg cfg = choose_cfg(st, g, scratch);
  ProfScope ps(st, GemmProfiler::GEMM64, 8.0 * (double)g.M * g.N * g.K * g.batch);
  run_cfg(st, g, cfg, scratch);
}

long long grouped_tiles(GroupedGemm* descs, int n) {
  long long t = 0;
  for (int i = 0; i < n; i++) {
    descs[i].tiles_m = ceil_div(descs[i].M, 64);
    const int tiles_n = ceil_div(descs[i].N, 64);
    descs[i].tile_begin = t;
    t += (long long)descs[i].tiles_m * tiles_n;
  }
  return t;
}

void zgemm_grouped(const Stream& st, const GroupedGemm* d_descs, int n, long long total_tiles, int ctas) {
  if (n <= 0 || total_tiles <= 0) return;
  zgemm_grouped_kernel<64, 64, 2, 4><<<ctas, 256, 0, st.s>>>(d_descs, n, total_tiles);
  after_launch(st);
}

}  // namespace mpsgpu
