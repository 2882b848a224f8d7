// The two contractions of the effective-Hamiltonian product L.W.R.x
// (src/wrapper/multipliers/TensorMultiplier.cpp:61-93, three zgemm calls
// and three full permutes there) and of the environment updates
// (src/core/cpp/Operator.cpp:273-387), as two kernels on the FP64 tensor
// pipe (DMMA, mma.sync m8n8k4 f64):
//
//   heff_gemm1w   T2 = W . (A B): the product C = A B with the rows of a CTA
//                 tile chosen as (x, i0) -> row x + X i0 and the columns as
//                 (i1, y) -> column i1 + n_i1 y, so that every "pixel" (x, y)
//                 of the tile holds all n_i0 n_i1 values the MPO-leg matrix
//                 Wm contracts; the epilogue applies Wm per pixel from shared
//                 memory and writes T2 with arbitrary strides.  The
//                 intermediate A B never reaches global memory.
//   heff_gemm3    C = alpha (A1 B1 [+ A2 B2]) + beta Cin: the K range (two
//                 sources concatenated along K for the Hermitian multiplier)
//                 is split over the CTAs of a thread-block cluster, whose
//                 partial tiles are summed through distributed shared memory
//                 in rank order (deterministic, no second kernel).
//
// Both take a group of independent problems (different shapes) in one
// launch; tiles of all problems are numbered consecutively.  Operands are
// streamed through a three-stage shared-memory ring filled by cp.async
// (16-byte copies, zero-fill beyond the edges); complex entries stay
// interleaved in shared memory and each product is four real DMMAs in
// independent accumulators (re.re, -im.im, re.im, im.re).
#include <cooperative_groups.h>

#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mpsgpu {

namespace {

constexpr int BK = 16;
constexpr int PADC = 2;      // complex padding of a shared row: conflict-free 16-byte fragment loads
constexpr int STAGES = 3;
// Warp groups splitting the k steps of every slab: two for 32-row tiles
// (twice the warps per SM for the small sweep shapes), one for 64-row
// tiles (whose accumulators already fill the registers); each group is 4
// warps, 2 x 2 over the tile.
template <int BM>
__host__ __device__ constexpr int kgroups() { return BM <= 32 ? 2 : 1; }
template <int BM>
__host__ __device__ constexpr int nthreads() { return 128 * kgroups<BM>(); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int BM, int BN>
struct Ring {
  cplx A[STAGES][BK][BM + PADC];
  cplx B[STAGES][BK][BN + PADC];
};

template <int BM, int BN>
constexpr size_t ring_bytes() {
  return sizeof(Ring<BM, BN>) > (size_t)BM * (BN + PADC) * sizeof(cplx) ? sizeof(Ring<BM, BN>)
                                                                       : (size_t)BM * (BN + PADC) * sizeof(cplx);
}

// Accumulators of a warp tile: [MT][NT][set][half]
template <int BM, int BN>
struct Acc {
  static constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 8, NT = WN / 8;
  double v[MT][NT][4][2];
};

// Main loop over k in [kbeg, kend): loadA(ring, stage, k0) / loadB(...)
// issue the cp.async copies of one BK slab.
template <int BM, int BN, class LA, class LB>
__device__ __forceinline__ void mainloop(Ring<BM, BN>& r, Acc<BM, BN>& acc, int kbeg, int kend, LA loadA, LB loadB) {
  using AC = Acc<BM, BN>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp & 1) * AC::WM, wn0 = ((warp >> 1) & 1) * AC::WN, kg = warp >> 2;
  const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
  for (int i = 0; i < AC::MT; i++)
#pragma unroll
    for (int j = 0; j < AC::NT; j++)
#pragma unroll
      for (int s = 0; s < 4; s++) acc.v[i][j][s][0] = acc.v[i][j][s][1] = 0.0;
  const int nslab = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nslab) {
      loadA(r, s, kbeg + s * BK);
      loadB(r, s, kbeg + s * BK);
    }
    cp_async_commit();
  }
  for (int it = 0; it < nslab; it++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int nx = it + STAGES - 1;
    if (nx < nslab) {
      loadA(r, nx % STAGES, kbeg + nx * BK);
      loadB(r, nx % STAGES, kbeg + nx * BK);
    }
    cp_async_commit();
    const int st = it % STAGES;
#pragma unroll
    for (int kk0 = 0; kk0 < BK; kk0 += 4 * kgroups<BM>()) {
      const int kk = kk0 + 4 * kg;  // this group's k step of the slab
      double are[AC::MT], aim[AC::MT], naim[AC::MT], bre[AC::NT], bim[AC::NT];
#pragma unroll
      for (int i = 0; i < AC::MT; i++) {
        const cplx a = r.A[st][kk + fc][wm0 + i * 8 + fr];
        are[i] = a.x;
        aim[i] = a.y;
        naim[i] = -a.y;
      }
#pragma unroll
      for (int j = 0; j < AC::NT; j++) {
        const cplx b = r.B[st][kk + fc][wn0 + j * 8 + fr];
        bre[j] = b.x;
        bim[j] = b.y;
      }
#pragma unroll
      for (int i = 0; i < AC::MT; i++)
#pragma unroll
        for (int j = 0; j < AC::NT; j++) {
          dmma(acc.v[i][j][0][0], acc.v[i][j][0][1], are[i], bre[j]);
          dmma(acc.v[i][j][1][0], acc.v[i][j][1][1], naim[i], bim[j]);
          dmma(acc.v[i][j][2][0], acc.v[i][j][2][1], are[i], bim[j]);
          dmma(acc.v[i][j][3][0], acc.v[i][j][3][1], aim[i], bre[j]);
        }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// Accumulators -> shared tile Cs[m][n] (ld BN + PADC): the warp groups'
// partial sums added in group order.  Every thread of the block calls it.
template <int BM, int BN>
__device__ __forceinline__ void acc_to_smem(const Acc<BM, BN>& acc, cplx* Cs) {
  using AC = Acc<BM, BN>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp & 1) * AC::WM, wn0 = ((warp >> 1) & 1) * AC::WN, kg = warp >> 2;
  const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
  for (int g = 0; g < kgroups<BM>(); g++) {
    if (kg == g) {
#pragma unroll
      for (int i = 0; i < AC::MT; i++)
#pragma unroll
        for (int j = 0; j < AC::NT; j++)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int m = wm0 + i * 8 + fr, n = wn0 + j * 8 + 2 * fc + h;
            const cplx v =
                make_double2(acc.v[i][j][0][h] + acc.v[i][j][1][h], acc.v[i][j][2][h] + acc.v[i][j][3][h]);
            cplx& c = Cs[m * (BN + PADC) + n];
            c = g == 0 ? v : cadd(c, v);
          }
    }
    __syncthreads();
  }
}

// tile t -> problem index (descriptors hold consecutive tile ranges)
template <class D>
__device__ __forceinline__ int problem_of(const D* d, int n, int t) {
  int q = 0;
  while (q + 1 < n && d[q + 1].tile_begin <= t) q++;
  return q;
}

// ---------------------------------------------------------------------------
// heff_gemm1w
// ---------------------------------------------------------------------------
template <int BM, int BN>
__global__ void __launch_bounds__(nthreads<BM>()) heff_gemm1w_kernel(const __grid_constant__ Gemm1wBatch b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NT_ = nthreads<BM>();
  Ring<BM, BN>& ring = *reinterpret_cast<Ring<BM, BN>*>(smem_raw);
  const int q = problem_of(b.d, b.n, blockIdx.x);
  const Gemm1wDesc& d = b.d[q];
  const int local = blockIdx.x - d.tile_begin;
  const int TX = BM / d.n_i0, TY = BN / d.n_i1;
  const int tx = local % d.tiles_x, ty = local / d.tiles_x;
  const int x0 = tx * TX, y0 = ty * TY;
  const int tid = threadIdx.x;
  // the (row, k) and (k, column) slots this thread copies are the same in
  // every slab: their row/column offsets are computed once (-1 = outside)
  constexpr int AE = BM * BK / NT_, BE = BN * BK / NT_;
  long long aoff[AE], boff[BE];
#pragma unroll
  for (int u = 0; u < AE; u++) {
    const int mt = (tid + u * NT_) % BM;
    const int xl = mt % TX, i0 = mt / TX, x = x0 + xl;
    aoff[u] = (i0 < d.n_i0 && x < d.X) ? x + (long long)d.X * i0 : -1;
  }
  {
    const int ncols = min(TY, d.Y - y0) * d.n_i1;
#pragma unroll
    for (int u = 0; u < BE; u++) {
      const int nt = (tid + u * NT_) / BK;
      boff[u] = nt < ncols ? ((long long)d.n_i1 * y0 + nt) * d.ldb : -1;
    }
  }
  auto loadA = [&](Ring<BM, BN>& r, int st, int k0) {
#pragma unroll
    for (int u = 0; u < AE; u++) {
      const int e = tid + u * NT_;
      const int mt = e % BM, kk = e / BM;
      const int k = k0 + kk;
      const bool ok = aoff[u] >= 0 && k < d.K;
      cp_async16(&r.A[st][kk][mt], ok ? d.A + aoff[u] + (long long)k * d.lda : d.A, ok);
    }
  };
  auto loadB = [&](Ring<BM, BN>& r, int st, int k0) {
#pragma unroll
    for (int u = 0; u < BE; u++) {
      const int e = tid + u * NT_;
      const int kk = e % BK, nt = e / BK;
      const int k = k0 + kk;
      const bool ok = boff[u] >= 0 && k < d.K;
      cp_async16(&r.B[st][kk][nt], ok ? d.B + k + boff[u] : d.B, ok);
    }
  };
  Acc<BM, BN> acc;
  mainloop<BM, BN>(ring, acc, 0, d.K, loadA, loadB);
  cplx* Cs = reinterpret_cast<cplx*>(smem_raw);
  acc_to_smem<BM, BN>(acc, Cs);
  __syncthreads();
  // per pixel (x, y): out[o0 + n_o0 o1] = sum_{i0, i1} Wm[o, i0 + n_i0 i1] C[(x, i0), (i1, y)]
  const int nin = d.n_i0 * d.n_i1, nout = d.n_o0 * d.n_o1;
  const int npix = TX * TY;
  for (int p = tid; p < npix * nout; p += NT_) {
    const int o = p / npix, pix = p % npix;
    const int xl = pix % TX, yl = pix / TX;
    const int x = x0 + xl, y = y0 + yl;
    if (x >= d.X || y >= d.Y) continue;
    cplx s = make_double2(0.0, 0.0);
    const cplx* wrow = d.Wm + o;
    for (int i = 0; i < nin; i++) {
      const int i0 = i % d.n_i0, i1 = i / d.n_i0;
      const cplx c = Cs[(xl + TX * i0) * (BN + PADC) + (i1 + d.n_i1 * yl)];
      s = cadd(s, cmul(__ldg(&wrow[(long long)nout * i]), c));
    }
    const int o0 = o % d.n_o0, o1 = o / d.n_o0;
    d.out[x * d.ox + y * d.oy + o0 * d.so0 + o1 * d.so1] = s;
  }
}

// ---------------------------------------------------------------------------
// heff_gemm3 (cluster split-K)
// ---------------------------------------------------------------------------
template <int BM, int BN, int CS>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(nthreads<BM>())
    heff_gemm3_kernel(const __grid_constant__ Gemm3Batch b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NT_ = nthreads<BM>();
  Ring<BM, BN>& ring = *reinterpret_cast<Ring<BM, BN>*>(smem_raw);
  const int tile = blockIdx.x / CS, rank = blockIdx.x % CS;
  const int q = problem_of(b.d, b.n, tile);
  const Gemm3Desc& d = b.d[q];
  const int local = tile - d.tile_begin;
  const int tm = local % d.tiles_m, tn = local / d.tiles_m;
  const int m0 = tm * BM, n0 = tn * BN;
  const int Ktot = d.K1 + d.K2;
  const int chunk = ((Ktot + CS - 1) / CS + BK - 1) / BK * BK;
  const int kbeg = min(Ktot, rank * chunk), kend = min(Ktot, kbeg + chunk);
  const int tid = threadIdx.x;
  auto loadA = [&](Ring<BM, BN>& r, int st, int k0) {
#pragma unroll
    for (int e = tid; e < BM * BK; e += NT_) {
      const int mt = e % BM, kk = e / BM;
      const int m = m0 + mt, k = k0 + kk;
      const bool ok = m < d.M && k < kend;
      const cplx* src = d.A1;
      if (ok) src = k < d.K1 ? d.A1 + m + (long long)k * d.lda1 : d.A2 + m + (long long)(k - d.K1) * d.lda2;
      cp_async16(&r.A[st][kk][mt], src, ok);
    }
  };
  auto loadB = [&](Ring<BM, BN>& r, int st, int k0) {
#pragma unroll
    for (int e = tid; e < BN * BK; e += NT_) {
      const int kk = e % BK, nt = e / BK;
      const int n = n0 + nt, k = k0 + kk;
      const bool ok = n < d.N && k < kend;
      const cplx* src = d.B1;
      if (ok) src = k < d.K1 ? d.B1 + k + (long long)n * d.ldb1 : d.B2 + (k - d.K1) + (long long)n * d.ldb2;
      cp_async16(&r.B[st][kk][nt], src, ok);
    }
  };
  Acc<BM, BN> acc;
  mainloop<BM, BN>(ring, acc, kbeg, kend, loadA, loadB);
  cplx* Cs = reinterpret_cast<cplx*>(smem_raw);
  acc_to_smem<BM, BN>(acc, Cs);
  // rows [r0, r1) of the tile are finished by this rank: the sum over the
  // ranks' partial tiles in rank order, then the epilogue
  constexpr int RPR = BM / CS;
  const int r0 = rank * RPR;
  if (CS > 1) {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    for (int e = tid; e < RPR * BN; e += NT_) {
      const int mt = r0 + e / BN, nt = e % BN;
      const int m = m0 + mt, n = n0 + nt;
      cplx s = make_double2(0.0, 0.0);
#pragma unroll
      for (int rr = 0; rr < CS; rr++) {
        const cplx* peer = cl.map_shared_rank(Cs, rr);
        s = cadd(s, peer[mt * (BN + PADC) + nt]);
      }
      if (m < d.M && n < d.N) {
        cplx out = cmul(d.alpha, s);
        if (d.Cin) out = cadd(out, cmul(d.beta, d.Cin[m + (long long)n * d.ldcin]));
        d.C[m + (long long)n * d.ldc] = out;
      }
    }
    cl.sync();  // peers' shared tiles stay alive until every rank has read them
  } else {
    __syncthreads();
    for (int e = tid; e < BM * BN; e += NT_) {
      const int mt = e % BM, nt = e / BM;
      const int m = m0 + mt, n = n0 + nt;
      if (m < d.M && n < d.N) {
        cplx out = cmul(d.alpha, Cs[mt * (BN + PADC) + nt]);
        if (d.Cin) out = cadd(out, cmul(d.beta, d.Cin[m + (long long)n * d.ldcin]));
        d.C[m + (long long)n * d.ldc] = out;
      }
    }
  }
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  MPSGPU_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

std::atomic<unsigned long long> g_heff_setup{0};
std::mutex g_heff_mu;

void heff_setup() {
  if (!device_needs_setup(g_heff_setup)) return;
  std::lock_guard<std::mutex> lk(g_heff_mu);
  set_smem(heff_gemm1w_kernel<64, 32>, ring_bytes<64, 32>());
  set_smem(heff_gemm1w_kernel<32, 32>, ring_bytes<32, 32>());
  set_smem(heff_gemm3_kernel<64, 32, 1>, ring_bytes<64, 32>());
  set_smem(heff_gemm3_kernel<64, 32, 2>, ring_bytes<64, 32>());
  set_smem(heff_gemm3_kernel<64, 32, 4>, ring_bytes<64, 32>());
  set_smem(heff_gemm3_kernel<64, 32, 8>, ring_bytes<64, 32>());
  set_smem(heff_gemm3_kernel<32, 32, 1>, ring_bytes<32, 32>());
  set_smem(heff_gemm3_kernel<32, 32, 2>, ring_bytes<32, 32>());
  set_smem(heff_gemm3_kernel<32, 32, 4>, ring_bytes<32, 32>());
  set_smem(heff_gemm3_kernel<32, 32, 8>, ring_bytes<32, 32>());
  mark_device_done(g_heff_setup);
}

int sm_count() {
  static std::atomic<int> n{0};
  int v = n.load();
  if (v == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      v = 148;
    n.store(v);
  }
  return v;
}

}  // namespace

void heff_gemm1w(const Stream& st, Gemm1wBatch& b) {
  MPSGPU_CHECK(b.n >= 1 && b.n <= GEMM_MAXP, MPSGPU_BAD_SHAPE, "gemm1w: group size");
  heff_setup();
  // tile rows: 32 (two warp groups splitting the k steps, twice the warps per
  // SM), measured faster for the grouped products of lockstep batches of 8
  // chains at D = 128 as well as for one chain; 64 only for groups that fill
  // the GPU many times over
  long long t64 = 0;
  for (int q = 0; q < b.n; q++) {
    const Gemm1wDesc& d = b.d[q];
    MPSGPU_CHECK(d.n_i0 >= 1 && d.n_i0 <= 32 && d.n_i1 >= 1 && d.n_i1 <= 32 && d.X > 0 && d.Y > 0 && d.K > 0,
                 MPSGPU_BAD_SHAPE, "gemm1w: leg dimensions");
    t64 += (long long)ceil_div(d.X, 64 / d.n_i0) * ceil_div(d.Y, 32 / d.n_i1);
  }
  const int bm = t64 >= 16LL * sm_count() ? 64 : 32;
  int tiles = 0;
  for (int q = 0; q < b.n; q++) {
    Gemm1wDesc& d = b.d[q];
    MPSGPU_CHECK(bm / d.n_i0 >= 1 && 32 / d.n_i1 >= 1, MPSGPU_BAD_SHAPE, "gemm1w: MPO legs wider than a tile");
    d.tiles_x = ceil_div(d.X, bm / d.n_i0);
    d.tiles_y = ceil_div(d.Y, 32 / d.n_i1);
    d.tile_begin = tiles;
    tiles += d.tiles_x * d.tiles_y;
  }
  double work = 0.0;  // GEMM flops plus the MPO-leg epilogue
  for (int q = 0; q < b.n; q++) {
    const Gemm1wDesc& d = b.d[q];
    const double nin = (double)d.n_i0 * d.n_i1, nout = (double)d.n_o0 * d.n_o1;
    work += 8.0 * ((double)d.X * d.n_i0 * d.Y * d.n_i1 * d.K + (double)d.X * d.Y * nout * nin);
  }
  ProfScope ps(st, GemmProfiler::GEMM64, work);
  if (bm == 64)
    heff_gemm1w_kernel<64, 32><<<tiles, nthreads<64>(), ring_bytes<64, 32>(), st.s>>>(b);
  else
    heff_gemm1w_kernel<32, 32><<<tiles, nthreads<32>(), ring_bytes<32, 32>(), st.s>>>(b);
  after_launch(st);
}

void heff_gemm3(const Stream& st, Gemm3Batch& b) {
  MPSGPU_CHECK(b.n >= 1 && b.n <= GEMM_MAXP, MPSGPU_BAD_SHAPE, "gemm3: group size");
  heff_setup();
  const int nsm = sm_count();
  // tile rows and split-K: the largest K chunk that still gives about one
  // CTA per SM
  long long t64 = 0, t32 = 0;
  int kmax = 0;
  for (int q = 0; q < b.n; q++) {
    const Gemm3Desc& d = b.d[q];
    MPSGPU_CHECK(d.M > 0 && d.N > 0 && d.K1 > 0 && d.K2 >= 0, MPSGPU_BAD_SHAPE, "gemm3: shape");
    t64 += (long long)ceil_div(d.M, 64) * ceil_div(d.N, 32);
    t32 += (long long)ceil_div(d.M, 32) * ceil_div(d.N, 32);
    kmax = std::max(kmax, d.K1 + d.K2);
  }
  // 64-row tiles (two CTAs per SM by shared memory) once they alone fill the
  // GPU twice; otherwise 32-row tiles (four per SM), with the K range split
  // over a cluster while that keeps within one wave and K chunks of at
  // least four slabs
  int bm = 64, cs = 1;
  if (t64 < 2LL * nsm) {
    bm = 32;
    while (cs < 8 && t32 * cs * 2 <= 4LL * nsm && kmax / (cs * 2) >= 4 * BK) cs *= 2;
  }
  int tiles = 0;
  for (int q = 0; q < b.n; q++) {
    Gemm3Desc& d = b.d[q];
    d.tiles_m = ceil_div(d.M, bm);
    d.tiles_n = ceil_div(d.N, 32);
    d.tile_begin = tiles;
    tiles += d.tiles_m * d.tiles_n;
  }
  const dim3 grid(tiles * cs);
  double work = 0.0;
  for (int q = 0; q < b.n; q++) work += 8.0 * (double)b.d[q].M * b.d[q].N * (b.d[q].K1 + b.d[q].K2);
  ProfScope ps(st, GemmProfiler::GEMM64, work);
#define MPSGPU_G3(BMv, CSv)                                                                   \
  heff_gemm3_kernel<BMv, 32, CSv><<<grid, nthreads<BMv>(), ring_bytes<BMv, 32>(), st.s>>>(b)
  if (bm == 64) {
    MPSGPU_G3(64, 1);
  } else if (cs == 1) {
    MPSGPU_G3(32, 1);
  } else if (cs == 2) {
    MPSGPU_G3(32, 2);
  } else if (cs == 4) {
    MPSGPU_G3(32, 4);
  } else {
    MPSGPU_G3(32, 8);
  }
#undef MPSGPU_G3
  after_launch(st);
}

}  // namespace mpsgpu
