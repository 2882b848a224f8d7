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
// Tiles: BM x BN complex per CTA, BK = 16 complex per stage, 4 warps in a
// 2x2 grid, each warp a (BM/2)x(BN/2) tile of 8x8 DMMA fragments.  Complex
// products are four real MMAs (re*re - im*im, re*im + im*re) accumulated in
// FP64 registers.  Operands are staged through shared memory as separate
// real/imaginary planes (padded rows: conflict-free fragment loads); the next
// K-slab is prefetched into registers while the current one is consumed.
// Large-K, small-MN problems are split over K into a workspace and reduced by
// a second kernel that also applies the epilogue (deterministic order).
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

template <int BM, int BN, int OPA, int OPB>
__global__ void __launch_bounds__(128)
zgemm_dmma_kernel(GemmArgs g, int splits, int kchunk, cplx* __restrict__ partial) {
  constexpr int WM = BM / 2, WN = BN / 2;
  constexpr int MT = WM / 8, NT = WN / 8;
  constexpr int AE = BM * BK / 128;  // complex elements per thread per slab
  constexpr int BE = BN * BK / 128;
  __shared__ double As_re[BK][BM + PAD], As_im[BK][BM + PAD];
  __shared__ double Bs_re[BK][BN + PAD], Bs_im[BK][BN + PAD];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp & 1) * WM, wn0 = (warp >> 1) * WN;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int zb = blockIdx.z / splits, zs = blockIdx.z % splits;
  const int kbeg = zs * kchunk;
  const int kend = min(g.K, kbeg + kchunk);

  const cplx* A = g.A + (long long)zb * g.strideA;
  const cplx* B = g.B + (long long)zb * g.strideB;

  double acc_re[MT][NT][2], acc_im[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; i++)
#pragma unroll
    for (int j = 0; j < NT; j++) {
      acc_re[i][j][0] = acc_re[i][j][1] = 0.0;
      acc_im[i][j][0] = acc_im[i][j][1] = 0.0;
    }

  cplx ra[AE], rb[BE];
  auto load_slab = [&](int k0) {
#pragma unroll
    for (int e = 0; e < AE; e++) {
      int idx = tid + e * 128;
      int m, k;
      if (OPA == OP_N) { m = idx % BM; k = idx / BM; }
      else { k = idx % BK; m = idx / BK; }
      int gm = m0 + m, gk = k0 + k;
      cplx v = make_double2(0.0, 0.0);
      if (gm < g.M && gk < kend) {
        long long off = (OPA == OP_N) ? (gm + (long long)gk * g.lda) : (gk + (long long)gm * g.lda);
        v = load_op<OPA>(A, off);
      }
      ra[e] = v;
    }
#pragma unroll
    for (int e = 0; e < BE; e++) {
      int idx = tid + e * 128;
      int n, k;
      if (OPB == OP_N) { k = idx % BK; n = idx / BK; }
      else { n = idx % BN; k = idx / BN; }
      int gn = n0 + n, gk = k0 + k;
      cplx v = make_double2(0.0, 0.0);
      if (gn < g.N && gk < kend) {
        long long off = (OPB == OP_N) ? (gk + (long long)gn * g.ldb) : (gn + (long long)gk * g.ldb);
        v = load_op<OPB>(B, off);
      }
      rb[e] = v;
    }
  };
  auto store_slab = [&]() {
#pragma unroll
    for (int e = 0; e < AE; e++) {
      int idx = tid + e * 128;
      int m, k;
      if (OPA == OP_N) { m = idx % BM; k = idx / BM; }
      else { k = idx % BK; m = idx / BK; }
      As_re[k][m] = ra[e].x;
      As_im[k][m] = ra[e].y;
    }
#pragma unroll
    for (int e = 0; e < BE; e++) {
      int idx = tid + e * 128;
      int n, k;
      if (OPB == OP_N) { k = idx % BK; n = idx / BK; }
      else { n = idx % BN; k = idx / BN; }
      Bs_re[k][n] = rb[e].x;
      Bs_im[k][n] = rb[e].y;
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
        are[i] = As_re[kk + fc][wm0 + i * 8 + fr];
        aim[i] = As_im[kk + fc][wm0 + i * 8 + fr];
        naim[i] = -aim[i];
      }
#pragma unroll
      for (int j = 0; j < NT; j++) {
        bre[j] = Bs_re[kk + fc][wn0 + j * 8 + fr];
        bim[j] = Bs_im[kk + fc][wn0 + j * 8 + fr];
      }
#pragma unroll
      for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++) {
          dmma(acc_re[i][j][0], acc_re[i][j][1], are[i], bre[j]);
          dmma(acc_re[i][j][0], acc_re[i][j][1], naim[i], bim[j]);
          dmma(acc_im[i][j][0], acc_im[i][j][1], are[i], bim[j]);
          dmma(acc_im[i][j][0], acc_im[i][j][1], aim[i], bre[j]);
        }
    }
  }

  // Epilogue: accumulator element (r, c) of fragment (i, j):
  // r = i*8 + lane/4, c = j*8 + 2*(lane%4) + h.
  if (splits == 1) {
    cplx* C = g.C + (long long)zb * g.strideC;
    const cplx* Cin = g.Cin ? g.Cin + (long long)zb * g.strideCin : nullptr;
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
      for (int j = 0; j < NT; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          int gm = m0 + wm0 + i * 8 + fr;
          int gn = n0 + wn0 + j * 8 + 2 * fc + h;
          if (gm < g.M && gn < g.N) {
            cplx v = make_double2(acc_re[i][j][h], acc_im[i][j][h]);
            cplx out = cmul(g.alpha, v);
            if (Cin) out = cadd(out, cmul(g.beta, Cin[gm + (long long)gn * g.ldcin]));
            C[gm + (long long)gn * g.ldc] = out;
          }
        }
  } else {
    cplx* P = partial + ((long long)zs * g.batch + zb) * (long long)g.M * g.N;
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
      for (int j = 0; j < NT; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          int gm = m0 + wm0 + i * 8 + fr;
          int gn = n0 + wn0 + j * 8 + 2 * fc + h;
          if (gm < g.M && gn < g.N)
            P[gm + (long long)gn * g.M] = make_double2(acc_re[i][j][h], acc_im[i][j][h]);
        }
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

template <int BM, int BN>
void launch_tiles(const Stream& st, const GemmArgs& g, int splits, int kchunk, cplx* partial) {
  dim3 grid(ceil_div(g.M, BM), ceil_div(g.N, BN), g.batch * splits);
#define MPSGPU_GEMM_CASE(oa, ob)                                                        \
  if (g.opA == oa && g.opB == ob) {                                                     \
    zgemm_dmma_kernel<BM, BN, oa, ob><<<grid, 128, 0, st.s>>>(g, splits, kchunk, partial); \
    after_launch(st);                                                                   \
    return;                                                                             \
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

size_t zgemm_workspace_bytes(const GemmArgs& g) {
  // Upper bound used by the split-K path (splits <= 8).
  return (size_t)8 * g.batch * (size_t)g.M * g.N * sizeof(cplx);
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
  // Tile choice: large tiles when they already fill the GPU, otherwise 32x32.
  const long long target = 2 * 148;
  long long ctas64 = (long long)ceil_div(g.M, 64) * ceil_div(g.N, 64) * g.batch;
  bool big = ctas64 >= target;
  int BMs = big ? 64 : 32;
  long long ctas = (long long)ceil_div(g.M, BMs) * ceil_div(g.N, BMs) * g.batch;
  int splits = 1;
  while (splits < 8 && ctas * splits * 2 <= target && g.K / (splits * 2) >= 4 * BK) splits *= 2;
  int kchunk = splits > 1 ? ceil_div(ceil_div(g.K, splits), BK) * BK : g.K;
  if (splits > 1) splits = ceil_div(g.K, kchunk);
  cplx* partial = nullptr;
  if (splits > 1)
    partial = (cplx*)scratch.get((size_t)splits * g.batch * (size_t)g.M * g.N * sizeof(cplx));
  const bool prof = st.prof && st.prof->sample();
  if (prof) {
    cudaEvent_t e0 = st.prof->next();
    if (e0) cudaEventRecord(e0, st.s);
  }
  if (big) launch_tiles<64, 64>(st, g, splits, kchunk, partial);
  else launch_tiles<32, 32>(st, g, splits, kchunk, partial);
  if (splits > 1) {
    long long total = (long long)g.M * g.N * g.batch;
    splitk_reduce_kernel<<<std::min<long long>(ceil_div(total, 256), 4096), 256, 0, st.s>>>(g, splits, partial);
    after_launch(st);
  }
  if (prof) {
    cudaEvent_t e1 = st.prof->next();
    if (e1) cudaEventRecord(e1, st.s);
    st.prof->flops += 8.0 * (double)g.M * g.N * g.K * g.batch;
    st.prof->calls++;
  }
}

}  // namespace mpsgpu
