// Fused Lanczos kernels: one iteration of the reorthogonalised Lanczos
// recurrence after the matvec, for the basis V[:, 0..j] (k = j+1 vectors)
// and w = (H - sigma) v_j, sigma the caller's latest Ritz value.  The local
// three-term step removes the large components along v_j and v_{j-1}
// first, so that one classical Gram-Schmidt pass over V usually suffices.
//
//   local       w = w - beta_{j-1} v_{j-1} ; a = v_j^H w
//   dots<1>     h = V^H w',  w' = w - a v_j                  (|w'|^2 too)
//   update<1>   w = w' - V h ; beta^2 = |w|^2 ; if beta^2 < |w'|^2 / 2 a
//               second pass is flagged (Daniel, Gragg, Kaufman, Stewart
//               1976), else alpha_j = sigma + Re(a + h_j), beta_j are final
//   dots<2>     h2 = V^H w                   (returns at once unless flagged)
//   update<2>   w -= V h2 ; beta_j = |w| ; alpha_j += Re h2_j   (idem)
//   scale       V[:, j+1] = w / beta_j
//
// The dot kernels run on a 2-D grid (row blocks x groups of 8 basis vectors)
// so that many independent loads are in flight; every block writes partial
// sums and the last block of each group (ticket counter, __threadfence)
// reduces them, one warp per vector with lane-strided loads and a shuffle
// tree, in a fixed order: results are deterministic.  alpha_j and beta_j
// are also written to a mapped host mirror, read by the host after the
// iteration's event.
#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int RB = 256;           // rows per block (one per thread) of the local and dot kernels
constexpr int UR = 64;            // rows per block of the update kernels
constexpr int UP = RB / UR;       // threads per row there (each takes every UP-th basis vector)
constexpr int NW = RB / 32;       // warps per block
constexpr int JG = 8;             // basis vectors per block of the dot kernels (== NW)
constexpr int KMAX = 256;         // Krylov vectors
constexpr double DGKS2 = 0.5;     // second pass when |w_after|^2 < 0.5 |w_before|^2
static_assert(JG == NW, "one warp per vector in the group reduction");

struct LzArgs {
  int n, k, j, nrb;
  const cplx* V;
  long long ldv;
  cplx* w;
  cplx* part;          // k x nrb partial dots
  double* pnorm;       // nrb partial squared norms
  cplx* h;             // first-pass coefficients (k)
  cplx* h2;            // second-pass coefficients (k)
  LanczosScalars* sc;
  LanczosScalars* mirror;
  unsigned* counters;  // [0, 32) first-pass groups, [32, 64) second-pass groups, 64, 65 updates, 66 local
  double sigma;
};

__device__ __forceinline__ cplx warp_sum(cplx s) {
  for (int o = 16; o > 0; o >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
  }
  return s;
}

__device__ __forceinline__ double warp_sumd(double s) {
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// true in the last block (of gridDim.x blocks) to pass the ticket counter
__device__ __forceinline__ bool last_block(unsigned* counter, unsigned nblocks) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = (atomicAdd(counter, 1u) == nblocks - 1);
  __syncthreads();
  return is_last;
}

__global__ void __launch_bounds__(RB) lz_local_kernel(LzArgs a) {
  __shared__ cplx red[NW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long i = (long long)blockIdx.x * RB + tid;
  cplx acc = make_double2(0.0, 0.0);
  if (i < a.n) {
    cplx wi = a.w[i];
    if (a.j > 0) {
      wi = csub(wi, cscale(a.V[i + (long long)(a.j - 1) * a.ldv], a.sc->beta[a.j - 1]));
      a.w[i] = wi;
    }
    acc = ccmul(a.V[i + (long long)a.j * a.ldv], wi);
  }
  acc = warp_sum(acc);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (tid == 0) {
    cplx s = make_double2(0.0, 0.0);
    for (int q = 0; q < NW; q++) s = cadd(s, red[q]);
    a.part[blockIdx.x] = s;
  }
  if (last_block(a.counters + 66, gridDim.x)) {
    cplx s = make_double2(0.0, 0.0);
    for (int q = tid; q < a.nrb; q += RB) s = cadd(s, __ldcg(&a.part[q]));
    s = warp_sum(s);
    __syncthreads();
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
      cplx t = make_double2(0.0, 0.0);
      for (int q = 0; q < NW; q++) t = cadd(t, red[q]);
      a.sc->loc = t;
      a.counters[66] = 0u;
    }
  }
}

template <int PASS>
__global__ void __launch_bounds__(RB) lz_dots_kernel(LzArgs a) {
  if (PASS == 2 && a.sc->flag == 0) return;  // written by update<1> (earlier kernel)
  __shared__ cplx red[NW][JG];
  __shared__ double rn[NW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = blockIdx.y;
  const int j0 = g * JG;
  const bool with_norm = (PASS == 1 && g == 0);
  // row blocks in grid-stride order (the second pass launches fewer blocks)
  for (int rb = blockIdx.x; rb < a.nrb; rb += gridDim.x) {
    const long long i = (long long)rb * RB + tid;
    const bool valid = i < a.n;
    cplx wi = valid ? a.w[i] : make_double2(0.0, 0.0);
    if (PASS == 1 && valid) wi = csub(wi, cmul(a.V[i + (long long)a.j * a.ldv], a.sc->loc));
    cplx acc[JG];
#pragma unroll
    for (int u = 0; u < JG; u++) {
      const int jj = j0 + u;
      acc[u] = (valid && jj < a.k) ? ccmul(a.V[i + (long long)jj * a.ldv], wi) : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < JG; u++) acc[u] = warp_sum(acc[u]);
    if (lane == 0) {
#pragma unroll
      for (int u = 0; u < JG; u++) red[warp][u] = acc[u];
    }
    if (with_norm) {
      const double s = warp_sumd(cabs2(wi));
      if (lane == 0) rn[warp] = s;
    }
    __syncthreads();
    if (tid < JG && j0 + tid < a.k) {
      cplx s = make_double2(0.0, 0.0);
      for (int q = 0; q < NW; q++) s = cadd(s, red[q][tid]);
      a.part[(long long)(j0 + tid) * a.nrb + rb] = s;
    }
    if (with_norm && tid == 0) {
      double s = 0.0;
      for (int q = 0; q < NW; q++) s += rn[q];
      a.pnorm[rb] = s;
    }
    __syncthreads();
  }
  unsigned* counter = a.counters + (PASS == 1 ? 0 : 32) + g;
  if (last_block(counter, gridDim.x)) {
    cplx* out = PASS == 1 ? a.h : a.h2;
    const int jj = j0 + warp;
    if (jj < a.k) {
      const cplx* pj = a.part + (long long)jj * a.nrb;
      cplx s = make_double2(0.0, 0.0);
      for (int q = lane; q < a.nrb; q += 32) s = cadd(s, __ldcg(&pj[q]));
      s = warp_sum(s);
      if (lane == 0) out[jj] = s;
    }
    if (with_norm && warp == 0) {
      double s = 0.0;
      for (int q = lane; q < a.nrb; q += 32) s += __ldcg(&a.pnorm[q]);
      s = warp_sumd(s);
      if (lane == 0) a.sc->nb2 = s;
    }
    if (tid == 0) *counter = 0u;
  }
}

template <int PASS>
__global__ void __launch_bounds__(RB) lz_update_kernel(LzArgs a) {
  if (PASS == 2 && a.sc->flag == 0) return;
  __shared__ cplx hs[KMAX];
  __shared__ double rn[NW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ cplx sp[UP][UR];
  const cplx* h = PASS == 1 ? a.h : a.h2;
  for (int t = tid; t < a.k; t += RB) hs[t] = h[t];
  __syncthreads();
  // UP threads per row: thread (r, p) sums V[i, jj] h[jj] over jj = p mod UP
  // with four independent accumulators, so that each row has 4 * UP loads
  // of V in flight and the grid has UP times more warps
  const int r = tid % UR, p = tid / UR;
  const int nub = (a.n + UR - 1) / UR;
  double bsum = 0.0;  // this block's sum of squares (thread 0)
  for (int ub = blockIdx.x; ub < nub; ub += gridDim.x) {
    const long long i = (long long)ub * UR + r;
    const bool valid = i < a.n;
    {
      cplx s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0, s3 = s0;
      if (valid) {
        int jj = p;
        for (; jj + 3 * UP < a.k; jj += 4 * UP) {
          s0 = cadd(s0, cmul(a.V[i + (long long)jj * a.ldv], hs[jj]));
          s1 = cadd(s1, cmul(a.V[i + (long long)(jj + UP) * a.ldv], hs[jj + UP]));
          s2 = cadd(s2, cmul(a.V[i + (long long)(jj + 2 * UP) * a.ldv], hs[jj + 2 * UP]));
          s3 = cadd(s3, cmul(a.V[i + (long long)(jj + 3 * UP) * a.ldv], hs[jj + 3 * UP]));
        }
        for (; jj < a.k; jj += UP) s0 = cadd(s0, cmul(a.V[i + (long long)jj * a.ldv], hs[jj]));
      }
      sp[p][r] = cadd(cadd(s0, s1), cadd(s2, s3));
    }
    __syncthreads();
    double nrm = 0.0;
    if (p == 0 && valid) {
      cplx wi = a.w[i];
      if (PASS == 1) wi = csub(wi, cmul(a.V[i + (long long)a.j * a.ldv], a.sc->loc));
      cplx t = sp[0][r];
      for (int q = 1; q < UP; q++) t = cadd(t, sp[q][r]);
      wi = csub(wi, t);
      a.w[i] = wi;
      nrm = cabs2(wi);
    }
    nrm = warp_sumd(nrm);
    if (lane == 0) rn[warp] = nrm;
    __syncthreads();
    if (tid == 0)
      for (int q = 0; q < NW; q++) bsum += rn[q];
    __syncthreads();
  }
  if (tid == 0) a.pnorm[blockIdx.x] = bsum;
  unsigned* counter = a.counters + 63 + PASS;
  if (last_block(counter, gridDim.x)) {
    double s = 0.0;
    for (int q = tid; q < (int)gridDim.x; q += RB) s += __ldcg(&a.pnorm[q]);
    s = warp_sumd(s);
    __syncthreads();
    if (lane == 0) rn[warp] = s;
    __syncthreads();
    if (tid == 0) {
      double b2 = 0.0;
      for (int q = 0; q < NW; q++) b2 += rn[q];
      LanczosScalars* sc = a.sc;
      const int j = a.j;
      bool final_now = true;
      double alpha;
      if (PASS == 1) {
        const double ap = sc->loc.x + __ldcg(&a.h[j].x);
        if (b2 < DGKS2 * sc->nb2) {
          sc->flag = 1;
          sc->ap = ap;
          final_now = false;
        } else {
          sc->flag = 0;
        }
        alpha = a.sigma + ap;
      } else {
        alpha = a.sigma + sc->ap + __ldcg(&a.h2[j].x);
      }
      if (final_now) {
        const double beta = sqrt(b2);
        sc->alpha[j] = alpha;
        sc->beta[j] = beta;
        if (a.mirror) {  // mapped host memory: visible to the host once the kernel is complete
          a.mirror->alpha[j] = alpha;
          a.mirror->beta[j] = beta;
        }
      }
      *counter = 0u;
    }
  }
}

__global__ void scale_next_kernel(int n, const cplx* __restrict__ w, const LanczosScalars* sc, int j,
                                  cplx* __restrict__ vnext) {
  const double inv = 1.0 / sc->beta[j];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    vnext[i] = cscale(w[i], inv);
}

}  // namespace

void lanczos_orthonormalize(const Stream& st, int n, int j, cplx* V, long long ldv, cplx* w, bool write_next,
                            double sigma, LanczosScalars* sc, LanczosScalars* mirror, cplx* h1, cplx* h2,
                            unsigned* counters, Scratch& scratch) {
  MPSGPU_CHECK(j + 1 <= KMAX, MPSGPU_BAD_SHAPE, "lanczos: more than 256 Krylov vectors");
  LzArgs a;
  a.n = n; a.k = j + 1; a.j = j;
  a.nrb = ceil_div(n, RB);
  a.V = V; a.ldv = ldv; a.w = w;
  const int nub = ceil_div(n, UR);  // blocks of the update kernels
  char* ws = (char*)scratch.get((size_t)a.nrb * a.k * sizeof(cplx) + (size_t)nub * sizeof(double) + 256);
  a.part = (cplx*)ws;
  a.pnorm = (double*)(ws + (size_t)a.nrb * a.k * sizeof(cplx));
  a.h = h1; a.h2 = h2;
  a.sc = sc; a.mirror = mirror;
  a.counters = counters;
  a.sigma = sigma;
  const dim3 g2(a.nrb, ceil_div(a.k, JG));
  lz_local_kernel<<<a.nrb, RB, 0, st.s>>>(a);
  after_launch(st);
  lz_dots_kernel<1><<<g2, RB, 0, st.s>>>(a);
  after_launch(st);
  lz_update_kernel<1><<<nub, RB, 0, st.s>>>(a);
  after_launch(st);
  // the second pass is usually skipped (flag clear): few blocks, grid-stride
  const dim3 g2b(std::min(a.nrb, 16), ceil_div(a.k, JG));
  lz_dots_kernel<2><<<g2b, RB, 0, st.s>>>(a);
  after_launch(st);
  lz_update_kernel<2><<<std::min(nub, 64), RB, 0, st.s>>>(a);
  after_launch(st);
  if (write_next) {
    const int g = std::min(ceil_div(n, 256), 148 * 8);
    scale_next_kernel<<<g, 256, 0, st.s>>>(n, w, sc, j, V + (long long)(j + 1) * ldv);
    after_launch(st);
  }
}

}  // namespace mpsgpu
