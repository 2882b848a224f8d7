// Fused Lanczos kernels: one iteration of the reorthogonalised Lanczos
// recurrence (after the matvec) in four launches.
//
//   stage 1   h1 = V^H w                                   (dots)
//   stage 2   w -= V h1 ; h2 = V^H w                       (update + dots)
//   stage 3   w -= V h2 ; beta_j = ||w|| ; alpha_j = Re(h1_j + h2_j)
//   stage 4   V[:, j+1] = w / beta_j
//
// Stages 1-3 split the rows into blocks of 256; every block writes partial
// sums, and the last block to finish (ticket counter, __threadfence) reduces
// the partials in a fixed order, so results are deterministic.  The
// classical Gram-Schmidt pass is applied twice ("twice is enough",
// Giraud, Langou, Rozloznik 2005), the full reorthogonalisation that the
// restarted Lanczos of engine.cu relies on.
#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int ROWS = 128;     // rows per block (= threads per block)
constexpr int KMAX = 256;     // Krylov vectors

__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return is_last;
}

// MODE 0: dots only; MODE 1: update then dots; MODE 2: update then norm.
template <int MODE>
__global__ void __launch_bounds__(ROWS)
gs_stage_kernel(int n, int k, const cplx* __restrict__ V, long long ldv, const cplx* __restrict__ h,
                cplx* __restrict__ w, cplx* __restrict__ part, double* __restrict__ partr,
                cplx* __restrict__ out, LanczosScalars* sc, const cplx* __restrict__ h1, int j,
                unsigned* counter) {
  __shared__ cplx hs[KMAX];
  __shared__ cplx ws[ROWS];
  __shared__ double red[ROWS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = ROWS / 32;
  const int b = blockIdx.x, nblk = gridDim.x;
  const long long r0 = (long long)b * ROWS;
  const long long i = r0 + tid;
  const bool valid = i < n;
  if (MODE >= 1)
    for (int t = tid; t < k; t += ROWS) hs[t] = h[t];
  __syncthreads();
  cplx wi = valid ? w[i] : make_double2(0.0, 0.0);
  if (MODE >= 1 && valid) {
    cplx s = make_double2(0.0, 0.0);
    // four independent accumulators keep several loads of V in flight
    cplx s1 = make_double2(0.0, 0.0), s2 = s1, s3 = s1;
    int jj = 0;
    for (; jj + 4 <= k; jj += 4) {
      const cplx v0 = V[i + jj * ldv], v1 = V[i + (jj + 1) * ldv];
      const cplx v2 = V[i + (jj + 2) * ldv], v3 = V[i + (jj + 3) * ldv];
      s = cadd(s, cmul(v0, hs[jj]));
      s1 = cadd(s1, cmul(v1, hs[jj + 1]));
      s2 = cadd(s2, cmul(v2, hs[jj + 2]));
      s3 = cadd(s3, cmul(v3, hs[jj + 3]));
    }
    for (; jj < k; jj++) s = cadd(s, cmul(V[i + jj * ldv], hs[jj]));
    s = cadd(cadd(s, s1), cadd(s2, s3));
    wi = csub(wi, s);
    w[i] = wi;
  }
  ws[tid] = wi;
  __syncthreads();
  const int rows = (int)min((long long)ROWS, (long long)n - r0);
  if (MODE <= 1) {
    // part[jj * nblk + b] = sum over the block's rows of conj(V[:, jj]) w
    for (int jj = warp; jj < k; jj += nw) {
      const cplx* v = V + jj * ldv + r0;
      cplx s = make_double2(0.0, 0.0);
      for (int r = lane; r < rows; r += 32) s = cadd(s, ccmul(v[r], ws[r]));
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) part[(long long)jj * nblk + b] = s;
    }
    if (last_block(counter)) {
      for (int jj = tid; jj < k; jj += ROWS) {
        cplx s = make_double2(0.0, 0.0);
        for (int q = 0; q < nblk; q++) s = cadd(s, __ldcg(&part[(long long)jj * nblk + q]));
        out[jj] = s;
      }
      if (tid == 0) *counter = 0u;
    }
  } else {
    double s = cabs2(ws[tid]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int q = 0; q < nw; q++) t += red[q];
      partr[b] = t;
    }
    if (last_block(counter)) {
      if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < nblk; q++) t += __ldcg(&partr[q]);
        sc->beta[j] = sqrt(t);
        sc->alpha[j] = __ldcg(&h1[j].x) + __ldcg(&h[j].x);
        *counter = 0u;
      }
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
                            LanczosScalars* sc, cplx* h1, cplx* h2, unsigned* counter, Scratch& scratch) {
  MPSGPU_CHECK(j + 1 <= KMAX, MPSGPU_BAD_SHAPE, "lanczos: more than 256 Krylov vectors");
  const int k = j + 1;
  const int nblk = ceil_div(n, ROWS);
  char* ws = (char*)scratch.get((size_t)nblk * KMAX * sizeof(cplx) + (size_t)nblk * sizeof(double) + 256);
  cplx* part = (cplx*)ws;
  double* partr = (double*)(ws + (size_t)nblk * KMAX * sizeof(cplx));
  gs_stage_kernel<0><<<nblk, ROWS, 0, st.s>>>(n, k, V, ldv, nullptr, w, part, partr, h1, sc, nullptr, j, counter);
  after_launch(st);
  gs_stage_kernel<1><<<nblk, ROWS, 0, st.s>>>(n, k, V, ldv, h1, w, part, partr, h2, sc, nullptr, j, counter);
  after_launch(st);
  gs_stage_kernel<2><<<nblk, ROWS, 0, st.s>>>(n, k, V, ldv, h2, w, part, partr, nullptr, sc, h1, j, counter);
  after_launch(st);
  if (write_next) {
    const int g = std::min(ceil_div(n, 256), 148 * 8);
    scale_next_kernel<<<g, 256, 0, st.s>>>(n, w, sc, j, V + (long long)(j + 1) * ldv);
    after_launch(st);
  }
}

}  // namespace mpsgpu
