// Singular values of a small complex matrix by one-sided Jacobi (Hestenes
// 1958; the complex form of Demmel & Veselic 1992): the columns of A are
// rotated pairwise until every pair is orthogonal to working precision;
// the singular values are then the column norms.  One CTA of 1024 threads
// processes the whole matrix (L2-resident workspace, column-major), one warp
// per column pair of the round-robin (tournament) ordering, so a sweep is
// n-1 steps of n/2 independent rotations.
//
// Used for the Schmidt values / entanglement entropy of a bond
// (Contractor::getSchmidtValues / getEntropy, Contractor.cpp:2045-2076 and
// :2243-2270: there the eigenvalues of the reduced density matrix; here the
// squares of the singular values of the bond matrix, which are the same
// numbers and carry full relative accuracy for the small ones).
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int JT = 1024;
constexpr int MAX_SWEEPS = 40;

__device__ __forceinline__ cplx warp_sum(cplx v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

__device__ __forceinline__ double warp_sumd(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// A: m x n (n even, column-major, ld m), rotated in place.  out: n column
// norms.  status[0] = sweeps used (MAX_SWEEPS + 1 if not converged).
__global__ void __launch_bounds__(JT) jacobi_sv_kernel(int m, int n, cplx* A, double* out, int* status) {
  __shared__ int rotated;
  __shared__ int perm[512];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = JT / 32;
  const double tol = 1e-15;
  int sweep = 0;
  for (sweep = 0; sweep < MAX_SWEEPS; sweep++) {
    if (threadIdx.x == 0) rotated = 0;
    for (int t = threadIdx.x; t < n; t += JT) perm[t] = t;
    __syncthreads();
    for (int step = 0; step < n - 1; step++) {
      // round-robin pairing: position k pairs with n-1-k; perm rotates all but slot 0
      for (int pr = warp; pr < n / 2; pr += nw) {
        const int p = perm[pr], q = perm[n - 1 - pr];
        cplx* ap = A + (long long)p * m;
        cplx* aq = A + (long long)q * m;
        double al = 0.0, be = 0.0;
        cplx ga = make_double2(0.0, 0.0);
        for (int r = lane; r < m; r += 32) {
          const cplx x = ap[r], y = aq[r];
          al += cabs2(x);
          be += cabs2(y);
          ga = cadd(ga, ccmul(x, y));
        }
        al = warp_sumd(al);
        be = warp_sumd(be);
        ga = warp_sum(ga);
        const double g = sqrt(cabs2(ga));
        if (g > tol * sqrt(al * be) && g > 1e-300) {
          // rotate (a_p, a_q conj(phase)) so that the pair becomes orthogonal
          const double zeta = (be - al) / (2.0 * g);
          const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
          const cplx ph = make_double2(ga.x / g, -ga.y / g);  // conj(gamma)/|gamma|
          for (int r = lane; r < m; r += 32) {
            const cplx x = ap[r];
            const cplx y = cmul(aq[r], ph);
            ap[r] = make_double2(cs * x.x - sn * y.x, cs * x.y - sn * y.y);
            aq[r] = make_double2(sn * x.x + cs * y.x, sn * x.y + cs * y.y);
          }
          if (lane == 0) rotated = 1;
        }
      }
      __syncthreads();
      // rotate perm[1..n-1] by one position
      if (threadIdx.x == 0) {
        const int last = perm[n - 1];
        for (int k = n - 1; k > 1; k--) perm[k] = perm[k - 1];
        perm[1] = last;
      }
      __syncthreads();
    }
    __syncthreads();
    if (!rotated) break;
    __syncthreads();
  }
  // column norms with the largest magnitude factored out, so that singular
  // values below 1e-154 (squares below the FP64 normal range) keep their
  // relative accuracy
  for (int col = warp; col < n; col += nw) {
    const cplx* a = A + (long long)col * m;
    double mx = 0.0;
    for (int r = lane; r < m; r += 32) mx = fmax(mx, fmax(fabs(a[r].x), fabs(a[r].y)));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    double s = 0.0;
    if (mx > 0.0) {
      const double inv = 1.0 / mx;
      for (int r = lane; r < m; r += 32) {
        const double u = a[r].x * inv, v = a[r].y * inv;
        s += u * u + v * v;
      }
    }
    s = warp_sumd(s);
    if (lane == 0) out[col] = mx * sqrt(s);
  }
  if (threadIdx.x == 0) status[0] = sweep < MAX_SWEEPS ? sweep + 1 : MAX_SWEEPS + 1;
}

}  // namespace

// Singular values (descending) of the m x n matrix at A (device, ld m);
// A is not modified.  Host-synchronous (returns the values on the host).
std::vector<double> singular_values(const Stream& st, int m, int n, const cplx* A, long long lda,
                                    Scratch& scratch) {
  MPSGPU_CHECK(m > 0 && n > 0, MPSGPU_BAD_SHAPE, "singular_values: empty matrix");
  // work on the orientation with at most as many columns as rows
  const bool tr = n > m;
  const int rows = tr ? n : m;
  int cols = tr ? m : n;
  const int colsp = cols + (cols & 1);  // even number of columns (zero column added)
  MPSGPU_CHECK(colsp <= 512 && rows <= 4096, MPSGPU_BAD_SHAPE, "singular_values: matrix too large");
  char* ws = (char*)scratch.get((size_t)rows * colsp * sizeof(cplx) + colsp * sizeof(double) + 64);
  cplx* W = (cplx*)ws;
  double* d_out = (double*)(ws + (size_t)rows * colsp * sizeof(cplx));
  int* d_status = (int*)(d_out + colsp);
  View2 v;
  if (!tr) { v.rd = 1; v.r0 = 0; v.r1 = 1; v.cd = 1; v.c0 = 0; v.c1 = lda; }
  else { v.rd = 1; v.r0 = 0; v.r1 = lda; v.cd = 1; v.c0 = 0; v.c1 = 1; v.conj = true; }
  zfill(st, (long long)rows * colsp, make_double2(0.0, 0.0), W);
  gather2(st, rows, cols, A, v, W);
  jacobi_sv_kernel<<<1, JT, 0, st.s>>>(rows, colsp, W, d_out, d_status);
  after_launch(st);
  std::vector<double> sv(colsp);
  int status = 0;
  MPSGPU_CUDA(cudaMemcpyAsync(sv.data(), d_out, colsp * sizeof(double), cudaMemcpyDeviceToHost, st.s));
  MPSGPU_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st.s));
  MPSGPU_CUDA(cudaStreamSynchronize(st.s));
  MPSGPU_CHECK(status <= MAX_SWEEPS, MPSGPU_NOT_CONVERGED, "singular_values: Jacobi did not converge");
  std::sort(sv.begin(), sv.end(), std::greater<double>());
  sv.resize(std::min(m, n));
  return sv;
}

}  // namespace mpsgpu
