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
constexpr int MAX_COLS = 1024;

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
// norms.  V (n x n, ld n, identity on entry) accumulates the rotations when
// non-null, so that A_in V = A_out.  status[0] = sweeps used (MAX_SWEEPS + 1
// if not converged).
__global__ void __launch_bounds__(JT) jacobi_sv_kernel(int m, int n, cplx* A, cplx* V, double* out, int* status) {
  __shared__ int rotated;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = JT / 32;
  const double tol = 1e-15;
  int sweep = 0;
  for (sweep = 0; sweep < MAX_SWEEPS; sweep++) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int step = 0; step < n - 1; step++) {
      // round-robin (circle) pairing: slot k pairs with slot n-1-k; slot 0
      // holds column 0, slot k >= 1 holds column ((k - 1 - step) mod (n-1)) + 1
      for (int pr = warp; pr < n / 2; pr += nw) {
        const int kq = n - 1 - pr;
        const int p = pr == 0 ? 0 : ((pr - 1 - step) % (n - 1) + (n - 1)) % (n - 1) + 1;
        const int q = ((kq - 1 - step) % (n - 1) + (n - 1)) % (n - 1) + 1;
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
          if (V) {
            cplx* vp = V + (long long)p * n;
            cplx* vq = V + (long long)q * n;
            for (int r = lane; r < n; r += 32) {
              const cplx x = vp[r];
              const cplx y = cmul(vq[r], ph);
              vp[r] = make_double2(cs * x.x - sn * y.x, cs * x.y - sn * y.y);
              vq[r] = make_double2(sn * x.x + cs * y.x, sn * x.y + cs * y.y);
            }
          }
          if (lane == 0) rotated = 1;
        }
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
  MPSGPU_CHECK(colsp <= MAX_COLS && rows <= 8192, MPSGPU_BAD_SHAPE, "singular_values: matrix too large");
  char* ws = (char*)scratch.get((size_t)rows * colsp * sizeof(cplx) + colsp * sizeof(double) + 64);
  cplx* W = (cplx*)ws;
  double* d_out = (double*)(ws + (size_t)rows * colsp * sizeof(cplx));
  int* d_status = (int*)(d_out + colsp);
  View2 v;
  if (!tr) { v.rd = 1; v.r0 = 0; v.r1 = 1; v.cd = 1; v.c0 = 0; v.c1 = lda; }
  else { v.rd = 1; v.r0 = 0; v.r1 = lda; v.cd = 1; v.c0 = 0; v.c1 = 1; v.conj = true; }
  zfill(st, (long long)rows * colsp, make_double2(0.0, 0.0), W);
  gather2(st, rows, cols, A, v, W);
  jacobi_sv_kernel<<<1, JT, 0, st.s>>>(rows, colsp, W, nullptr, d_out, d_status);
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

namespace {

// Kept singular triplets in descending order (idx[j] = Jacobi column of the
// j-th largest value).  Not transposed (m >= n, W = A V): U[:, j] =
// W[:, idx_j] / s_j, SVh[j, :] = s_j V[:, idx_j]^H.  Transposed (W = A^H V'):
// A = V' S U'^H, so U[:, j] = V'[:, idx_j] and SVh[j, :] = W[:, idx_j]^H.
// left_s moves diag(s) to the left factor: U diag(s) and V^H.
__global__ void svd_finish_kernel(int m, int n, int rows, int cols, bool tr, const cplx* __restrict__ W,
                                  const cplx* __restrict__ V, const int* __restrict__ idx,
                                  const double* __restrict__ sig, int keep, bool left_s, cplx* __restrict__ U,
                                  cplx* __restrict__ SVh) {
  const long long totU = (long long)m * keep, totS = (long long)keep * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < totU + totS;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < totU) {
      const int i = (int)(t % m), j = (int)(t / m);
      const int c = idx[j];
      cplx u = tr ? V[i + (long long)c * cols] : cscale(W[i + (long long)c * rows], 1.0 / sig[c]);
      if (left_s) u = cscale(u, sig[c]);
      U[t] = u;
    } else {
      const long long q = t - totU;
      const int j = (int)(q % keep), k = (int)(q / keep);
      const int c = idx[j];
      cplx x = tr ? W[k + (long long)c * rows] : cscale(V[k + (long long)c * cols], sig[c]);
      if (left_s) x = cscale(x, 1.0 / sig[c]);
      SVh[j + (long long)k * keep] = make_double2(x.x, -x.y);
    }
  }
}

__global__ void identity_kernel(int n, cplx* __restrict__ V) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x)
    V[t] = make_double2((t % n) == (t / n) ? 1.0 : 0.0, 0.0);
}

}  // namespace

// Thin SVD with the cut of wrapper::svd(A, tol = 0, Xi = cut) (svd.cpp:23-118):
// keep = min(cut, min(m, n)) (cut <= 0: all), then only the values > 0 among
// those.  A (m x n, ld m) is not modified.  Writes U (m x keep, ld m) and
// diag(s) V^H (keep x n, ld keep) -- or, with left_s, U diag(s) and V^H;
// sv gets all min(m, n) values descending.
int svd_cut(const Stream& st, int m, int n, const cplx* A, long long lda, int cut, cplx* U, cplx* SVh,
            std::vector<double>& sv, Scratch& scratch, bool left_s) {
  MPSGPU_CHECK(m > 0 && n > 0, MPSGPU_BAD_SHAPE, "svd: empty matrix");
  const bool tr = n > m;
  const int rows = tr ? n : m;
  const int cols = tr ? m : n;
  const int colsp = cols + (cols & 1);
  MPSGPU_CHECK(colsp <= MAX_COLS && rows <= 8192, MPSGPU_BAD_SHAPE, "svd: matrix too large");
  const size_t wbytes = (size_t)rows * colsp * sizeof(cplx), vbytes = (size_t)colsp * colsp * sizeof(cplx);
  char* ws = (char*)scratch.get(wbytes + vbytes + colsp * (sizeof(double) + sizeof(int)) + 256);
  cplx* W = (cplx*)ws;
  cplx* V = (cplx*)(ws + wbytes);
  double* d_sig = (double*)(ws + wbytes + vbytes);
  int* d_idx = (int*)(d_sig + colsp);
  int* d_status = d_idx + colsp;
  View2 v;
  if (!tr) { v.rd = 1; v.r0 = 0; v.r1 = 1; v.cd = 1; v.c0 = 0; v.c1 = lda; }
  else { v.rd = 1; v.r0 = 0; v.r1 = lda; v.cd = 1; v.c0 = 0; v.c1 = 1; v.conj = true; }
  zfill(st, (long long)rows * colsp, make_double2(0.0, 0.0), W);
  gather2(st, rows, cols, A, v, W);
  identity_kernel<<<std::min(ceil_div((long long)colsp * colsp, 256), 1184), 256, 0, st.s>>>(colsp, V);
  after_launch(st);
  jacobi_sv_kernel<<<1, JT, 0, st.s>>>(rows, colsp, W, V, d_sig, d_status);
  after_launch(st);
  std::vector<double> all(colsp);
  int status = 0;
  MPSGPU_CUDA(cudaMemcpyAsync(all.data(), d_sig, colsp * sizeof(double), cudaMemcpyDeviceToHost, st.s));
  MPSGPU_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st.s));
  MPSGPU_CUDA(cudaStreamSynchronize(st.s));
  MPSGPU_CHECK(status <= MAX_SWEEPS, MPSGPU_NOT_CONVERGED, "svd: Jacobi did not converge");
  // descending order over the real columns (the padding column is not a value)
  std::vector<int> idx(cols);
  for (int j = 0; j < cols; j++) idx[j] = j;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return all[a] > all[b]; });
  sv.resize(cols);
  for (int j = 0; j < cols; j++) sv[j] = all[idx[j]];
  int keep = cut > 0 ? std::min(cut, cols) : cols;
  int pos = 0;
  while (pos < keep && sv[pos] > 0.0) pos++;
  keep = pos;
  MPSGPU_CHECK(keep > 0, MPSGPU_BAD_SHAPE, "svd: no singular value above 0");
  MPSGPU_CUDA(cudaMemcpyAsync(d_idx, idx.data(), keep * sizeof(int), cudaMemcpyHostToDevice, st.s));
  const long long tot = (long long)m * keep + (long long)keep * n;
  svd_finish_kernel<<<std::min(ceil_div(tot, 256), 1184), 256, 0, st.s>>>(m, n, rows, colsp, tr, W, V, d_idx,
                                                                           d_sig, keep, left_s, U, SVh);
  after_launch(st);
  // idx is a host vector: wait for its copy before it goes out of scope
  MPSGPU_CUDA(cudaStreamSynchronize(st.s));
  return keep;
}

}  // namespace mpsgpu
