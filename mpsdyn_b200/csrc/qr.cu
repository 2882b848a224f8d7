// Blocked Householder QR of a complex FP64 matrix with the LAPACK
// conventions the reference relies on (wrapper::qr -> zgeqrf + zungqr,
// src/wrapper/qr.cpp:33-110; wrapper::lq is the same factorisation of the
// conjugate transpose).  Reflector of a column (alpha, x):
//   beta = -sign(Re alpha) * sqrt(|alpha|^2 + |x|^2),
//   tau = (beta - alpha)/beta, v = (1, x/(alpha - beta)),
//   tau = 0 (H = I) when x = 0 and Im alpha = 0
// (Golub & Van Loan, "Matrix Computations" 5.1; LAPACK zlarfg), the block
// form I - V T V^H with T upper triangular (Schreiber & Van Loan 1989;
// LAPACK zlarft, forward columnwise), and Q = H_1 H_2 ... H_K applied to the
// first K columns of the identity (zungqr).  Keeping these conventions keeps
// the gauge of rank-deficient, zero-padded sites identical to the reference.
//
// Device organisation: one cooperative launch factors the matrix in place
// (column-major, L2-resident workspace).  Panels of nb columns are factored
// by CTA 0 in shared memory; after a grid barrier every CTA applies the
// panel's block reflector to its own nb-column slices of the trailing matrix;
// another barrier closes the panel.  A second launch forms Q column slice by
// column slice (independent, no barrier) and extracts R.
#include <cooperative_groups.h>

#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mpsgpu {

namespace {

constexpr int QR_THREADS = 512;

// sqrt(a^2 + b^2 + c^2) with the largest magnitude factored out (dlapy3).
__device__ __forceinline__ double hypot3(double a, double b, double c) {
  a = fabs(a); b = fabs(b); c = fabs(c);
  const double w = fmax(a, fmax(b, c));
  if (w == 0.0) return 0.0;
  a /= w; b /= w; c /= w;
  return w * sqrt(a * a + b * b + c * c);
}

// 1 / z by Smith's algorithm (R. L. Smith, "Algorithm 116: Complex
// division", CACM 5(8), 1962), which never squares |z|.
__device__ __forceinline__ cplx recip_smith(cplx z) {
  if (fabs(z.x) >= fabs(z.y)) {
    const double r = z.y / z.x, t = 1.0 / (z.x + z.y * r);
    return make_double2(t, -r * t);
  }
  const double r = z.x / z.y, t = 1.0 / (z.y + z.x * r);
  return make_double2(r * t, -t);
}

// Smallest |beta| handled without rescaling: the underflow threshold divided
// by the machine epsilon (LAPACK zlarfg's SAFMIN = dlamch('S') / dlamch('E')).
constexpr double kSafeMin = 2.2250738585072014e-308 / 1.1102230246251565e-16;

// Shared-memory plan of both kernels: the column slice C (mp x nb, ld mp),
// a staging chunk of QR_CH rows of V, the block factor T (nb x nb), the
// product W (nb x nb) and W2 (nb x nb, also the per-thread partial sums of
// W: QR_THREADS entries).
constexpr int QR_CH = 128;
__host__ __device__ constexpr size_t qr_smem_bytes(int m, int nb) {
  return ((size_t)m * nb + (size_t)QR_CH * nb + 2 * (size_t)nb * nb +
          ((size_t)nb * nb > (size_t)QR_THREADS ? (size_t)nb * nb : (size_t)QR_THREADS)) *
         sizeof(cplx);
}
// The largest plan the launchers use (m <= 640 with 16-column panels; above,
// 8-column panels up to m = 1280 need less); the dynamic limit must leave
// room for the kernels' static shared memory within the 227 KB per block.
constexpr int QR_SMEM_ATTR = (int)(qr_smem_bytes(640, 16) > qr_smem_bytes(1280, 8) ? qr_smem_bytes(640, 16)
                                                                                   : qr_smem_bytes(1280, 8));
static_assert(QR_SMEM_ATTR + 4096 <= 227 * 1024, "QR shared-memory plan exceeds the per-block limit");

// Apply (I - V T' V^H) to the mp x cw column slice C (shared, ld = ldc), where
// V (mp x jb, unit lower trapezoidal: its upper triangle and diagonal are not
// read) and T (jb x jb) are in global memory and T' = T^H (conjT = true, for
// Q^H A) or T (for Q E).  V is staged through shared memory in chunks of
// QR_CH rows (coalesced copies), T once; Vs, Ts, W, W2 are shared.
__device__ void apply_block_reflector(int mp, int jb, int cw, const cplx* __restrict__ V, long long ldv,
                                      const cplx* __restrict__ T, int ldt, bool conjT, cplx* C, int ldc,
                                      cplx* Vs, cplx* Ts, cplx* W, cplx* W2) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int t = tid; t < jb * jb; t += nt) Ts[t] = T[(t % jb) + (long long)(t / jb) * ldt];
  const int npair = jb * cw;
  // W[l, q] = sum_r conj(V[r, l]) C[r, q]; threads own pairs (l, q), further
  // groups of threads take every groups-th row when the block has threads to spare
  const int groups = max(1, nt / max(1, npair));
  const int pair = tid % max(1, npair), grp = tid / max(1, npair);
  cplx acc = make_double2(0.0, 0.0);
  for (int r0 = 0; r0 < mp; r0 += QR_CH) {
    const int rows = min(QR_CH, mp - r0);
    __syncthreads();
    for (int t = tid; t < rows * jb; t += nt) {
      const int r = t % rows, l = t / rows, gr = r0 + r;
      cplx v = make_double2(0.0, 0.0);
      if (gr > l) v = V[gr + (long long)l * ldv];
      else if (gr == l) v = make_double2(1.0, 0.0);
      Vs[r + l * QR_CH] = v;
    }
    __syncthreads();
    if (pair < npair && grp < groups) {
      const int l = pair % jb, q = pair / jb;
      for (int r = grp; r < rows; r += groups) acc = cadd(acc, ccmul(Vs[r + l * QR_CH], C[r0 + r + q * ldc]));
    }
  }
  __syncthreads();
  // combine the row groups in a fixed order
  if (pair < npair && grp < groups) W2[pair + grp * npair] = acc;  // W2 as scratch (groups * npair <= nt)
  __syncthreads();
  for (int t = tid; t < npair; t += nt) {
    cplx s = make_double2(0.0, 0.0);
    for (int g = 0; g < groups; g++) s = cadd(s, W2[t + g * npair]);
    W[t] = s;
  }
  __syncthreads();
  // W2 = T' W  (T' = T^H lower triangular, or T upper triangular)
  for (int t = tid; t < npair; t += nt) {
    const int i = t % jb, q = t / jb;
    cplx s = make_double2(0.0, 0.0);
    if (conjT) {
      for (int l = 0; l <= i; l++) s = cadd(s, ccmul(Ts[l + i * jb], W[l + q * jb]));
    } else {
      for (int l = i; l < jb; l++) s = cadd(s, cmul(Ts[i + l * jb], W[l + q * jb]));
    }
    W2[t] = s;
  }
  // C -= V W2, chunk by chunk
  for (int r0 = 0; r0 < mp; r0 += QR_CH) {
    const int rows = min(QR_CH, mp - r0);
    __syncthreads();
    for (int t = tid; t < rows * jb; t += nt) {
      const int r = t % rows, l = t / rows, gr = r0 + r;
      cplx v = make_double2(0.0, 0.0);
      if (gr > l) v = V[gr + (long long)l * ldv];
      else if (gr == l) v = make_double2(1.0, 0.0);
      Vs[r + l * QR_CH] = v;
    }
    __syncthreads();
    for (int t = tid; t < rows * cw; t += nt) {
      const int r = t % rows, q = t / rows;
      cplx s = make_double2(0.0, 0.0);
      for (int l = 0; l < jb; l++) s = cadd(s, cmul(Vs[r + l * QR_CH], W2[l + q * jb]));
      C[r0 + r + q * ldc] = csub(C[r0 + r + q * ldc], s);
    }
  }
  __syncthreads();
}

struct QrParams {
  int m, n, K, nb, npanel;
  cplx* A;      // m x n, ld = m (in: matrix; out: R above, V below the diagonal)
  cplx* T;      // npanel blocks of nb x nb
  cplx* tau;    // K
};

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ cplx warp_csum(cplx v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// 2-norm of x[0..n) by one warp, with the largest component magnitude
// factored out before squaring (the scaled sum of LAPACK's dznrm2):
// rank-deficient sites produce trailing columns with entries far below
// 1e-154, whose plain squares underflow to zero.  Every lane gets the result.
__device__ double warp_scaled_norm(int n, const cplx* x) {
  const int lane = threadIdx.x & 31;
  double mx = 0.0;
  for (int r = lane; r < n; r += 32) mx = fmax(mx, fmax(fabs(x[r].x), fabs(x[r].y)));
  mx = warp_max(mx);
  if (mx == 0.0) return 0.0;
  const double inv = 1.0 / mx;
  double part = 0.0;
  for (int r = lane; r < n; r += 32) {
    const double a = x[r].x * inv, b = x[r].y * inv;
    part += a * a + b * b;
  }
  return mx * sqrt(warp_sum(part));
}

// Householder reflector of column c of the panel P (rows c..mp-1, ld mp),
// computed by one warp (zlarfg): overwrites P[c, c] with beta and the rows
// below with v (v_c = 1 implicit); returns tau.
__device__ cplx warp_reflector(cplx* P, int mp, int c) {
  const int lane = threadIdx.x & 31;
  cplx* x = P + (c + 1) + (long long)c * mp;
  const int nx = mp - c - 1;
  double xnorm = warp_scaled_norm(nx, x);
  cplx alpha = P[c + (long long)c * mp];
  if (xnorm == 0.0 && alpha.y == 0.0) return make_double2(0.0, 0.0);  // H = I
  double nrm = hypot3(alpha.x, alpha.y, xnorm);
  double beta = alpha.x >= 0.0 ? -nrm : nrm;
  // |beta| below kSafeMin: scale the column up (at most 20 times) so that
  // 1 / (alpha - beta) stays finite; beta is scaled back at the end, tau and
  // v are scale-invariant
  int knt = 0;
  while (fabs(beta) < kSafeMin && knt < 20) {
    __syncwarp();
    for (int r = lane; r < nx; r += 32) x[r] = cscale(x[r], 1.0 / kSafeMin);
    beta /= kSafeMin;
    alpha = cscale(alpha, 1.0 / kSafeMin);
    knt++;
  }
  if (knt > 0) {
    __syncwarp();
    xnorm = warp_scaled_norm(nx, x);
    nrm = hypot3(alpha.x, alpha.y, xnorm);
    beta = alpha.x >= 0.0 ? -nrm : nrm;
  }
  const cplx tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
  const cplx scale = recip_smith(make_double2(alpha.x - beta, alpha.y));
  for (int k = 0; k < knt; k++) beta *= kSafeMin;
  __syncwarp();
  for (int r = lane; r < nx; r += 32) x[r] = cmul(x[r], scale);
  __syncwarp();
  if (lane == 0) P[c + (long long)c * mp] = make_double2(beta, 0.0);
  __syncwarp();
  return tau;
}

// Factor the panel P (mp x jb, shared, ld mp) in place and build its block
// factor T (jb x jb, forward columnwise, zlarft) into Tg; taus into taug.
// Warp q owns panel column q: it applies the reflectors of the columns to
// its left to its own column, then, on its turn, computes its reflector, so
// one block barrier per column orders the reflectors.
__device__ void factor_panel(cplx* P, int mp, int jb, cplx* Tg, int ldt, cplx* taug, cplx* Wsh, cplx* taus,
                             cplx* Tsh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c < jb; c++) {
    if (warp == c) {
      const cplx tau = warp_reflector(P, mp, c);
      if (lane == 0) taus[c] = tau;
    }
    __syncthreads();
    // warps to the right apply H_c^H = I - conj(tau_c) v v^H to their column
    if (warp > c && warp < jb) {
      const cplx tau = taus[c];
      if (tau.x != 0.0 || tau.y != 0.0) {
        cplx* a = P + (long long)warp * mp;
        const cplx* v = P + (long long)c * mp;
        cplx s = make_double2(0.0, 0.0);
        for (int r = c + lane; r < mp; r += 32) s = cadd(s, ccmul(r == c ? make_double2(1.0, 0.0) : v[r], a[r]));
        s = cmul(cconj(tau), warp_csum(s));
        for (int r = c + lane; r < mp; r += 32) a[r] = csub(a[r], cmul(r == c ? make_double2(1.0, 0.0) : v[r], s));
      }
      __syncwarp();
    }
  }
  // T: T[i, i] = tau_i, T[0:i, i] = -tau_i T[0:i, 0:i] (V[:, 0:i]^H v_i).
  // First the Gram products G[l, i] = V[:, l]^H v_i (l < i), one warp each.
  const int nw = blockDim.x >> 5;
  for (int t = warp; t < jb * jb; t += nw) {
    const int l = t % jb, i = t / jb;
    if (l >= i) continue;
    cplx s = make_double2(0.0, 0.0);
    for (int r = i + lane; r < mp; r += 32) {
      const cplx vl = P[r + (long long)l * mp];  // r > l
      const cplx vi = (r == i) ? make_double2(1.0, 0.0) : P[r + (long long)i * mp];
      s = cadd(s, ccmul(vl, vi));
    }
    s = warp_csum(s);
    if (lane == 0) Wsh[l + i * jb] = s;
  }
  __syncthreads();
  if (warp == 0) {
    // column by column (one lane per row l < i), T built in shared memory
    // (Tsh, jb x jb) and written to global memory once; jb <= 32
    for (int i = 0; i < jb; i++) {
      const cplx ti = taus[i];
      cplx v = make_double2(0.0, 0.0);
      if (lane < i) {
        cplx s = make_double2(0.0, 0.0);
        for (int q = lane; q < i; q++) s = cadd(s, cmul(Tsh[lane + q * jb], Wsh[q + i * jb]));
        v = cmul(make_double2(-ti.x, -ti.y), s);
      } else if (lane == i) {
        v = ti;
      }
      __syncwarp();
      if (lane < jb) Tsh[lane + i * jb] = v;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < jb * jb; t += blockDim.x) Tg[(t % jb) + (long long)(t / jb) * ldt] = Tsh[t];
  for (int t = threadIdx.x; t < jb; t += blockDim.x) taug[t] = taus[t];
  __syncthreads();
}

__global__ void __launch_bounds__(QR_THREADS) qr_factor_kernel(QrParams p) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double smem_d[];
  const int m = p.m, nb = p.nb;
  cplx* C = reinterpret_cast<cplx*>(smem_d);       // m x nb
  cplx* Vs = C + (size_t)m * nb;                    // QR_CH x nb
  cplx* Ts = Vs + (size_t)QR_CH * nb;               // nb x nb
  cplx* W = Ts + (size_t)nb * nb;
  cplx* W2 = W + (size_t)nb * nb;
  __shared__ cplx taus[32];
  const int G = gridDim.x;
  auto load_slice = [&](int r0, int c0, int rows, int cw) {
    for (int t = threadIdx.x; t < rows * cw; t += blockDim.x) {
      const int r = t % rows, c = t / rows;
      C[t] = p.A[(r0 + r) + (long long)(c0 + c) * m];
    }
    __syncthreads();
  };
  auto store_slice = [&](int r0, int c0, int rows, int cw) {
    __syncthreads();
    for (int t = threadIdx.x; t < rows * cw; t += blockDim.x) {
      const int r = t % rows, c = t / rows;
      p.A[(r0 + r) + (long long)(c0 + c) * m] = C[t];
    }
  };
  for (int pi = 0; pi < p.npanel; pi++) {
    const int j0 = pi * nb;
    const int jb = min(nb, p.K - j0);
    const int mp = m - j0;
    cplx* Tp = p.T + (long long)pi * nb * nb;
    if (blockIdx.x == 0) {
      // the panel's columns were brought up to date by this CTA (look-ahead)
      load_slice(j0, j0, mp, jb);
      factor_panel(C, mp, jb, Tp, nb, p.tau + j0, W, taus, Ts);
      store_slice(j0, j0, mp, jb);
      __threadfence();
    }
    grid.sync();
    // trailing update of columns j0+jb .. n-1 in slices of nb columns: slice
    // 0 (the next panel) by CTA 0, so that it can start on that panel while
    // the other CTAs update the rest
    const int first = j0 + jb;
    const int nslices = (p.n - first + nb - 1) / nb;
    const cplx* V = p.A + j0 + (long long)j0 * m;  // mp x jb, ld = m
    for (int sl = 0; sl < nslices; sl++) {
      const int owner = (sl == 0 || G == 1) ? 0 : 1 + (sl - 1) % (G - 1);
      if (owner != (int)blockIdx.x) continue;
      const int c0 = first + sl * nb;
      const int cw = min(nb, p.n - c0);
      load_slice(j0, c0, mp, cw);
      apply_block_reflector(mp, jb, cw, V, m, Tp, nb, true, C, mp, Vs, Ts, W, W2);
      store_slice(j0, c0, mp, cw);
      __syncthreads();
    }
    __threadfence();
    // CTA 0 goes on with the next panel at once; the other CTAs must not
    // start the next trailing update before that panel is factored, which
    // the barrier at the top of the next iteration ensures
  }
}

// Form Q (m x K) slice by slice and extract R (K x n, zero below the diagonal).
__global__ void __launch_bounds__(QR_THREADS) qr_form_q_kernel(QrParams p, cplx* Q, long long ldq,
                                                               cplx* R, long long ldr) {
  extern __shared__ double smem_d[];
  const int m = p.m, nb = p.nb;
  cplx* C = reinterpret_cast<cplx*>(smem_d);
  cplx* Vs = C + (size_t)m * nb;
  cplx* Ts = Vs + (size_t)QR_CH * nb;
  cplx* W = Ts + (size_t)nb * nb;
  cplx* W2 = W + (size_t)nb * nb;
  const int nslices = (p.K + nb - 1) / nb;
  if (R) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)p.K * p.n;
         t += (long long)gridDim.x * blockDim.x) {
      int i = (int)(t % p.K), j = (int)(t / p.K);
      R[i + j * ldr] = (i <= j) ? p.A[i + (long long)j * m] : make_double2(0.0, 0.0);
    }
  }
  if (!Q) return;
  for (int sl = blockIdx.x; sl < nslices; sl += gridDim.x) {
    const int c0 = sl * nb;
    const int cw = min(nb, p.K - c0);
    for (int t = threadIdx.x; t < m * cw; t += blockDim.x) {
      int r = t % m, c = t / m;
      C[t] = make_double2(r == c0 + c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    // H_j only touch rows >= j0: panels that start below the slice's last
    // column leave its unit columns unchanged
    for (int pi = min(p.npanel - 1, (c0 + cw - 1) / nb); pi >= 0; pi--) {
      const int j0 = pi * nb;
      const int jb = min(nb, p.K - j0);
      apply_block_reflector(m - j0, jb, cw, p.A + j0 + (long long)j0 * m, m, p.T + (long long)pi * nb * nb, nb,
                            false, C + j0, m, Vs, Ts, W, W2);
    }
    for (int t = threadIdx.x; t < m * cw; t += blockDim.x) {
      int r = t % m, c = t / m;
      Q[r + (long long)(c0 + c) * ldq] = C[t];
    }
    __syncthreads();
  }
}

}  // namespace

// Factor the m x n column-major matrix A (ld = m, overwritten).  Q (m x K,
// ld = ldq) and R (K x n, ld = ldr) are written when non-null.
void householder_qr_inplace(const Stream& st, int m, int n, cplx* A, cplx* Q, long long ldq,
                            cplx* R, long long ldr, Scratch& scratch) {
  MPSGPU_CHECK(m > 0 && n > 0, MPSGPU_BAD_SHAPE, "qr: empty matrix");
  const int K = std::min(m, n);
  const int nb = (m <= 640) ? 16 : 8;
  // factorisation and explicit Q, complex flops (8 per complex MAC)
  ProfScope ps(st, GemmProfiler::QR,
               16.0 * (2.0 * m * n * K - (double)(m + n) * K * K + 2.0 * (double)K * K * K / 3.0));
  MPSGPU_CHECK(m <= 1280, MPSGPU_BAD_SHAPE, "qr: more than 1280 rows is not supported");
  QrParams p;
  p.m = m; p.n = n; p.K = K; p.nb = nb; p.npanel = (K + nb - 1) / nb;
  p.A = A;
  char* ws = (char*)scratch.get((size_t)p.npanel * nb * nb * sizeof(cplx) + (size_t)K * sizeof(cplx) + 256);
  p.T = (cplx*)ws;
  p.tau = p.T + (size_t)p.npanel * nb * nb;
  const size_t smem = qr_smem_bytes(m, nb);
  static std::atomic<unsigned long long> attr_done{0};
  if (device_needs_setup(attr_done)) {
    MPSGPU_CUDA(cudaFuncSetAttribute(qr_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, QR_SMEM_ATTR));
    MPSGPU_CUDA(cudaFuncSetAttribute(qr_form_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, QR_SMEM_ATTR));
    mark_device_done(attr_done);
  }
  int dev = 0, nsm = 148, per_sm = 1;
  MPSGPU_CUDA(cudaGetDevice(&dev));
  MPSGPU_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  MPSGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qr_factor_kernel, QR_THREADS, smem));
  MPSGPU_CHECK(per_sm >= 1, MPSGPU_BAD_SHAPE, "qr: kernel does not fit on an SM");
  int trailing_slices = std::max(1, (n + nb - 1) / nb);
  int grid = std::min(trailing_slices, nsm * per_sm);
  void* args[] = {&p};
  MPSGPU_CUDA(cudaLaunchCooperativeKernel((void*)qr_factor_kernel, dim3(grid), dim3(QR_THREADS), args, smem, st.s));
  after_launch(st);
  int qgrid = std::max(1, std::min((K + nb - 1) / nb, nsm));
  if (R && !Q) qgrid = std::max(qgrid, 8);
  qr_form_q_kernel<<<qgrid, QR_THREADS, smem, st.s>>>(p, Q, ldq, R, ldr);
  after_launch(st);
}

}  // namespace mpsgpu

// ---------------------------------------------------------------------------
// QR without allocation (mpsgpu_qr_device_noalloc, include/mpsgpu.h).
//
// Some callers cannot allocate device memory at the moment they need a gauge
// move: a serving process whose memory manager has reserved the whole HBM
// for its request slots, or a real-time loop that must not meet an
// allocation failure half way through a sweep.
// For them this variant keeps every byte of its working memory in one
// file-scope device array: the working copy of A (factored in place), the
// block-reflector factors T and the scalars tau.  CUDA loads a module's
// device code (and places its __device__ arrays) lazily, on first use in a
// context, so mpsgpu_create places the array on its device at once
// (noalloc_qr_prepare below): after a context exists on a GPU, the entry
// point needs no new device memory there.  The array is held until exit.
// ---------------------------------------------------------------------------

namespace mpsgpu {
namespace {

// Capacity: m*n <= 131072 complex (for example 512 x 256), m, n <= 640
// (nb = 16), i.e. at most 40 panels of 16 x 16 T factors and 640 tau values.
constexpr long long NOALLOC_MAX_ELEMS = 131072;
constexpr int NOALLOC_MAX_DIM = 640;
constexpr int NOALLOC_NB = 16;
constexpr long long NOALLOC_T_ELEMS = (long long)(NOALLOC_MAX_DIM / NOALLOC_NB) * NOALLOC_NB * NOALLOC_NB;
constexpr long long NOALLOC_TOTAL = NOALLOC_MAX_ELEMS + NOALLOC_T_ELEMS + NOALLOC_MAX_DIM;

// 2.1 MiB.  Host code must not use this name as an address: it is a host-side
// stand-in for the device symbol; the device address comes from
// cudaGetSymbolAddress, once per device (noalloc_scratch_on below).
static __device__ __align__(256) double2 g_qr_noalloc_scratch[NOALLOC_TOTAL];

constexpr int MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double2* g_noalloc_ptr[MAX_DEVICES] = {nullptr};
bool g_noalloc_attr[MAX_DEVICES] = {false};

// Device address of the scratch array on the current device (set-up on the
// first call per device; later calls only read the cached pointer).
mpsgpu_status noalloc_scratch_on(int dev, double2** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_qr_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return MPSGPU_CUDA_ERROR;
    g_noalloc_ptr[dev] = static_cast<double2*>(p);
  }
  if (!g_noalloc_attr[dev]) {
    if (cudaFuncSetAttribute(qr_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, QR_SMEM_ATTR) !=
            cudaSuccess ||
        cudaFuncSetAttribute(qr_form_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, QR_SMEM_ATTR) !=
            cudaSuccess)
      return MPSGPU_CUDA_ERROR;
    g_noalloc_attr[dev] = true;
  }
  *out = g_noalloc_ptr[dev];
  return MPSGPU_OK;
}

}  // namespace

// Called by mpsgpu_create with `dev` current: loads this file's module on the
// device, which places the scratch array, and sets the kernel attributes.
mpsgpu_status noalloc_qr_prepare(int dev) {
  if (dev < 0 || dev >= MAX_DEVICES) return MPSGPU_CUDA_ERROR;
  double2* p = nullptr;
  return noalloc_scratch_on(dev, &p);
}

}  // namespace mpsgpu

extern "C" mpsgpu_status mpsgpu_qr_device_noalloc(int m, int n, const double* A, double* Q, double* R,
                                                  void* stream) {
  using namespace mpsgpu;
  if (m <= 0 || n <= 0 || !A || (!Q && !R)) return MPSGPU_INVALID;
  if (m > NOALLOC_MAX_DIM || n > NOALLOC_MAX_DIM || (long long)m * n > NOALLOC_MAX_ELEMS) {
    fprintf(stderr,
            "mpsgpu_qr_device_noalloc: %d x %d exceeds the fixed scratch (m, n <= %d and m*n <= %lld)\n", m,
            n, NOALLOC_MAX_DIM, NOALLOC_MAX_ELEMS);
    return MPSGPU_BAD_SHAPE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return MPSGPU_CUDA_ERROR;
  double2* scratch = nullptr;
  mpsgpu_status st = noalloc_scratch_on(dev, &scratch);
  if (st != MPSGPU_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int K = std::min(m, n);
  QrParams p;
  p.m = m; p.n = n; p.K = K; p.nb = NOALLOC_NB; p.npanel = (K + NOALLOC_NB - 1) / NOALLOC_NB;
  // Layout of the shared array: [A copy | T factors | tau].  Every element
  // the kernels read is written first in the same call (the copy of A, then
  // T and tau by the factorisation), so nothing needs clearing.
  p.A = scratch;
  p.T = scratch + NOALLOC_MAX_ELEMS;
  p.tau = p.T + NOALLOC_T_ELEMS;
  if (cudaMemcpyAsync(p.A, A, (size_t)m * n * sizeof(double2), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return MPSGPU_CUDA_ERROR;
  const size_t smem = qr_smem_bytes(m, NOALLOC_NB);
  int nsm = 148, per_sm = 1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qr_factor_kernel, QR_THREADS, smem) != cudaSuccess ||
      per_sm < 1)
    return MPSGPU_CUDA_ERROR;
  const int grid = std::min(std::max(1, (n + NOALLOC_NB - 1) / NOALLOC_NB), nsm * per_sm);
  void* args[] = {&p};
  if (cudaLaunchCooperativeKernel((void*)qr_factor_kernel, dim3(grid), dim3(QR_THREADS), args, smem, s) !=
      cudaSuccess)
    return MPSGPU_CUDA_ERROR;
  int qgrid = std::max(1, std::min((K + NOALLOC_NB - 1) / NOALLOC_NB, nsm));
  if (R && !Q) qgrid = std::max(qgrid, 8);
  // launched through cudaLaunchKernel, whose return code is this launch's
  // alone (cudaGetLastError would also report, and clear, an unrelated
  // earlier error of the calling thread)
  double2* Qd = reinterpret_cast<double2*>(Q);
  double2* Rd = reinterpret_cast<double2*>(R);
  long long ldq = m, ldr = K;
  void* qargs[] = {&p, &Qd, &ldq, &Rd, &ldr};
  if (cudaLaunchKernel((const void*)qr_form_q_kernel, dim3(qgrid), dim3(QR_THREADS), qargs, smem, s) !=
      cudaSuccess)
    return MPSGPU_CUDA_ERROR;
  return MPSGPU_OK;
}
