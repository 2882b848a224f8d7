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
  double beta = -copysign(nrm, alpha.x);  // -sign(Re alpha) nrm, signed zero as LAPACK
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
    beta = -copysign(nrm, alpha.x);
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

// ---------------------------------------------------------------------------
// Cluster QR: the whole matrix in the shared memory of one thread-block
// cluster of S <= 8 CTAs (m <= 256 rows).  Column slice q (16 columns) lives
// in CTA q % S; panel q is the first min(16, K - 16q) columns of slice q, so
// its owner factors it where it lies and the other CTAs read its reflectors
// V and block factor T through distributed shared memory after one cluster
// barrier.  Q is formed slice by slice in the same launch (slice q by the
// owner of panel q, applying H_q, H_{q-1}, ..., H_0 to unit columns), so
// neither the factored matrix nor T ever goes to global memory.
//
// Inside a panel, thread i holds row i of the panel (16 columns) in
// registers.  For column c one block reduction of 16 slots gives at once
// the squared norm of x = A[c+1:, c] (slot c; its imaginary part carries
// sum_r max(|Re x_r|, |Im x_r|), a scale and zero test), the products
// x^H A[c+1:, q] with the panel's later columns (slots q > c), and the
// products V[c+1:, l]^H x with the earlier reflectors (slots l < c), from
// which the column of T follows (zlarft's V^H v), since v = x / (alpha -
// beta) below its unit entry.  When the scale test finds x tiny or huge
// (entries of rank-deficient sites below 1e-154 square to zero), the slots
// are summed again with x / scale, as zlarfg rescales.
// ---------------------------------------------------------------------------

constexpr int CQ_NB = 16;    // slice and panel width
constexpr int CQ_T = 256;    // threads per CTA: one panel row each
constexpr int CQ_MAXM = CQ_T;
constexpr int CQ_MAXS = 8;   // CTAs per cluster (portable limit)
static_assert(CQ_T == 256, "the 16 x 16 scratch is staged one entry per thread");

struct CqParams {
  int m, n, K;
  int npa, np;     // column slices of A (ceil(n/16)); panels = slices of Q (ceil(K/16))
  int S, nA, nQ;   // cluster size; slices of A and of Q per CTA (most)
  const cplx* A;   // m x n, ld m (read only)
  cplx* Q; long long ldq;
  cplx* R; long long ldr;
};

// Shared memory of the cluster kernel in complex entries: A slices, Q
// slices, the staging copy of a panel's V (m x 16), the T factors of the
// panels owned, and 16 x 16 scratch: T staging, W, W2, the Gram columns G,
// the warps' slot sums (8 x 16), the slot totals, two row buffers, tau and
// the column's update coefficients.
__host__ __device__ constexpr size_t cq_smem_elems(int m, int nA, int nQ) {
  return (size_t)(nA + nQ + 1) * m * CQ_NB + (size_t)nQ * 256 + 4 * 256 + (CQ_T / 32) * 16 + 16 + 32 + 16 + 16;
}

// Sum of v[0..31] over the lanes of a warp by a transposing butterfly: after
// the five exchange steps lane L holds the total of v[L].
__device__ __forceinline__ cplx warp_sum32(cplx (&v)[32]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int half = 16; half >= 1; half >>= 1) {
    const bool up = lane & half;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const cplx send = up ? v[i] : v[i + half];
      cplx keep = up ? v[i + half] : v[i];
      keep.x += __shfl_xor_sync(0xffffffffu, send.x, half);
      keep.y += __shfl_xor_sync(0xffffffffu, send.y, half);
      v[i] = keep;
    }
  }
  return v[0];
}

// The same for 16 values: afterwards lanes L and L ^ 1 hold the total of
// v[L >> 1].
__device__ __forceinline__ cplx warp_sum16x(cplx (&v)[16]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int half = 8, mask = 16; half >= 1; half >>= 1, mask >>= 1) {
    const bool up = lane & mask;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const cplx send = up ? v[i] : v[i + half];
      cplx keep = up ? v[i + half] : v[i];
      keep.x += __shfl_xor_sync(0xffffffffu, send.x, mask);
      keep.y += __shfl_xor_sync(0xffffffffu, send.y, mask);
      v[i] = keep;
    }
  }
  cplx r = v[0];
  r.x += __shfl_xor_sync(0xffffffffu, r.x, 1);
  r.y += __shfl_xor_sync(0xffffffffu, r.y, 1);
  return r;
}

// Copy panel (V, T) of slice Vr (possibly another CTA's shared memory, ld
// m) into Vs (rows j0.. as rows 0.., ld mp, unit lower trapezoidal in its
// first jb columns, zero elsewhere) and Ts (16 x 16, zero outside jb x jb).
__device__ void cq_stage(const cplx* Vr, const cplx* Tr, int m, int j0, int jb, cplx* Vs, cplx* Ts) {
  const int mp = m - j0;
  // every load issued before the first store: a load from another CTA's
  // shared memory takes several hundred cycles
  constexpr int PER = CQ_MAXM * CQ_NB / CQ_T;
  cplx v[PER];
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int t = threadIdx.x + u * CQ_T;
    const int r = t % mp, l = t / mp;
    v[u] = make_double2(0.0, 0.0);
    if (t < mp * CQ_NB && l < jb) {
      if (r > l) v[u] = Vr[j0 + r + (long long)l * m];
      else if (r == l) v[u] = make_double2(1.0, 0.0);
    }
  }
  const cplx tv = threadIdx.x < 256 && (threadIdx.x % 16) < jb && (threadIdx.x / 16) < jb ? Tr[threadIdx.x]
                                                                                        : make_double2(0.0, 0.0);
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int t = threadIdx.x + u * CQ_T;
    if (t < mp * CQ_NB) Vs[t] = v[u];
  }
  if (threadIdx.x < 256) Ts[threadIdx.x] = tv;
  __syncthreads();
}

// C[j0:, 0:16] <- (I - V T' V^H) C[j0:, 0:16] for the staged panel (Vs, Ts);
// T' = T^H (conjT: the factorisation's H^H) or T (forming Q).  C is a slice
// in this CTA's shared memory (ld m).  W = V^H C by warps owning 4 x 8
// blocks (lanes take rows), W2 = T' W, then C -= V W2 by rows.
__device__ void cq_apply(cplx* C, int m, int j0, const cplx* Vs, const cplx* Ts, bool conjT, cplx* W, cplx* W2) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int mp = m - j0;
  {
    const int l0 = (warp >> 1) * 4, q0 = (warp & 1) * 8;
    cplx acc[32];
#pragma unroll
    for (int e = 0; e < 32; e++) acc[e] = make_double2(0.0, 0.0);
    for (int r = lane; r < mp; r += 32) {
      cplx v[4], c[8];
#pragma unroll
      for (int i = 0; i < 4; i++) v[i] = Vs[r + (l0 + i) * mp];
#pragma unroll
      for (int k = 0; k < 8; k++) c[k] = C[j0 + r + (long long)(q0 + k) * m];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int k = 0; k < 8; k++) acc[i * 8 + k] = cadd(acc[i * 8 + k], ccmul(v[i], c[k]));
    }
    const cplx s = warp_sum32(acc);
    W[(l0 + (lane >> 3)) + 16 * (q0 + (lane & 7))] = s;
  }
  __syncthreads();
  {
    const int i = tid & 15, q = tid >> 4;  // 256 threads: one entry of W2 each
    cplx s = make_double2(0.0, 0.0);
    if (conjT) {
      for (int l = 0; l <= i; l++) s = cadd(s, ccmul(Ts[l + 16 * i], W[l + 16 * q]));
    } else {
      for (int l = i; l < 16; l++) s = cadd(s, cmul(Ts[i + 16 * l], W[l + 16 * q]));
    }
    W2[i + 16 * q] = s;
  }
  __syncthreads();
  for (int it = tid; it < mp * 4; it += CQ_T) {
    const int r = it % mp, q0 = (it / mp) * 4;
    cplx a0 = make_double2(0.0, 0.0), a1 = a0, a2 = a0, a3 = a0;
#pragma unroll
    for (int l = 0; l < 16; l++) {
      const cplx v = Vs[r + l * mp];
      a0 = cadd(a0, cmul(v, W2[l + 16 * (q0 + 0)]));
      a1 = cadd(a1, cmul(v, W2[l + 16 * (q0 + 1)]));
      a2 = cadd(a2, cmul(v, W2[l + 16 * (q0 + 2)]));
      a3 = cadd(a3, cmul(v, W2[l + 16 * (q0 + 3)]));
    }
    cplx* c = C + j0 + r + (long long)q0 * m;
    c[0] = csub(c[0], a0);
    c[m] = csub(c[m], a1);
    c[2LL * m] = csub(c[2LL * m], a2);
    c[3LL * m] = csub(c[3LL * m], a3);
  }
  __syncthreads();
}

// Block sum of the 16 slots of every thread: warp sums, then threads 0..15
// add the warps' values in a fixed order into tot[0..15].
__device__ __forceinline__ void cq_reduce16(cplx (&s)[16], cplx* red, cplx* tot) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const cplx r = warp_sum16x(s);
  if ((lane & 1) == 0) red[warp * 16 + (lane >> 1)] = r;
  __syncthreads();
  if (tid < 16) {
    cplx a = make_double2(0.0, 0.0);
#pragma unroll
    for (int w = 0; w < CQ_T / 32; w++) a = cadd(a, red[w * 16 + tid]);
    tot[tid] = a;
  }
  __syncthreads();
}

// The 16 slots of one row for column c: conj(V[i, l]) x (l < c), conj(x)
// A[i, q] (q > c) and (|x|^2, max(|Re x|, |Im x|)) in slot c.  Both kinds
// are p_l = conj(a_l) x, conjugated for l > c; register indices are
// compile-time and c only enters through predicates, so one copy of the
// code serves every column.
__device__ __forceinline__ void cq_slots(const cplx (&a)[16], int c, cplx x, bool with_max, cplx (&s)[16]) {
#pragma unroll
  for (int l = 0; l < 16; l++) {
    const cplx p = ccmul(a[l], x);
    s[l] = make_double2(p.x, l > c ? -p.y : p.y);
  }
  const double mx = with_max ? fmax(fabs(x.x), fabs(x.y)) : 0.0;
  const double n2 = cabs2(x);
#pragma unroll
  for (int l = 0; l < 16; l++)
    if (l == c) s[l] = make_double2(n2, mx);
}

// One column of the panel factorisation (zlarfg for column c, then H_c^H on
// the panel's later columns), for the panel row held in a (this thread's
// row i of the panel; i < 0: no row).  tq (16, shared) carries the update
// coefficients conj(tau) s_q, computed once per column.
__device__ __forceinline__ void cq_column(cplx (&a)[16], int c, int i, cplx* red, cplx* tot, cplx* rowbuf, cplx* G,
                                          cplx* taus, cplx* tq) {
  const int tid = threadIdx.x;
  cplx* rb = rowbuf + (c & 1) * 16;
  if (i == c) {
#pragma unroll
    for (int l = 0; l < 16; l++) rb[l] = a[l];
  }
  const bool below = i > c;
  cplx ac = make_double2(0.0, 0.0);  // a[c] without a runtime register index
#pragma unroll
  for (int l = 0; l < 16; l++)
    if (l == c) ac = a[l];
  cplx s[16];
  cq_slots(a, c, below ? ac : make_double2(0.0, 0.0), true, s);
  cq_reduce16(s, red, tot);
  const cplx alpha = rb[c];
  const double x1 = tot[c].y;
  // scale test: x exactly zero, or every square and product representable
  const bool slow = x1 != 0.0 && (x1 < 1e-140 || x1 > 1e140 || fabs(alpha.x) > 1e140 || fabs(alpha.y) > 1e140);
  double sig = 1.0;
  if (slow) {  // uniform over the block: every thread read the same total
    sig = x1;
    // x / sig by division (1 / sig may overflow)
    cq_slots(a, c, below ? make_double2(ac.x / sig, ac.y / sig) : make_double2(0.0, 0.0), false, s);
    cq_reduce16(s, red, tot);
  }
  const double n2 = tot[c].x;
  const cplx al = slow ? make_double2(alpha.x / sig, alpha.y / sig) : alpha;
  cplx tau = make_double2(0.0, 0.0), sv = make_double2(0.0, 0.0);
  double beta = alpha.x;
  const bool identity = (n2 == 0.0 && al.y == 0.0);
  if (!identity) {
    // |alpha|^2 + |x|^2 directly while it is representable (alpha alone can
    // be tiny when x is exactly zero), else with the largest part factored out
    const double nrm2 = al.x * al.x + al.y * al.y + n2;
    const double nrm = (!slow && nrm2 > 1e-280 && nrm2 < 1e280) ? sqrt(nrm2) : hypot3(al.x, al.y, sqrt(n2));
    const double bp = -copysign(nrm, al.x);  // -sign(Re alpha) nrm, signed zero as LAPACK
    tau = make_double2((bp - al.x) / bp, -al.y / bp);
    sv = recip_smith(make_double2(al.x - bp, al.y));
    beta = bp * sig;
  }
  if (tid < 16) {
    // Gram column c of T: V[:, l]^H v_c = conj(V[c, l]) + sv * (V[c+1:, l]^H x');
    // update coefficients: s_q = v^H A[:, q] = A[c, q] + conj(sv) (x'^H A[c+1:, q])
    if (tid < c) G[tid + 16 * c] = cadd(cconj(rb[tid]), cmul(sv, tot[tid]));
    tq[tid] = (tid > c && !identity) ? cmul(cconj(tau), cadd(rb[tid], ccmul(sv, tot[tid]))) : make_double2(0.0, 0.0);
    if (tid == 0) taus[c] = tau;
  }
  __syncthreads();
  if (i >= c) {
    // A[:, q] -= conj(tau) s_q v for q > c (tq is zero elsewhere)
    const cplx v = i == c ? make_double2(1.0, 0.0) : cmul(slow ? make_double2(ac.x / sig, ac.y / sig) : ac, sv);
#pragma unroll
    for (int q = 0; q < 16; q++) a[q] = csub(a[q], cmul(tq[q], v));
    const cplx diag = i == c ? make_double2(beta, 0.0) : v;
    if (!identity || i == c) {
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (q == c) a[q] = diag;
    }
  }
}

// Factor panel rows j0.. of slice As (this CTA, ld m), jb columns, in place
// (R on and above the diagonal, V below), and build its block factor T
// (16 x 16, zero outside jb x jb, ld 16) into Tout.
__device__ void cq_factor_panel(cplx* As, int m, int j0, int jb, cplx* Tout, cplx* red, cplx* tot, cplx* rowbuf,
                                cplx* G, cplx* taus, cplx* tq) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int mp = m - j0;
  const int i = tid < mp ? tid : -1;
  cplx a[16];
#pragma unroll
  for (int l = 0; l < 16; l++) a[l] = i >= 0 ? As[j0 + i + (long long)l * m] : make_double2(0.0, 0.0);
#pragma unroll 1
  for (int c = 0; c < jb; c++) cq_column(a, c, i, red, tot, rowbuf, G, taus, tq);
  if (i >= 0) {
#pragma unroll
    for (int l = 0; l < 16; l++) As[j0 + i + (long long)l * m] = a[l];
  }
  __syncthreads();
  // T column by column (zlarft, forward, columnwise): T[c, c] = tau_c,
  // T[0:c, c] = -tau_c T[0:c, 0:c] G[0:c, c]; lane l keeps row l of T in
  // registers
  if (warp == 0) {
    cplx trow[16];
#pragma unroll
    for (int q = 0; q < 16; q++) trow[q] = make_double2(0.0, 0.0);
    for (int c = 0; c < jb; c++) {
      const cplx tc = taus[c];
      cplx acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (q >= lane && q < c) acc = cadd(acc, cmul(trow[q], G[q + 16 * c]));
      const cplx v = lane < c ? cmul(make_double2(-tc.x, -tc.y), acc) : (lane == c ? tc : make_double2(0.0, 0.0));
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (q == c) trow[q] = v;
    }
    if (lane < 16) {
#pragma unroll
      for (int q = 0; q < 16; q++) Tout[lane + 16 * q] = trow[q];
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(CQ_T, 1) qr_cluster_kernel(const __grid_constant__ CqParams p) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double smem_d[];
  const int m = p.m, S = p.S;
  const int rank = (int)cl.block_rank();
  const long long sl = (long long)m * CQ_NB;
  cplx* As = reinterpret_cast<cplx*>(smem_d);
  cplx* Qs = As + p.nA * sl;
  cplx* Vs = Qs + p.nQ * sl;
  cplx* Tl = Vs + sl;
  cplx* Ts = Tl + p.nQ * 256;
  cplx* W = Ts + 256;
  cplx* W2 = W + 256;
  cplx* G = W2 + 256;
  cplx* red = G + 256;
  cplx* tot = red + (CQ_T / 32) * 16;
  cplx* rowbuf = tot + 16;
  cplx* taus = rowbuf + 32;
  cplx* tq = taus + 16;
  const int tid = threadIdx.x;

  // this CTA's slices q = rank + i S of A (columns past n are zero)
  for (int i = 0; i < p.nA; i++) {
    const int q = rank + i * S;
    if (q >= p.npa) break;
    for (int t = tid; t < m * CQ_NB; t += CQ_T) {
      const int r = t % m, j = q * CQ_NB + t / m;
      As[i * sl + t] = j < p.n ? p.A[r + (long long)j * m] : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();

  for (int pn = 0; pn < p.np; pn++) {
    const int owner = pn % S, li = pn / S;
    const int j0 = pn * CQ_NB, jb = min(CQ_NB, p.K - j0);
    if (rank == owner) cq_factor_panel(As + li * sl, m, j0, jb, Tl + li * 256, red, tot, rowbuf, G, taus, tq);
    cl.sync();  // panel pn published to the cluster
    bool staged = false;
    for (int i = 0; i < p.nA; i++) {
      const int q = rank + i * S;
      if (q >= p.npa) break;
      if (q <= pn) continue;
      if (!staged) {
        cq_stage(cl.map_shared_rank(As + li * sl, owner), cl.map_shared_rank(Tl + li * 256, owner), m, j0, jb, Vs,
                 Ts);
        staged = true;
      }
      cq_apply(As + i * sl, m, j0, Vs, Ts, true, W, W2);
    }
  }

  // Q slice q = H_0 H_1 ... H_q applied to unit columns q*16.. (H_p leaves
  // rows above 16p and the unit columns left of 16p alone)
  for (int i = 0; i < p.nQ; i++) {
    const int q = rank + i * S;
    if (q >= p.np) break;
    cplx* C = Qs + i * sl;
    for (int t = tid; t < m * CQ_NB; t += CQ_T) {
      const int r = t % m, j = q * CQ_NB + t / m;
      C[t] = make_double2((r == j && j < p.K) ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int pn = q; pn >= 0; pn--) {
      const int owner = pn % S, li = pn / S;
      const int j0 = pn * CQ_NB, jb = min(CQ_NB, p.K - j0);
      cq_stage(cl.map_shared_rank(As + li * sl, owner), cl.map_shared_rank(Tl + li * 256, owner), m, j0, jb, Vs, Ts);
      cq_apply(C, m, j0, Vs, Ts, false, W, W2);
    }
  }

  // R (K x n): the upper trapezoid of the factored slices; Q (m x K)
  if (p.R) {
    for (int i = 0; i < p.nA; i++) {
      const int q = rank + i * S;
      if (q >= p.npa) break;
      for (int t = tid; t < p.K * CQ_NB; t += CQ_T) {
        const int r = t % p.K, j = q * CQ_NB + t / p.K;
        if (j < p.n) p.R[r + (long long)j * p.ldr] = r <= j ? As[i * sl + r + (long long)(j - q * CQ_NB) * m]
                                                            : make_double2(0.0, 0.0);
      }
    }
  }
  if (p.Q) {
    for (int i = 0; i < p.nQ; i++) {
      const int q = rank + i * S;
      if (q >= p.np) break;
      for (int t = tid; t < m * CQ_NB; t += CQ_T) {
        const int r = t % m, j = q * CQ_NB + t / m;
        if (j < p.K) p.Q[r + (long long)j * p.ldq] = Qs[i * sl + t];
      }
    }
  }
  cl.sync();  // the panels stay in shared memory until every CTA has read them
}

// Dynamic shared memory limit of the cluster kernel (the largest plan, m =
// 256 with one slice of A and one of Q per CTA, takes 215 KB).
constexpr size_t CQ_SMEM_ATTR = 225 * 1024;
static_assert(cq_smem_elems(CQ_MAXM, 1, 1) * sizeof(cplx) <= CQ_SMEM_ATTR, "cluster QR plan exceeds its limit");

std::atomic<unsigned long long> g_cq_setup{0};
bool g_cq_ok[64] = {false};

// The cluster QR when the matrix fits (m <= 256 and its slices within the
// shared-memory limit) and the device can place a cluster of 8 such CTAs;
// false otherwise (the caller then runs the global-memory kernels).
bool cluster_qr(const Stream& st, int m, int n, const cplx* A, cplx* Q, long long ldq, cplx* R, long long ldr) {
  if (m > CQ_MAXM) return false;
  CqParams p;
  p.m = m; p.n = n; p.K = std::min(m, n);
  p.npa = ceil_div(n, CQ_NB);
  p.np = ceil_div(p.K, CQ_NB);
  p.S = std::min(CQ_MAXS, p.npa);
  p.nA = ceil_div(p.npa, p.S);
  p.nQ = ceil_div(p.np, p.S);
  const size_t smem = cq_smem_elems(m, p.nA, p.nQ) * sizeof(cplx);
  if (smem > CQ_SMEM_ATTR) return false;
  int dev = 0;
  MPSGPU_CUDA(cudaGetDevice(&dev));
  if (dev >= 64) return false;
  if (device_needs_setup(g_cq_setup)) {
    MPSGPU_CUDA(cudaFuncSetAttribute(qr_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)CQ_SMEM_ATTR));
    // can a cluster of the largest size and plan be placed at all?
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CQ_MAXS);
    cfg.blockDim = dim3(CQ_T);
    cfg.dynamicSmemBytes = cq_smem_elems(CQ_MAXM, 1, 1) * sizeof(cplx);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CQ_MAXS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    g_cq_ok[dev] = cudaOccupancyMaxActiveClusters(&clusters, qr_cluster_kernel, &cfg) == cudaSuccess && clusters > 0;
    (void)cudaGetLastError();
    mark_device_done(g_cq_setup);
  }
  if (!g_cq_ok[dev]) return false;
  p.A = A; p.Q = Q; p.ldq = ldq; p.R = R; p.ldr = ldr;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(p.S);
  cfg.blockDim = dim3(CQ_T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st.s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.S;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  MPSGPU_CUDA(cudaLaunchKernelEx(&cfg, qr_cluster_kernel, p));
  after_launch(st);
  return true;
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
  if (cluster_qr(st, m, n, A, Q, ldq, R, ldr)) return;
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
