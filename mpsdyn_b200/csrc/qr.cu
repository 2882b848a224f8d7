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

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; w++) s += red[w];
  return s;
}

__device__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; w++) s = fmax(s, red[w]);
  return s;
}

// 2-norm of x[0..n) without underflow or overflow of the squares: the
// entries are divided by the largest component magnitude before squaring
// (the scaled sum of LAPACK's dznrm2).  Rank-deficient sites produce
// trailing columns with entries far below 1e-154, whose plain squares
// underflow to zero.  Every thread of the block gets the result.
__device__ double block_scaled_norm(int n, const cplx* x, double* red) {
  double mx = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) mx = fmax(mx, fmax(fabs(x[r].x), fabs(x[r].y)));
  mx = block_max(mx, red);
  if (mx == 0.0) return 0.0;
  const double inv = 1.0 / mx;
  double part = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double a = x[r].x * inv, b = x[r].y * inv;
    part += a * a + b * b;
  }
  return mx * sqrt(block_sum(part, red));
}

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

// Apply (I - V T' V^H) to the mp x cw column slice C (shared, ld = mp), where
// V (mp x jb, unit lower trapezoidal) and T (jb x jb) are in global memory
// and T' = T^H (conjT = true, for Q^H A) or T (for Q E).  W is jb x cw shared.
__device__ void apply_block_reflector(int mp, int jb, int cw, const cplx* __restrict__ V,
                                      long long ldv, const cplx* __restrict__ T, int ldt,
                                      bool conjT, cplx* C, int ldc, cplx* W, cplx* W2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // W[l, q] = sum_r conj(V[r, l]) C[r, q]  (V[r,l] = 0 for r < l, 1 for r = l)
  for (int t = warp; t < jb * cw; t += nw) {
    int l = t % jb, q = t / jb;
    cplx s = make_double2(0.0, 0.0);
    for (int r = l + lane; r < mp; r += 32) {
      cplx v = (r == l) ? make_double2(1.0, 0.0) : V[r + (long long)l * ldv];
      s = cadd(s, ccmul(v, C[r + q * ldc]));
    }
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) W[l + q * jb] = s;
  }
  __syncthreads();
  // W2 = T' W  (T' = T^H lower triangular, or T upper triangular)
  for (int t = threadIdx.x; t < jb * cw; t += blockDim.x) {
    int i = t % jb, q = t / jb;
    cplx s = make_double2(0.0, 0.0);
    if (conjT) {
      for (int l = 0; l <= i; l++) s = cadd(s, ccmul(T[l + i * ldt], W[l + q * jb]));
    } else {
      for (int l = i; l < jb; l++) s = cadd(s, cmul(T[i + l * ldt], W[l + q * jb]));
    }
    W2[i + q * jb] = s;
  }
  __syncthreads();
  // C -= V W2
  for (int t = threadIdx.x; t < mp * cw; t += blockDim.x) {
    int r = t % mp, q = t / mp;
    cplx s = make_double2(0.0, 0.0);
    int lmax = min(r, jb - 1);
    for (int l = 0; l <= lmax; l++) {
      cplx v = (r == l) ? make_double2(1.0, 0.0) : V[r + (long long)l * ldv];
      s = cadd(s, cmul(v, W2[l + q * jb]));
    }
    C[r + q * ldc] = csub(C[r + q * ldc], s);
  }
  __syncthreads();
}

struct QrParams {
  int m, n, K, nb, npanel;
  cplx* A;      // m x n, ld = m (in: matrix; out: R above, V below the diagonal)
  cplx* T;      // npanel blocks of nb x nb
  cplx* tau;    // K
};

__global__ void __launch_bounds__(QR_THREADS) qr_factor_kernel(QrParams p) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double smem_d[];
  cplx* sm = reinterpret_cast<cplx*>(smem_d);
  __shared__ double red[QR_THREADS / 32];
  __shared__ cplx Wsh[16 * 16], W2sh[16 * 16];
  __shared__ cplx coef;
  const int m = p.m, nb = p.nb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;

  for (int pi = 0; pi < p.npanel; pi++) {
    const int j0 = pi * nb;
    const int jb = min(nb, p.K - j0);
    const int mp = m - j0;
    cplx* Tp = p.T + (long long)pi * nb * nb;
    if (blockIdx.x == 0) {
      cplx* P = sm;  // mp x jb, ld = mp
      for (int t = threadIdx.x; t < mp * jb; t += blockDim.x) {
        int r = t % mp, c = t / mp;
        P[t] = p.A[(j0 + r) + (long long)(j0 + c) * m];
      }
      __syncthreads();
      for (int c = 0; c < jb; c++) {
        // reflector of column c, rows c..mp-1 (block-uniform control flow:
        // every thread holds the same norms, alpha and beta)
        cplx* x = P + (c + 1) + c * mp;
        const int nx = mp - c - 1;
        double xnorm = block_scaled_norm(nx, x, red);
        cplx alpha = P[c + c * mp];
        cplx tau, scale;
        bool ident = (xnorm == 0.0 && alpha.y == 0.0);
        double beta = 0.0;
        if (ident) {
          tau = make_double2(0.0, 0.0);
          scale = make_double2(0.0, 0.0);
        } else {
          double nrm = hypot3(alpha.x, alpha.y, xnorm);
          beta = alpha.x >= 0.0 ? -nrm : nrm;
          // |beta| below kSafeMin: scale the column up (at most 20 times)
          // so that 1 / (alpha - beta) stays finite; beta is scaled back
          // at the end, tau and v are scale-invariant
          int knt = 0;
          while (fabs(beta) < kSafeMin && knt < 20) {
            __syncthreads();
            for (int r = threadIdx.x; r < nx; r += blockDim.x) x[r] = cscale(x[r], 1.0 / kSafeMin);
            beta /= kSafeMin;
            alpha = cscale(alpha, 1.0 / kSafeMin);
            knt++;
          }
          if (knt > 0) {
            __syncthreads();
            xnorm = block_scaled_norm(nx, x, red);
            nrm = hypot3(alpha.x, alpha.y, xnorm);
            beta = alpha.x >= 0.0 ? -nrm : nrm;
          }
          tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
          scale = recip_smith(make_double2(alpha.x - beta, alpha.y));
          for (int k = 0; k < knt; k++) beta *= kSafeMin;
        }
        __syncthreads();
        if (!ident) {
          for (int r = threadIdx.x; r < nx; r += blockDim.x) x[r] = cmul(x[r], scale);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          if (!ident) P[c + c * mp] = make_double2(beta, 0.0);
          p.tau[j0 + c] = tau;
          coef = cconj(tau);
        }
        __syncthreads();
        // apply H^H = I - conj(tau) v v^H to panel columns c+1..jb-1
        if (!ident) {
          for (int q = c + 1 + warp; q < jb; q += nw) {
            cplx s = make_double2(0.0, 0.0);
            for (int r = c + lane; r < mp; r += 32) {
              cplx v = (r == c) ? make_double2(1.0, 0.0) : P[r + c * mp];
              s = cadd(s, ccmul(v, P[r + q * mp]));
            }
            for (int o = 16; o > 0; o >>= 1) {
              s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
              s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
            }
            s = cmul(coef, s);
            for (int r = c + lane; r < mp; r += 32) {
              cplx v = (r == c) ? make_double2(1.0, 0.0) : P[r + c * mp];
              P[r + q * mp] = csub(P[r + q * mp], cmul(v, s));
            }
          }
        }
        __syncthreads();
      }
      // T factor (zlarft forward, columnwise)
      for (int i = 0; i < jb; i++) {
        cplx ti = p.tau[j0 + i];
        // Wsh[l] = -tau_i * sum_r conj(V[r,l]) v_i[r], l < i
        for (int l = warp; l < i; l += nw) {
          cplx s = make_double2(0.0, 0.0);
          for (int r = i + lane; r < mp; r += 32) {
            cplx vl = P[r + l * mp];  // r > l always (r >= i > l)
            cplx vi = (r == i) ? make_double2(1.0, 0.0) : P[r + i * mp];
            s = cadd(s, ccmul(vl, vi));
          }
          for (int o = 16; o > 0; o >>= 1) {
            s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
            s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
          }
          if (lane == 0) Wsh[l] = cmul(make_double2(-ti.x, -ti.y), s);
        }
        __syncthreads();
        // T[0:i, i] = T[0:i, 0:i] * Wsh
        for (int l = threadIdx.x; l < i; l += blockDim.x) {
          cplx s = make_double2(0.0, 0.0);
          for (int q = l; q < i; q++) s = cadd(s, cmul(Tp[l + q * nb], Wsh[q]));
          W2sh[l] = s;
        }
        __syncthreads();
        for (int l = threadIdx.x; l < nb; l += blockDim.x) {
          cplx v = make_double2(0.0, 0.0);
          if (l < i) v = W2sh[l];
          else if (l == i) v = ti;
          Tp[l + i * nb] = v;
        }
        __threadfence_block();
        __syncthreads();
      }
      // write the panel back
      for (int t = threadIdx.x; t < mp * jb; t += blockDim.x) {
        int r = t % mp, c = t / mp;
        p.A[(j0 + r) + (long long)(j0 + c) * m] = P[t];
      }
      __threadfence();
    }
    grid.sync();
    // trailing update of columns j0+jb .. n-1 in slices of nb columns
    const int first = j0 + jb;
    const int nslices = (p.n - first + nb - 1) / nb;
    const cplx* V = p.A + j0 + (long long)j0 * m;  // mp x jb, ld = m
    for (int sl = blockIdx.x; sl < nslices; sl += gridDim.x) {
      int c0 = first + sl * nb;
      int cw = min(nb, p.n - c0);
      cplx* C = sm;  // mp x cw
      for (int t = threadIdx.x; t < mp * cw; t += blockDim.x) {
        int r = t % mp, c = t / mp;
        C[t] = p.A[(j0 + r) + (long long)(c0 + c) * m];
      }
      __syncthreads();
      apply_block_reflector(mp, jb, cw, V, m, Tp, nb, true, C, mp, Wsh, W2sh);
      for (int t = threadIdx.x; t < mp * cw; t += blockDim.x) {
        int r = t % mp, c = t / mp;
        p.A[(j0 + r) + (long long)(c0 + c) * m] = C[t];
      }
      __syncthreads();
    }
    __threadfence();
    grid.sync();
  }
}

// Form Q (m x K) slice by slice and extract R (K x n, zero below the diagonal).
__global__ void __launch_bounds__(QR_THREADS) qr_form_q_kernel(QrParams p, cplx* Q, long long ldq,
                                                               cplx* R, long long ldr) {
  extern __shared__ double smem_d[];
  cplx* sm = reinterpret_cast<cplx*>(smem_d);
  __shared__ cplx Wsh[16 * 16], W2sh[16 * 16];
  const int m = p.m, nb = p.nb;
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
    cplx* C = sm;  // m x cw : columns c0.. of the identity
    for (int t = threadIdx.x; t < m * cw; t += blockDim.x) {
      int r = t % m, c = t / m;
      C[t] = make_double2(r == c0 + c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int pi = p.npanel - 1; pi >= 0; pi--) {
      const int j0 = pi * nb;
      const int jb = min(nb, p.K - j0);
      // H_j only touch rows >= j0; columns c < j0 of E stay unit vectors above
      apply_block_reflector(m - j0, jb, cw, p.A + j0 + (long long)j0 * m, m,
                            p.T + (long long)pi * nb * nb, nb, false, C + j0, m, Wsh, W2sh);
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
  MPSGPU_CHECK(m <= 1280, MPSGPU_BAD_SHAPE, "qr: more than 1280 rows is not supported");
  QrParams p;
  p.m = m; p.n = n; p.K = K; p.nb = nb; p.npanel = (K + nb - 1) / nb;
  p.A = A;
  char* ws = (char*)scratch.get((size_t)p.npanel * nb * nb * sizeof(cplx) + (size_t)K * sizeof(cplx) + 256);
  p.T = (cplx*)ws;
  p.tau = p.T + (size_t)p.npanel * nb * nb;
  size_t smem = (size_t)m * nb * sizeof(cplx);
  static std::atomic<unsigned long long> attr_done{0};
  if (device_needs_setup(attr_done)) {
    MPSGPU_CUDA(cudaFuncSetAttribute(qr_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    MPSGPU_CUDA(cudaFuncSetAttribute(qr_form_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
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
// block-reflector factors T and the scalars tau.  The array is reserved when
// the library is loaded, on every GPU that loads it, and held until exit.
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
    if (cudaFuncSetAttribute(qr_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) !=
            cudaSuccess ||
        cudaFuncSetAttribute(qr_form_q_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) !=
            cudaSuccess)
      return MPSGPU_CUDA_ERROR;
    g_noalloc_attr[dev] = true;
  }
  *out = g_noalloc_ptr[dev];
  return MPSGPU_OK;
}

}  // namespace
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
  const size_t smem = (size_t)m * NOALLOC_NB * sizeof(double2);
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
  qr_form_q_kernel<<<qgrid, QR_THREADS, smem, s>>>(p, reinterpret_cast<double2*>(Q), m,
                                                   reinterpret_cast<double2*>(R), K);
  if (cudaGetLastError() != cudaSuccess) return MPSGPU_CUDA_ERROR;
  return MPSGPU_OK;
}
