// Bandwidth-bound kernels of the sweep: the MPO-leg contraction between the
// two GEMMs of every matvec / environment update, the Lanczos vector
// operations (classical Gram-Schmidt projections, norms, scaling), layout
// conversions and the seeded Gaussian generator.  All complex FP64.
#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int TPB = 256;

inline int grid_for(long long n, int tpb = TPB, int cap = 148 * 16) {
  long long g = (n + tpb - 1) / tpb;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// ---- MPO-leg contraction ---------------------------------------------------
// One thread per pixel (x, y); x is the fastest (unit-stride) coordinate of
// both input and output, so loads and stores coalesce.  The small matrix Wm
// (nout x nin complex) sits in shared memory; the pixel's nin inputs stay in
// registers (NIN is the compile-time bound of nin).
constexpr int WMAX = 32;

template <int NIN>
__global__ void wcontract_kernel(WContractArgs a) {
  extern __shared__ double wsm[];
  cplx* wm = reinterpret_cast<cplx*>(wsm);
  const int nin = a.n_i0 * a.n_i1, nout = a.n_o0 * a.n_o1;
  for (int t = threadIdx.x; t < nin * nout; t += blockDim.x) wm[t] = a.Wm[t];
  __syncthreads();
  const long long npix = (long long)a.nx * a.ny;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % a.nx), y = (int)(p / a.nx);
    cplx in[NIN];
    const cplx* ib = a.in + x * a.ix + y * a.iy;
#pragma unroll
    for (int i = 0; i < NIN; i++) {
      if (i < nin) {
        const int i0 = i % a.n_i0, i1 = i / a.n_i0;
        in[i] = ib[i0 * a.si0 + i1 * a.si1];
      } else {
        in[i] = make_double2(0.0, 0.0);
      }
    }
    cplx* ob = a.out + x * a.ox + y * a.oy;
    for (int o = 0; o < nout; o++) {
      const int o0 = o % a.n_o0, o1 = o / a.n_o0;
      cplx s = make_double2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < NIN; i++) {
        if (i < nin) {
          const cplx w = wm[o + nout * i];
          s.x += w.x * in[i].x - w.y * in[i].y;
          s.y += w.x * in[i].y + w.y * in[i].x;
        }
      }
      ob[o0 * a.so0 + o1 * a.so1] = s;
    }
  }
}

// Same contraction for leg products above WMAX (the doubled operator O^dag O
// of contract2 has w^2 legs): the inputs are read from global memory (L1)
// for every output instead of being held in registers.
__global__ void wcontract_wide_kernel(WContractArgs a) {
  extern __shared__ double wsm[];
  cplx* wm = reinterpret_cast<cplx*>(wsm);
  const int nin = a.n_i0 * a.n_i1, nout = a.n_o0 * a.n_o1;
  for (int t = threadIdx.x; t < nin * nout; t += blockDim.x) wm[t] = a.Wm[t];
  __syncthreads();
  const long long npix = (long long)a.nx * a.ny;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % a.nx), y = (int)(p / a.nx);
    const cplx* ib = a.in + x * a.ix + y * a.iy;
    cplx* ob = a.out + x * a.ox + y * a.oy;
    for (int o = 0; o < nout; o++) {
      const int o0 = o % a.n_o0, o1 = o / a.n_o0;
      cplx s = make_double2(0.0, 0.0);
      for (int i = 0; i < nin; i++) {
        const int i0 = i % a.n_i0, i1 = i / a.n_i0;
        const cplx v = ib[i0 * a.si0 + i1 * a.si1];
        const cplx w = wm[o + nout * i];
        s.x += w.x * v.x - w.y * v.y;
        s.y += w.x * v.y + w.y * v.x;
      }
      ob[o0 * a.so0 + o1 * a.so1] = s;
    }
  }
}

// ---- Gram-Schmidt projections ----------------------------------------------
constexpr int DOT_CHUNK = 4096;

// partial[j * nblk + b] = sum over rows of chunk b of conj(V[:, j]) w
__global__ void cgemv_c_partial(int n, int k, const cplx* __restrict__ V, long long ldv,
                                const cplx* __restrict__ w, cplx* __restrict__ partial, int nblk) {
  __shared__ double rs[TPB / 32], is[TPB / 32];
  const int b = blockIdx.x, j = blockIdx.y;
  const int r0 = b * DOT_CHUNK, r1 = min(n, r0 + DOT_CHUNK);
  const cplx* v = V + (long long)j * ldv;
  cplx s = make_double2(0.0, 0.0);
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) s = cadd(s, ccmul(v[r], w[r]));
  for (int o = 16; o > 0; o >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { rs[warp] = s.x; is[warp] = s.y; }
  __syncthreads();
  if (threadIdx.x == 0) {
    cplx t = make_double2(0.0, 0.0);
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t = cadd(t, make_double2(rs[q], is[q]));
    partial[(long long)j * nblk + b] = t;
  }
}

__global__ void reduce_partials(int k, int nblk, const cplx* __restrict__ partial, cplx* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  cplx s = make_double2(0.0, 0.0);
  for (int b = 0; b < nblk; b++) s = cadd(s, partial[(long long)j * nblk + b]);
  out[j] = s;
}

__global__ void cgemv_n_sub_kernel(int n, int k, const cplx* __restrict__ V, long long ldv,
                                   const cplx* __restrict__ h, cplx* __restrict__ w, double sign) {
  __shared__ cplx hs[256];
  for (int t = threadIdx.x; t < k; t += blockDim.x) hs[t] = h[t];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    cplx s = make_double2(0.0, 0.0);
    for (int j = 0; j < k; j++) s = cadd(s, cmul(V[i + j * ldv], hs[j]));
    w[i] = cadd(w[i], cscale(s, sign));
  }
}

__global__ void nrm2_partial(int n, const cplx* __restrict__ x, double* __restrict__ partial) {
  __shared__ double rs[TPB / 32];
  const int r0 = blockIdx.x * DOT_CHUNK, r1 = min(n, r0 + DOT_CHUNK);
  double s = 0.0;
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) s += cabs2(x[r]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) rs[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += rs[q];
    partial[blockIdx.x] = t;
  }
}

__global__ void nrm2_final(int nblk, const double* __restrict__ partial, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += partial[b];
    out[0] = sqrt(s);
  }
}

__global__ void zscal_inv_kernel(int n, const cplx* __restrict__ x, const double* __restrict__ nrm,
                                 cplx* __restrict__ y) {
  const double inv = 1.0 / nrm[0];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cscale(x[i], inv);
}

__global__ void zaxpby_kernel(int n, cplx a, const cplx* __restrict__ x, cplx b, cplx* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = cadd(cmul(a, x[i]), cmul(b, y[i]));
}

__global__ void combine_real_kernel(int n, int k, const cplx* __restrict__ V, long long ldv,
                                    const double* __restrict__ s, cplx* __restrict__ y) {
  __shared__ double ss[256];
  for (int t = threadIdx.x; t < k; t += blockDim.x) ss[t] = s[t];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    cplx acc = make_double2(0.0, 0.0);
    for (int j = 0; j < k; j++) acc = cadd(acc, cscale(V[i + j * ldv], ss[j]));
    y[i] = acc;
  }
}

__global__ void zcopy_kernel(long long n, const cplx* __restrict__ s, cplx* __restrict__ d) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = s[i];
}

__global__ void zfill_kernel(long long n, cplx v, cplx* __restrict__ d) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = v;
}

// ---- layouts -----------------------------------------------------------------
// ref A(s, a, r) at s + d a + d Dl r  <->  dev X(a, s, r) at a + Dl s + Dl d r
__global__ void site_ref_to_dev_kernel(int d, int Dl, int Dr, const cplx* __restrict__ ref,
                                       cplx* __restrict__ dev) {
  const long long n = (long long)d * Dl * Dr;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int a = (int)(t % Dl);
    long long rest = t / Dl;
    int s = (int)(rest % d);
    long long r = rest / d;
    dev[t] = ref[s + (long long)d * a + (long long)d * Dl * r];
  }
}

__global__ void site_dev_to_ref_kernel(int d, int Dl, int Dr, const cplx* __restrict__ dev,
                                       cplx* __restrict__ ref) {
  const long long n = (long long)d * Dl * Dr;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int s = (int)(t % d);
    long long rest = t / d;
    int a = (int)(rest % Dl);
    long long r = rest / Dl;
    ref[t] = dev[a + (long long)Dl * s + (long long)Dl * d * r];
  }
}

__global__ void transpose_pqr_kernel(int P, int Q, int R, const cplx* __restrict__ in,
                                     cplx* __restrict__ out, bool conj) {
  const long long n = (long long)P * Q * R;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    // out(r, q, p) at r + R q + R Q p ; t enumerates out
    int r = (int)(t % R);
    long long rest = t / R;
    int q = (int)(rest % Q);
    long long p = rest / Q;
    cplx v = in[p + (long long)P * q + (long long)P * Q * r];
    if (conj) v.y = -v.y;
    out[t] = v;
  }
}

__device__ __forceinline__ uint64_t splitmix64_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void gaussian_site_kernel(uint64_t seed, long long offset, int d, int Dl, int Dr,
                                     cplx* __restrict__ dev) {
  const long long n = (long long)d * Dl * Dr;
  const double two_pi = 6.283185307179586476925286766559;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    // t enumerates the reference order (s fastest)
    int s = (int)(t % d);
    long long rest = t / d;
    int a = (int)(rest % Dl);
    long long r = rest / Dl;
    uint64_t e = (uint64_t)(offset + t);
    uint64_t z1 = splitmix64_at(seed, 2 * e), z2 = splitmix64_at(seed, 2 * e + 1);
    double u1 = ((double)(z1 >> 11) + 0.5) * 0x1.0p-53;
    double u2 = ((double)(z2 >> 11) + 0.5) * 0x1.0p-53;
    double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincos(two_pi * u2, &sn, &cs);
    dev[a + (long long)Dl * s + (long long)Dl * d * r] = make_double2(rad * cs, rad * sn);
  }
}

__device__ __forceinline__ long long view_off(const View2& v, long long i, long long j) {
  return (i % v.rd) * v.r0 + (i / v.rd) * v.r1 + (j % v.cd) * v.c0 + (j / v.cd) * v.c1;
}

__global__ void gather2_kernel(int m, int n, const cplx* __restrict__ src, View2 v,
                               cplx* __restrict__ dst) {
  const long long tot = (long long)m * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    long long i = t % m, j = t / m;
    cplx x = src[view_off(v, i, j)];
    if (v.conj) x.y = -x.y;
    dst[t] = x;
  }
}

__global__ void scatter2_kernel(int m, int n, const cplx* __restrict__ src, cplx* __restrict__ dst,
                                View2 v) {
  const long long tot = (long long)m * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    long long i = t % m, j = t / m;
    cplx x = src[t];
    if (v.conj) x.y = -x.y;
    dst[view_off(v, i, j)] = x;
  }
}

}  // namespace

void wcontract(const Stream& st, const WContractArgs& a) {
  const int nin = a.n_i0 * a.n_i1, nout = a.n_o0 * a.n_o1;
  long long npix = (long long)a.nx * a.ny;
  if (npix <= 0) return;
  const size_t smem = (size_t)nin * nout * sizeof(cplx);
  const int grid = grid_for(npix, 128);
  if (nin > WMAX || nout > WMAX) {
    MPSGPU_CHECK(smem <= 48 * 1024, MPSGPU_BAD_SHAPE,
                 "wcontract: MPO leg product too large (nin * nout <= 3072)");
    wcontract_wide_kernel<<<grid, 128, smem, st.s>>>(a);
    after_launch(st);
    return;
  }
  if (nin <= 4) wcontract_kernel<4><<<grid, 128, smem, st.s>>>(a);
  else if (nin <= 8) wcontract_kernel<8><<<grid, 128, smem, st.s>>>(a);
  else if (nin <= 16) wcontract_kernel<16><<<grid, 128, smem, st.s>>>(a);
  else wcontract_kernel<32><<<grid, 128, smem, st.s>>>(a);
  after_launch(st);
}

void cgemv_c(const Stream& st, int n, int k, const cplx* V, long long ldv, const cplx* w, cplx* dots,
             Scratch& scratch) {
  if (k <= 0) return;
  int nblk = ceil_div(n, DOT_CHUNK);
  cplx* partial = (cplx*)scratch.get((size_t)nblk * k * sizeof(cplx));
  cgemv_c_partial<<<dim3(nblk, k), TPB, 0, st.s>>>(n, k, V, ldv, w, partial, nblk);
  after_launch(st);
  reduce_partials<<<ceil_div(k, 64), 64, 0, st.s>>>(k, nblk, partial, dots);
  after_launch(st);
}

void cgemv_n_sub(const Stream& st, int n, int k, const cplx* V, long long ldv, const cplx* h, cplx* w,
                 double sign) {
  MPSGPU_CHECK(k <= 256, MPSGPU_BAD_SHAPE, "cgemv_n_sub: k > 256");
  if (k <= 0) return;
  cgemv_n_sub_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, k, V, ldv, h, w, sign);
  after_launch(st);
}

void dznrm2(const Stream& st, int n, const cplx* x, double* out, Scratch& scratch) {
  int nblk = ceil_div(n, DOT_CHUNK);
  double* partial = (double*)scratch.get((size_t)nblk * sizeof(double));
  nrm2_partial<<<nblk, TPB, 0, st.s>>>(n, x, partial);
  after_launch(st);
  nrm2_final<<<1, 32, 0, st.s>>>(nblk, partial, out);
  after_launch(st);
}

void zscal_inv(const Stream& st, int n, const cplx* x, const double* nrm, cplx* y) {
  zscal_inv_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, x, nrm, y);
  after_launch(st);
}

void zaxpby(const Stream& st, int n, cplx a, const cplx* x, cplx b, cplx* y) {
  zaxpby_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, a, x, b, y);
  after_launch(st);
}

void combine_real(const Stream& st, int n, int k, const cplx* V, long long ldv, const double* s, cplx* y) {
  MPSGPU_CHECK(k <= 256, MPSGPU_BAD_SHAPE, "combine_real: k > 256");
  combine_real_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, k, V, ldv, s, y);
  after_launch(st);
}

void zcopy(const Stream& st, int n, const cplx* src, cplx* dst) {
  if (n <= 0) return;
  zcopy_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, src, dst);
  after_launch(st);
}

void zfill(const Stream& st, long long n, cplx v, cplx* dst) {
  if (n <= 0) return;
  zfill_kernel<<<grid_for(n), TPB, 0, st.s>>>(n, v, dst);
  after_launch(st);
}

void site_ref_to_dev(const Stream& st, int d, int Dl, int Dr, const cplx* ref, cplx* dev) {
  site_ref_to_dev_kernel<<<grid_for((long long)d * Dl * Dr), TPB, 0, st.s>>>(d, Dl, Dr, ref, dev);
  after_launch(st);
}

void site_dev_to_ref(const Stream& st, int d, int Dl, int Dr, const cplx* dev, cplx* ref) {
  site_dev_to_ref_kernel<<<grid_for((long long)d * Dl * Dr), TPB, 0, st.s>>>(d, Dl, Dr, dev, ref);
  after_launch(st);
}

void transpose_pqr_to_rqp(const Stream& st, int p, int q, int r, const cplx* in, cplx* out, bool conj) {
  transpose_pqr_kernel<<<grid_for((long long)p * q * r), TPB, 0, st.s>>>(p, q, r, in, out, conj);
  after_launch(st);
}

void gaussian_site(const Stream& st, uint64_t seed, long long offset, int d, int Dl, int Dr, cplx* dev) {
  gaussian_site_kernel<<<grid_for((long long)d * Dl * Dr), TPB, 0, st.s>>>(seed, offset, d, Dl, Dr, dev);
  after_launch(st);
}

void gather2(const Stream& st, int m, int n, const cplx* src, const View2& v, cplx* dst) {
  gather2_kernel<<<grid_for((long long)m * n), TPB, 0, st.s>>>(m, n, src, v, dst);
  after_launch(st);
}

void scatter2(const Stream& st, int m, int n, const cplx* src, cplx* dst, const View2& v) {
  scatter2_kernel<<<grid_for((long long)m * n), TPB, 0, st.s>>>(m, n, src, dst, v);
  after_launch(st);
}

}  // namespace mpsgpu
