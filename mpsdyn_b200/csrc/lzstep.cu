// One reorthogonalised Lanczos step for a group of independent local
// eigenproblems, in a single cooperative launch (replaces the
// orthogonalisation inside the PRIMME call of Contractor::solveEigs,
// src/core/cpp/Contractor.cpp:3067-3138).
//
// For every instance q, with k = j+1 basis vectors V[:, 0..j] and
// w = (H - sigma) v_j computed by the matvec:
//   projector  w += U (U^H v_j)        (excited states: U holds sqrt(pen) u_t)
//   pass 1     w' = w - beta_{j-1} v_{j-1};  h = V^H w', |w'|^2;  w'' = w' - V h
//   pass 2     only when |w''|^2 < |w'|^2 / 2 (Daniel, Gragg, Kaufman,
//              Stewart 1976): h2 = V^H w''; w''' = w'' - V h2
//   alpha_j = sigma + Re(h_j + h2_j), beta_j = |w|, V[:, j+1] = w / beta_j.
// Without a second pass |w''|^2 = |w'|^2 - |h|^2 (V orthonormal; the test
// bounds the cancellation to a factor 2), so beta_j is known before the
// update and the update writes v_{j+1} directly.
//
// Work split: the rows of an instance are cut into row blocks of 256 (one
// row per thread), and every instance owns its own set of CTAs, which take
// its row blocks in strided order.  Partial sums per row block go to global
// memory; after a barrier among the instance's CTAs every one of them sums
// the partials of the instance itself, in the same fixed order, so all of
// them hold the same coefficients and reach the same second-pass decision
// without a second barrier.  An unflagged step therefore costs one barrier
// among the instance's CTAs; the results are identical from run to run and do
// not depend on the other instances of the group or on the CTA count.
// Barriers are bounded: a CTA that waits longer than 2 s sets the error word
// and returns (the host reports MPSGPU_TIMEOUT and resets the barrier words);
// the kernel has no copies in flight at any barrier.
#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

constexpr int T = LZ_THREADS;         // threads per CTA
constexpr int RB = T;                 // rows per row block (one per thread)
constexpr int NW = T / 32;
constexpr int KMAXS = 256;            // Krylov vectors
constexpr double DGKS2 = 0.5;

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded barrier over the n co-resident CTAs of one instance: bar[0] counts
// the arrivals, bar[1] is the generation the last arrival advances.  Returns
// false (and sets *err) when the wait ran out.
__device__ bool group_barrier(unsigned* bar, unsigned n, int* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == n - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = gtimer();
      while (*gen == g) {
        __nanosleep(32);
        if (gtimer() - t0 > 2000000000ull) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ double warp_sumd(double s) {
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

__device__ __forceinline__ cplx warp_sumc(cplx s) {
  for (int o = 16; o > 0; o >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
  }
  return s;
}

// Sum of v[0..15] over the 32 lanes of a warp by a transposing butterfly:
// every exchange step halves the values a lane keeps, so afterwards the
// lanes with (lane & 1) == 0 hold the totals, lane L the one of vector
// sum16_vector_of_lane(L).
__device__ __forceinline__ cplx warp_sum16(cplx (&v)[16]) {
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
// lane bits (4, 3, 2, 1) select vector 8*b4 + 4*b3 + 2*b2 + b1
__device__ __forceinline__ int sum16_vector_of_lane(int lane) {
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}

// Partial dots over the rows [r0, r0 + RB) of an n-row instance:
// part[rb * KMAXS + l] = sum_rows conj(V[:, l]) x for l < k (V with leading
// dimension ldv), and the partial |x|^2 into pn[rb] when pn is non-null.
// Vectors go in groups of 16 whose loads are all issued before use; the
// warps' sums collect in shared memory (red, NW x KMAXS) and are added in a
// fixed order after one barrier.
__device__ void block_dots(const cplx* __restrict__ V, long long ldv, long long n, long long r0, int rb,
                           const cplx* __restrict__ x, int k, cplx* part, double* pn, cplx (*red)[KMAXS],
                           double* redn) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long row = r0 + tid;
  const bool ok = row < n;
  const cplx xv = ok ? x[row] : make_double2(0.0, 0.0);
  if (pn) {
    const double s = warp_sumd(cabs2(xv));
    if (lane == 0) redn[warp] = s;
  }
  const cplx* vr = V + (ok ? row : 0);
  for (int l0 = 0; l0 < k; l0 += 16) {
    cplx v[16];
#pragma unroll
    for (int t = 0; t < 16; t++)
      v[t] = (ok && l0 + t < k) ? __ldcg(&vr[(long long)(l0 + t) * ldv]) : make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < 16; t++) v[t] = ccmul(v[t], xv);
    const cplx r = warp_sum16(v);
    const int l = l0 + sum16_vector_of_lane(lane);
    if ((lane & 1) == 0 && l < k) red[warp][l] = r;
  }
  __syncthreads();
  for (int l = tid; l < k; l += T) {
    cplx s = make_double2(0.0, 0.0);
    for (int q = 0; q < NW; q++) s = cadd(s, red[q][l]);
    part[(long long)rb * KMAXS + l] = s;
  }
  if (pn && tid == 0) {
    double s = 0.0;
    for (int q = 0; q < NW; q++) s += redn[q];
    pn[rb] = s;
  }
  __syncthreads();
}

// x -= V h over row block r of the instance (h in shared memory, k entries);
// partial |x|^2 into pn[rb0 + r].  Sixteen loads of V in flight per thread.
__device__ void block_update(const LzInst& in, int r, cplx* __restrict__ x, const cplx* hs, int k, double* pn,
                             double* redn) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long i = (long long)r * RB + tid;
  double s2 = 0.0;
  if (i < in.n) {
    cplx a0 = make_double2(0.0, 0.0), a1 = a0, a2 = a0, a3 = a0;
    const cplx* v = in.V + i;
    for (int l0 = 0; l0 < k; l0 += 16) {
      cplx vv[16];
#pragma unroll
      for (int t = 0; t < 16; t++)
        vv[t] = l0 + t < k ? __ldcg(&v[(long long)(l0 + t) * in.ldv]) : make_double2(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < 16; t += 4) {
        if (l0 + t < k) a0 = cadd(a0, cmul(vv[t], hs[l0 + t]));
        if (l0 + t + 1 < k) a1 = cadd(a1, cmul(vv[t + 1], hs[l0 + t + 1]));
        if (l0 + t + 2 < k) a2 = cadd(a2, cmul(vv[t + 2], hs[l0 + t + 2]));
        if (l0 + t + 3 < k) a3 = cadd(a3, cmul(vv[t + 3], hs[l0 + t + 3]));
      }
    }
    const cplx xi = csub(x[i], cadd(cadd(a0, a1), cadd(a2, a3)));
    x[i] = xi;
    s2 = cabs2(xi);
  }
  s2 = warp_sumd(s2);
  if (lane == 0) redn[warp] = s2;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < NW; q++) s += redn[q];
    pn[in.rb0 + r] = s;
  }
  __syncthreads();
}

// x -= V h over row block r, then V[:, j+1] = x / beta (or x itself stored
// back into w when the basis is full: the residual the restart needs).  No
// reduction.
__device__ void block_update_final(const LzInst& in, int r, const cplx* hs, int k, double inv_beta) {
  const int tid = threadIdx.x;
  const long long i = (long long)r * RB + tid;
  if (i < in.n) {
    cplx a0 = make_double2(0.0, 0.0), a1 = a0, a2 = a0, a3 = a0;
    const cplx* v = in.V + i;
    for (int l0 = 0; l0 < k; l0 += 16) {
      cplx vv[16];
#pragma unroll
      for (int t = 0; t < 16; t++)
        vv[t] = l0 + t < k ? __ldcg(&v[(long long)(l0 + t) * in.ldv]) : make_double2(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < 16; t += 4) {
        if (l0 + t < k) a0 = cadd(a0, cmul(vv[t], hs[l0 + t]));
        if (l0 + t + 1 < k) a1 = cadd(a1, cmul(vv[t + 1], hs[l0 + t + 1]));
        if (l0 + t + 2 < k) a2 = cadd(a2, cmul(vv[t + 2], hs[l0 + t + 2]));
        if (l0 + t + 3 < k) a3 = cadd(a3, cmul(vv[t + 3], hs[l0 + t + 3]));
      }
    }
    const cplx xi = csub(in.w[i], cadd(cadd(a0, a1), cadd(a2, a3)));
    if (in.write_next) in.V[(long long)(in.j + 1) * in.ldv + i] = cscale(xi, inv_beta);
    else in.w[i] = xi;
  }
}

// out[l] = sum over the instance's nrb row blocks of part[r * KMAXS + l],
// l < k: one warp per coefficient, lanes over the row blocks, then the warp
// butterfly -- a fixed order, so every CTA of the instance gets the same
// values.  Every thread of the block calls it; out is read after a barrier.
__device__ void reduce_coeffs(const cplx* __restrict__ part, int nrb, int k, cplx* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int l = warp; l < k; l += NW) {
    cplx s = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int r = lane; r < nrb; r += 32) s = cadd(s, __ldcg(&part[(long long)r * KMAXS + l]));
    s = warp_sumc(s);
    if (lane == 0) out[l] = s;
  }
}

// sum over the row blocks of the instance of pn (fixed order; every thread
// of every CTA gets the same value)
__device__ double sum_norms(const LzInst& in, const double* pn, double* redn) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double s = 0.0;
  for (int r = tid; r < in.nrb; r += T) s += __ldcg(&pn[in.rb0 + r]);
  s = warp_sumd(s);
  __syncthreads();
  if (lane == 0) redn[warp] = s;
  __syncthreads();
  double t = 0.0;
  for (int q = 0; q < NW; q++) t += redn[q];
  __syncthreads();
  return t;
}

// sum_l |h_l|^2 over l < k in a fixed order (every thread gets the value)
__device__ double coeff_norm(const cplx* hs, int k, double* redn) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (warp == 0) {
    double s = 0.0;
    for (int l = lane; l < k; l += 32) s += cabs2(hs[l]);
    s = warp_sumd(s);
    if (lane == 0) redn[0] = s;
  }
  __syncthreads();
  const double v = redn[0];
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(T) lanczos_step_kernel(const __grid_constant__ LzBatch b) {
  __shared__ cplx red[NW][KMAXS];
  __shared__ double redn[NW];
  __shared__ cplx hs[KMAXS];
  __shared__ cplx hs2[KMAXS];
  __shared__ cplx ucs[LZ_MAXU];
  const int tid = threadIdx.x;
  // the instance this CTA serves (instances own consecutive CTA ranges)
  int q = 0;
  while (q + 1 < b.ninst && b.in[q + 1].cta0 <= (int)blockIdx.x) q++;
  const LzInst& in = b.in[q];
  const int rank = (int)blockIdx.x - in.cta0;
  if (rank < 0 || rank >= in.ncta) return;
  unsigned* bar = b.bar + 2 * q;
  const unsigned nct = (unsigned)in.ncta;

  // ---- projector (excited states): c = U^H v_j, then w += U c ----
  if (in.nu > 0) {
    for (int r = rank; r < in.nrb; r += in.ncta)
      block_dots(in.U, in.n, in.n, (long long)r * RB, in.rb0 + r, in.V + (long long)in.j * in.ldv, in.nu,
                 b.part2, nullptr, red, redn);
    if (!group_barrier(bar, nct, b.err)) return;
    reduce_coeffs(b.part2 + (long long)in.rb0 * KMAXS, in.nrb, in.nu, ucs);
    __syncthreads();
    for (int r = rank; r < in.nrb; r += in.ncta) {
      const long long i = (long long)r * RB + tid;
      if (i < in.n) {
        cplx a = in.w[i];
        for (int t = 0; t < in.nu; t++) a = cadd(a, cmul(in.U[i + (long long)t * in.n], ucs[t]));
        in.w[i] = a;
      }
    }
    // pass 1 reads w only in the rows this thread has just written
  }

  // ---- pass 1: w' = w - beta_{j-1} v_{j-1}; partial h = V^H w', |w'|^2 ----
  {
    const double bp = in.j > 0 ? in.sc->beta[in.j - 1] : 0.0;
    const cplx* vp = in.V + (long long)(in.j > 0 ? in.j - 1 : 0) * in.ldv;
    for (int r = rank; r < in.nrb; r += in.ncta) {
      const long long r0 = (long long)r * RB;
      if (in.j > 0) {
        const long long i = r0 + tid;
        if (i < in.n) in.w[i] = csub(in.w[i], cscale(__ldcg(&vp[i]), bp));
      }
      block_dots(in.V, in.ldv, in.n, r0, in.rb0 + r, in.w, in.k, b.part, b.pn1, red, redn);
    }
  }
  if (!group_barrier(bar, nct, b.err)) return;

  // ---- every CTA of the instance: h, |w'|^2 and the DGKS test (after the
  // first pass |w''|^2 = |w'|^2 - |h|^2, the basis being orthonormal; a second
  // pass when that drops below half of |w'|^2, else beta_j = |w''| at once) ----
  reduce_coeffs(b.part + (long long)in.rb0 * KMAXS, in.nrb, in.k, hs);
  const double nw = sum_norms(in, b.pn1, redn);  // its barriers also publish hs
  const double b2 = nw - coeff_norm(hs, in.k, redn);
  const bool flag = b2 < DGKS2 * nw;
  double beta = sqrt(fmax(b2, 0.0));
  double alpha = in.sigma + hs[in.j].x;

  if (!flag) {
    // w'' / beta_j straight into the basis
    const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
    for (int r = rank; r < in.nrb; r += in.ncta) block_update_final(in, r, hs, in.k, inv);
  } else {
    // keep w'' in w and take its second-pass dots
    for (int r = rank; r < in.nrb; r += in.ncta) {
      block_update(in, r, in.w, hs, in.k, b.pn2, redn);
      block_dots(in.V, in.ldv, in.n, (long long)r * RB, in.rb0 + r, in.w, in.k, b.part2, nullptr, red, redn);
    }
    if (!group_barrier(bar, nct, b.err)) return;
    reduce_coeffs(b.part2 + (long long)in.rb0 * KMAXS, in.nrb, in.k, hs2);
    __syncthreads();
    alpha += hs2[in.j].x;
    // pn1 is free again: every CTA of the instance read it before the barrier
    for (int r = rank; r < in.nrb; r += in.ncta) block_update(in, r, in.w, hs2, in.k, b.pn1, redn);
    // the norm after the second pass is summed explicitly (no cancellation
    // argument holds for it)
    if (!group_barrier(bar, nct, b.err)) return;
    beta = sqrt(sum_norms(in, b.pn1, redn));
    if (in.write_next) {
      const double inv = beta > 0.0 ? 1.0 / beta : 0.0;
      cplx* vn = in.V + (long long)(in.j + 1) * in.ldv;
      for (int r = rank; r < in.nrb; r += in.ncta) {
        const long long i = (long long)r * RB + tid;
        if (i < in.n) vn[i] = cscale(in.w[i], inv);
      }
    }
  }

  // ---- alpha_j, beta_j ----
  if (rank == 0 && tid == 0) {
    in.sc->alpha[in.j] = alpha;
    in.sc->beta[in.j] = beta;
    in.sc->flag = flag ? 1 : 0;
    if (in.mirror) {  // mapped host memory, read by the host after the launch's event
      in.mirror->alpha[in.j] = alpha;
      in.mirror->beta[in.j] = beta;
    }
  }
}

std::atomic<unsigned long long> g_lz_setup{0};
int g_lz_grid[64] = {0};

}  // namespace

int lanczos_step_rows_per_block() { return RB; }

void lanczos_step(const Stream& st, LzBatch& b) {
  MPSGPU_CHECK(b.ninst >= 1 && b.ninst <= LZ_MAXI, MPSGPU_BAD_SHAPE, "lanczos step: group size");
  int rb = 0;
  double wsum = 0.0;
  for (int q = 0; q < b.ninst; q++) {
    LzInst& in = b.in[q];
    MPSGPU_CHECK(in.k == in.j + 1 && in.k <= KMAXS && in.n > 0, MPSGPU_BAD_SHAPE, "lanczos step: basis size");
    MPSGPU_CHECK(in.nu <= LZ_MAXU && in.nu <= KMAXS, MPSGPU_BAD_SHAPE, "lanczos step: projector size");
    in.rb0 = rb;
    in.nrb = ceil_div(in.n, RB);
    rb += in.nrb;
    wsum += (double)in.nrb * (2.0 * in.k + 6.0 + 2.0 * in.nu);
  }
  b.nrb_total = rb;
  int dev = 0;
  MPSGPU_CUDA(cudaGetDevice(&dev));
  if (device_needs_setup(g_lz_setup)) {
    int nsm = 148, per = 1;
    MPSGPU_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    MPSGPU_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, lanczos_step_kernel, T, 0));
    MPSGPU_CHECK(per >= 1, MPSGPU_BAD_SHAPE, "lanczos step: kernel does not fit on an SM");
    // at most two CTAs per SM: a group of several instances has row blocks
    // enough for both, and room stays for the kernels of other streams
    g_lz_grid[dev] = nsm * std::min(per, 2);
    mark_device_done(g_lz_setup);
  }
  const int G = g_lz_grid[dev];
  // CTAs per instance in proportion to its bytes, at most one per row block,
  // then evened out so that every CTA of an instance takes the same number
  // of row blocks; all of them co-resident (cooperative launch)
  std::vector<int> nc(b.ninst);
  int total = 0;
  for (int q = 0; q < b.ninst; q++) {
    const LzInst& in = b.in[q];
    const double w = (double)in.nrb * (2.0 * in.k + 6.0 + 2.0 * in.nu);
    int c = std::max(1, std::min(in.nrb, (int)(G * w / wsum)));
    c = ceil_div(in.nrb, ceil_div(in.nrb, c));
    nc[q] = c;
    total += c;
  }
  while (total > G) {  // only when many instances took their minimum of one
    int big = 0;
    for (int q = 1; q < b.ninst; q++)
      if (nc[q] > nc[big]) big = q;
    MPSGPU_CHECK(nc[big] > 1, MPSGPU_BAD_SHAPE, "lanczos step: more instances than co-resident CTAs");
    nc[big]--;
    total--;
  }
  int c0 = 0;
  for (int q = 0; q < b.ninst; q++) {
    b.in[q].cta0 = c0;
    b.in[q].ncta = nc[q];
    c0 += nc[q];
  }
  // algorithmic bytes: the basis read twice (projections, update), w read
  // and written three times (three-term step, update, normalisation) and
  // v_{j-1} once; the projector vectors twice
  double bytes = 0.0;
  for (int q = 0; q < b.ninst; q++)
    bytes += 16.0 * (double)b.in[q].n * (2.0 * b.in[q].k + 6.0 + 2.0 * b.in[q].nu);
  ProfScope ps(st, GemmProfiler::LZSTEP, bytes);
  void* args[] = {&b};
  MPSGPU_CUDA(cudaLaunchCooperativeKernel((void*)lanczos_step_kernel, dim3(c0), dim3(T), args, 0, st.s));
  after_launch(st);
}

}  // namespace mpsgpu
