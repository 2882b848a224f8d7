// Grouped effective-Hamiltonian matvec: y_i = L_i . W_i . R_i . x_i for many
// independent instances of different shapes (bond dimensions, MPO bonds) in
// three launches -- grouped GEMM (L.x), grouped MPO-leg contraction, grouped
// GEMM (.R) -- each a persistent grid over the flattened tiles or pixels of
// all instances.  The three launches can be captured once in a CUDA graph and
// replayed.  Instances are scheduled largest first so that the tail of each
// launch is filled by small tiles.
#include <algorithm>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

namespace {

// Wm[(s' + du*c) + (du*wr)*(b + wl*s)] = W[s' + du*(b + wl*(s + dd*c))] for every instance
struct WPerm {
  const cplx* W;
  cplx* Wm;
  int du, wl, dd, wr;
  long long begin;
};

__global__ void wperm_kernel(const WPerm* __restrict__ d, int n, long long total) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (d[mid].begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const WPerm& p = d[lo];
    long long e = t - p.begin;
    const int sp = (int)(e % p.du); e /= p.du;
    const int b = (int)(e % p.wl); e /= p.wl;
    const int s = (int)(e % p.dd); e /= p.dd;
    const int c = (int)e;
    p.Wm[(sp + p.du * c) + (long long)(p.du * p.wr) * (b + p.wl * s)] = p.W[t - p.begin];
  }
}

// One block per chunk of PX * WC_THREADS pixels of one problem (problems start
// on multiples of WC_CHUNK, itself a multiple of every chunk): the problem's
// leg matrix is staged in shared memory, and every thread takes PX pixels
// WC_THREADS apart (coalesced loads for every pixel index).
template <int NIN, int PX>
__global__ void __launch_bounds__(WC_THREADS) wcontract_grouped_kernel(const WGroup* __restrict__ g, int n,
                                                                       long long chunks) {
  __shared__ cplx Ws[32 * 32];
  for (long long ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
    const long long t0 = ch * (PX * WC_THREADS);
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (g[mid].pix_begin <= t0) lo = mid;
      else hi = mid - 1;
    }
    const WContractArgs& a = g[lo].a;
    const int parts = g[lo].parts;
    const long long pstride = g[lo].part_stride;
    const int nin = a.n_i0 * a.n_i1, nout = a.n_o0 * a.n_o1;
    const long long npix = (long long)a.nx * a.ny;
    __syncthreads();  // the previous chunk's reads of Ws are done
    for (int e = threadIdx.x; e < nin * nout; e += WC_THREADS) Ws[e] = a.Wm[e];
    __syncthreads();
    cplx in[PX][NIN];
    bool live[PX];
#pragma unroll
    for (int px = 0; px < PX; px++) {
      const long long p = t0 - g[lo].pix_begin + threadIdx.x + (long long)px * WC_THREADS;
      live[px] = p < npix;
      const int x = live[px] ? (int)(p % a.nx) : 0, y = live[px] ? (int)(p / a.nx) : 0;
      const cplx* ib = a.in + x * a.ix + y * a.iy;
#pragma unroll
      for (int i = 0; i < NIN; i++) {
        cplx v = make_double2(0.0, 0.0);
        if (i < nin && live[px]) {
          const long long off = (i % a.n_i0) * a.si0 + (i / a.n_i0) * a.si1;
          v = ib[off];
          for (int q = 1; q < parts; q++) v = cadd(v, ib[off + q * pstride]);
        }
        in[px][i] = v;
      }
    }
    for (int o = 0; o < nout; o++) {
      cplx acc[PX];
#pragma unroll
      for (int px = 0; px < PX; px++) acc[px] = make_double2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < NIN; i++) {
        if (i < nin) {
          const cplx w = Ws[o + nout * i];
#pragma unroll
          for (int px = 0; px < PX; px++) acc[px] = cadd(acc[px], cmul(w, in[px][i]));
        }
      }
#pragma unroll
      for (int px = 0; px < PX; px++) {
        if (!live[px]) continue;
        const long long p = t0 - g[lo].pix_begin + threadIdx.x + (long long)px * WC_THREADS;
        const int x = (int)(p % a.nx), y = (int)(p / a.nx);
        a.out[x * a.ox + y * a.oy + (o % a.n_o0) * a.so0 + (o / a.n_o0) * a.so1] = acc[px];
      }
    }
  }
}

}  // namespace

long long wcontract_chunked(long long pixels) { return (pixels + WC_CHUNK - 1) / WC_CHUNK * WC_CHUNK; }

void wcontract_grouped(const Stream& st, const WGroup* d_wg, int n, long long pixels, int maxnin, int maxnout) {
  MPSGPU_CHECK(maxnin >= 1 && maxnin <= 32 && maxnout >= 1 && maxnin * maxnout <= 32 * 32, MPSGPU_BAD_SHAPE,
               "wcontract_grouped: MPO legs too wide");
  if (pixels <= 0) return;
  auto launch = [&](auto kernel, int px) {
    const long long chunks = (pixels + px * WC_THREADS - 1) / (px * WC_THREADS);
    const int g = (int)std::min<long long>(chunks, 148LL * 16);
    kernel<<<g, WC_THREADS, 0, st.s>>>(d_wg, n, chunks);
  };
  // one pixel per thread: enough blocks to fill the SMs several times over at
  // the sweep shapes (two or four pixels per thread halved the blocks and
  // measured slower)
  if (maxnin <= 8) launch(wcontract_grouped_kernel<8, 1>, 1);
  else if (maxnin <= 16) launch(wcontract_grouped_kernel<16, 1>, 1);
  else launch(wcontract_grouped_kernel<32, 1>, 1);
  after_launch(st);
}

GroupedMatvecPlan::~GroupedMatvecPlan() {}

void grouped_matvec_plan(const Stream& st, const std::vector<HeffInstance>& inst, GroupedMatvecPlan& plan,
                         int nsm, bool split) {
  const int n = (int)inst.size();
  MPSGPU_CHECK(n > 0, MPSGPU_INVALID, "grouped matvec: no instances");
  // largest first
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  auto work = [&](int i) { return (double)inst[i].Dl * inst[i].Dr * (inst[i].Dl + inst[i].Dr) * inst[i].wl; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  long long t1_total = 0, wm_total = 0, pix_total = 0, wel_total = 0;
  for (const auto& h : inst) {
    MPSGPU_CHECK(h.d > 0 && h.wl > 0 && h.wr > 0 && h.Dl > 0 && h.Dr > 0 && h.d * h.wl <= 32 && h.d * h.wr <= 32,
                 MPSGPU_BAD_SHAPE, "grouped matvec: bad instance shape");
    t1_total += (long long)h.Dl * h.wl * h.d * h.Dr;
    wm_total += (long long)h.d * h.wl * h.d * h.wr;
    pix_total += (long long)h.Dl * h.Dr;
  }
  wel_total = wm_total;
  plan.n = n;
  dbuf_alloc(st, plan.t1, t1_total);
  dbuf_alloc(st, plan.t2, t1_total);
  dbuf_alloc(st, plan.wm, wm_total);
  std::vector<GroupedGemm> g1(n), g3(n);
  std::vector<WGroup> wg(n);
  std::vector<WPerm> wp(n);
  // split form: byte offsets of every prepared operand in one buffer
  std::vector<SplitProblem> s1(split ? n : 0), s3(split ? n : 0);
  std::vector<SplitPrepJob> jenv(split ? 2 * n : 0), jx(split ? n : 0), jt(split ? n : 0);
  std::vector<long long> offL(n), offX(n), offT(n), offR(n);
  long long spb = 0;
  auto take = [&](long long bytes) {
    const long long o = spb;
    spb += (bytes + 255) / 256 * 256;
    return o;
  };
  long long o1 = 0, ow = 0, pix = 0;
  int maxnin = 1, maxnout = 1;
  for (int q = 0; q < n; q++) {
    const int i = order[q];
    const HeffInstance& h = inst[i];
    const int d = h.d, wl = h.wl, wr = h.wr, Dl = h.Dl, Dr = h.Dr;
    cplx* T1 = plan.t1.p + o1;
    cplx* T2 = plan.t2.p + o1;
    cplx* Wm = plan.wm.p + ow;
    wp[q] = WPerm{h.W, Wm, d, wl, d, wr, ow};
    GroupedGemm& a = g1[q];
    a.M = Dl * wl; a.N = d * Dr; a.K = Dl;
    a.A = h.L; a.lda = (long long)Dl * wl;
    a.B = h.x; a.ldb = Dl;
    a.C = T1; a.ldc = (long long)Dl * wl;
    WContractArgs& w = wg[q].a;
    w.nx = Dl; w.ny = Dr;
    w.in = T1; w.ix = 1; w.iy = (long long)Dl * wl * d; w.si0 = Dl; w.si1 = (long long)Dl * wl;
    w.n_i0 = wl; w.n_i1 = d;
    w.out = T2; w.ox = 1; w.oy = (long long)Dl * d; w.so0 = Dl; w.so1 = (long long)Dl * d * Dr;
    w.n_o0 = d; w.n_o1 = wr;
    w.Wm = Wm;
    wg[q].pix_begin = pix;
    GroupedGemm& b = g3[q];
    b.M = Dl * d; b.N = Dr; b.K = Dr * wr;
    b.A = T2; b.lda = (long long)Dl * d;
    b.B = h.Rt; b.ldb = (long long)Dr * wr;
    b.C = h.y; b.ldc = (long long)Dl * d;
    o1 += (long long)Dl * wl * d * Dr;
    ow += (long long)d * wl * d * wr;
    pix += wcontract_chunked((long long)Dl * Dr);
    maxnin = std::max(maxnin, wl * d);
    maxnout = std::max(maxnout, d * wr);
    if (split) {
      offL[q] = take(split_operand_bytes(Dl * wl, Dl, 128));
      offX[q] = take(split_operand_bytes(d * Dr, Dl, 128));
      offT[q] = take(split_operand_bytes(Dl * d, Dr * wr, 128));
      offR[q] = take(split_operand_bytes(Dr, Dr * wr, 128));
      // L as A (rows Dl*wl), x as B (rows = columns of T1), T2 as A, Rt as B
      jenv[2 * q] = SplitPrepJob{Dl * wl, Dl, 0, h.L, 1, (long long)Dl * wl, nullptr, 0};
      jenv[2 * q + 1] = SplitPrepJob{Dr, Dr * wr, 0, h.Rt, (long long)Dr * wr, 1, nullptr, 0};
      jx[q] = SplitPrepJob{d * Dr, Dl, 0, h.x, Dl, 1, nullptr, 0};
      jt[q] = SplitPrepJob{Dl * d, Dr * wr, 0, T2, 1, (long long)Dl * d, nullptr, 0};
      s1[q].M = Dl * wl; s1[q].N = d * Dr; s1[q].K = Dl;
      s1[q].C = T1; s1[q].ldc = (long long)Dl * wl;
      s3[q].M = Dl * d; s3[q].N = Dr; s3[q].K = Dr * wr;
      s3[q].C = h.y; s3[q].ldc = (long long)Dl * d;
    }
    plan.flops += 8.0 * ((double)Dl * wl * Dl * d * Dr + (double)Dl * d * d * wl * wr * Dr +
                         (double)Dl * d * Dr * wr * Dr);
  }
  plan.tiles1 = grouped_tiles(g1.data(), n);
  plan.tiles3 = grouped_tiles(g3.data(), n);
  plan.pixels = pix;
  plan.wel = wel_total;
  plan.maxnin = maxnin;
  plan.maxnout = maxnout;
  // descriptor tables in device memory
  const size_t bytes = n * (2 * sizeof(GroupedGemm) + sizeof(WGroup) + sizeof(WPerm));
  MPSGPU_CUDA(cudaMallocAsync(&plan.desc, bytes, st.s));
  char* p = (char*)plan.desc;
  plan.d_g1 = (GroupedGemm*)p; p += n * sizeof(GroupedGemm);
  plan.d_g3 = (GroupedGemm*)p; p += n * sizeof(GroupedGemm);
  plan.d_wg = p; p += n * sizeof(WGroup);
  plan.d_wp = p;
  MPSGPU_CUDA(cudaMemcpyAsync(plan.d_g1, g1.data(), n * sizeof(GroupedGemm), cudaMemcpyHostToDevice, st.s));
  MPSGPU_CUDA(cudaMemcpyAsync(plan.d_g3, g3.data(), n * sizeof(GroupedGemm), cudaMemcpyHostToDevice, st.s));
  MPSGPU_CUDA(cudaMemcpyAsync(plan.d_wg, wg.data(), n * sizeof(WGroup), cudaMemcpyHostToDevice, st.s));
  MPSGPU_CUDA(cudaMemcpyAsync(plan.d_wp, wp.data(), n * sizeof(WPerm), cudaMemcpyHostToDevice, st.s));
  MPSGPU_CUDA(cudaStreamSynchronize(st.s));
  plan.ctas = nsm;
  plan.split = split;
  if (split) {
    dbuf_alloc(st, plan.sp, (spb + (long long)sizeof(cplx) - 1) / (long long)sizeof(cplx));
    uint8_t* base = reinterpret_cast<uint8_t*>(plan.sp.p);
    for (int q = 0; q < n; q++) {
      jenv[2 * q].out = base + offL[q];
      jenv[2 * q + 1].out = base + offR[q];
      jx[q].out = base + offX[q];
      jt[q].out = base + offT[q];
      s1[q].Ap = base + offL[q]; s1[q].Bp = base + offX[q];
      s3[q].Ap = base + offT[q]; s3[q].Bp = base + offR[q];
    }
    plan.stiles1 = split_group_tiles(s1.data(), n);
    plan.stiles3 = split_group_tiles(s3.data(), n);
    plan.thr_env = split_prepare_jobs(jenv.data(), 2 * n);
    plan.thr_x = split_prepare_jobs(jx.data(), n);
    plan.thr_t = split_prepare_jobs(jt.data(), n);
    const size_t sbytes = 2 * n * sizeof(SplitProblem) + 4 * n * sizeof(SplitPrepJob) + 256;
    MPSGPU_CUDA(cudaMallocAsync(&plan.sdesc, sbytes, st.s));
    char* sq = (char*)plan.sdesc;
    plan.d_s1 = (SplitProblem*)sq; sq += n * sizeof(SplitProblem);
    plan.d_s3 = (SplitProblem*)sq; sq += n * sizeof(SplitProblem);
    plan.d_jenv = (SplitPrepJob*)sq; sq += 2 * n * sizeof(SplitPrepJob);
    plan.d_jx = (SplitPrepJob*)sq; sq += n * sizeof(SplitPrepJob);
    plan.d_jt = (SplitPrepJob*)sq; sq += n * sizeof(SplitPrepJob);
    plan.err = (int*)sq;
    MPSGPU_CUDA(cudaMemcpyAsync(plan.d_s1, s1.data(), n * sizeof(SplitProblem), cudaMemcpyHostToDevice, st.s));
    MPSGPU_CUDA(cudaMemcpyAsync(plan.d_s3, s3.data(), n * sizeof(SplitProblem), cudaMemcpyHostToDevice, st.s));
    MPSGPU_CUDA(cudaMemcpyAsync(plan.d_jenv, jenv.data(), 2 * n * sizeof(SplitPrepJob), cudaMemcpyHostToDevice, st.s));
    MPSGPU_CUDA(cudaMemcpyAsync(plan.d_jx, jx.data(), n * sizeof(SplitPrepJob), cudaMemcpyHostToDevice, st.s));
    MPSGPU_CUDA(cudaMemcpyAsync(plan.d_jt, jt.data(), n * sizeof(SplitPrepJob), cudaMemcpyHostToDevice, st.s));
    MPSGPU_CUDA(cudaMemsetAsync(plan.err, 0, sizeof(int), st.s));
    MPSGPU_CUDA(cudaStreamSynchronize(st.s));
  }
}

void grouped_matvec_prepare_env(const Stream& st, GroupedMatvecPlan& plan) {
  MPSGPU_CHECK(plan.split, MPSGPU_INVALID, "grouped matvec: not planned in split precision");
  split_prepare_grouped(st, plan.d_jenv, 2 * plan.n, plan.thr_env);
}

void grouped_matvec_run(const Stream& st, GroupedMatvecPlan& plan) {
  // W leg matrices (cheap; part of every product so inputs stay the raw W)
  wperm_kernel<<<std::min<long long>(ceil_div(plan.wel, 256), 4096), 256, 0, st.s>>>(
      (const WPerm*)plan.d_wp, plan.n, plan.wel);
  after_launch(st);
  if (plan.split) {
    split_prepare_grouped(st, plan.d_jx, plan.n, plan.thr_x);
    zgemm_split_grouped(st, plan.d_s1, plan.n, plan.stiles1, plan.err);
  } else {
    zgemm_grouped(st, plan.d_g1, plan.n, plan.tiles1, plan.ctas);
  }
  wcontract_grouped(st, (const WGroup*)plan.d_wg, plan.n, plan.pixels, plan.maxnin, plan.maxnout);
  if (plan.split) {
    split_prepare_grouped(st, plan.d_jt, plan.n, plan.thr_t);
    zgemm_split_grouped(st, plan.d_s3, plan.n, plan.stiles3, plan.err);
  } else {
    zgemm_grouped(st, plan.d_g3, plan.n, plan.tiles3, plan.ctas);
  }
}

void grouped_matvec_free(const Stream& st, GroupedMatvecPlan& plan) {
  if (plan.desc) cudaFreeAsync(plan.desc, st.s);
  plan.desc = nullptr;
  if (plan.sdesc) cudaFreeAsync(plan.sdesc, st.s);
  plan.sdesc = nullptr;
  for (DevMem* b : {&plan.t1, &plan.t2, &plan.wm, &plan.sp})
    if (b->p) {
      cudaFreeAsync(b->p, st.s);
      b->p = nullptr;
    }
}

}  // namespace mpsgpu
