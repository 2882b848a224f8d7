// Split-precision complex GEMM on the fifth-generation tensor cores
// (tcgen05.mma, kind::f16 with BF16 operands, FP32 accumulators in TMEM).
//
// Every FP64 real number x is written as three BF16 limbs
//   x = h + m + l,  h = bf16(x), m = bf16(x - h), l = bf16(x - h - m)
// (24 significant bits in all), and a complex product C = A B is the sum of
// the limb products with i + j <= 2 (the dropped terms are below 2^-24 of
// |A||B|):
//   Re C = sum Re A_i Re B_j - Im A_i Im B_j,   Im C = sum Re A_i Im B_j + Im A_i Re B_j
// i.e. 24 BF16 MMAs per k-step of 16, accumulated in two TMEM accumulators
// (the minus sign is the instruction descriptor's negate-A bit).  The result
// carries FP32-class accuracy (relative error about 1e-7 of |A||B| per
// entry), which is what the split-precision sweep mode uses for its early
// half-sweeps; the FP64 path (zgemm.cu) finishes the solve.
//
// Data path.  split_prepare converts one operand into six BF16 planes (re
// h/m/l, im h/m/l) already tiled in the canonical K-major, no-swizzle UMMA
// layout: for a tile of R rows and one k-step of 16, a plane is two 8-column
// halves (R * 16 bytes apart, the descriptor's leading byte offset), each a
// stack of 8-row x 16-byte core matrices (128 bytes apart, the stride byte
// offset).  The six planes of one (row tile, k-step) are contiguous, so one
// pipeline stage of the GEMM is two contiguous bulk copies (cp.async.bulk,
// untiled, completion counted on an mbarrier), issued with the MMAs by a
// single thread over a four-stage ring.  The epilogue reads TMEM with
// tcgen05.ld (warp w owns lanes 32w..32w+31 = rows of the tile) and writes
// FP64 C = alpha (Cr + i Ci) + beta Cin, or FP64 partial products when K is
// split over CTAs (reduced by split_reduce_kernel).
//
// Every mbarrier wait is bounded (2 s of %globaltimer); a wait that runs out
// sets the error flag, the issuing thread waits (bounded) for its own bulk
// copies still in flight, the TMEM columns are released and the kernel
// returns; the host turns the flag into MPSGPU_TIMEOUT.
#include <cuda_bf16.h>

#include "kernels.h"

namespace mpsgpu {
namespace {

constexpr int SP_BM = 128;       // rows of an A tile = TMEM lanes of the accumulator
constexpr int SP_BK = 16;        // K of one BF16 MMA = one pipeline stage
constexpr int SP_PLANES = 6;     // re h/m/l, im h/m/l
constexpr int SP_STAGES = 4;      // ring depth of the 64- and 128-column tiles
// stages of the ring for a column tile: 128 x 256 tiles (72 KB a stage) fit three
__host__ __device__ constexpr int sp_stages(int bn) { return bn == 256 ? 3 : SP_STAGES; }
constexpr int SP_THREADS = 128;
constexpr int SP_GROUP_BN = 128;  // column tile of grouped launches
constexpr unsigned long long SP_WAIT_NS = 2000000000ULL;

__host__ __device__ constexpr int sp_plane_bytes(int rows) { return rows * SP_BK * 2; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete; false after SP_WAIT_NS.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try(bar, parity)) {
    if (global_ns() - t0 > SP_WAIT_NS) return false;
  }
  return true;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Untiled bulk copy global -> shared, completion counted in bytes on `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n; negate_a flips the sign of A.
__host__ __device__ constexpr uint32_t mma_idesc(int n, bool negate_a) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (negate_a ? (1u << 13) : 0u) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(SP_BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

// Arrives on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- operand preparation ---------------------------------------------------

__device__ __forceinline__ void split3(double x, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __double2bfloat16(x);
  const double r1 = x - (double)__bfloat162float(h);
  m = __double2bfloat16(r1);
  const double r2 = r1 - (double)__bfloat162float(m);
  l = __double2bfloat16(r2);
}

// One thread per (row, 8 consecutive k): reads 8 complex entries
// X[row * rs + k * ks] (zero outside rows x K) and writes 16 bytes to each
// of the six planes of its (row tile, k-step).
__global__ void split_prepare_kernel(int rows, int K, int KS, int RT, const cplx* __restrict__ X, long long rs,
                                     long long kst, uint8_t* __restrict__ out) {
  const long long total = (long long)((rows + RT - 1) / RT) * KS * 2 * RT;
  const int groups = RT / 8;
  const int plane = sp_plane_bytes(RT);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx & 7);
    long long q = idx >> 3;
    const int g = (int)(q % groups);
    q /= groups;
    const int kg = (int)(q & 1);
    q >>= 1;
    const int ks = (int)(q % KS);
    const long long rt = q / KS;
    const long long row = rt * RT + g * 8 + r;
    const int k0 = ks * SP_BK + kg * 8;
    union {
      __nv_bfloat16 h[8];
      uint4 u;
    } pk[SP_PLANES];
#pragma unroll
    for (int kk = 0; kk < 8; kk++) {
      const int k = k0 + kk;
      cplx x = cmake(0.0, 0.0);
      if (row < rows && k < K) x = X[row * rs + (long long)k * kst];
      split3(x.x, pk[0].h[kk], pk[1].h[kk], pk[2].h[kk]);
      split3(x.y, pk[3].h[kk], pk[4].h[kk], pk[5].h[kk]);
    }
    uint8_t* base = out + ((rt * KS + ks) * SP_PLANES) * plane + (long long)kg * (RT * 16) + g * 128 + r * 16;
#pragma unroll
    for (int p = 0; p < SP_PLANES; p++) *reinterpret_cast<uint4*>(base + (long long)p * plane) = pk[p].u;
  }
}

// ---- the GEMM ----------------------------------------------------------------

struct SplitGemmParams {
  int M, N, KS, ks_per_split;
  const uint8_t* Ap;  // prepared A, row tile 128
  const uint8_t* Bp;  // prepared B (rows = columns of C), row tile BN
  cplx* C;
  long long ldc;
  cplx alpha;
  const cplx* Cin;
  long long ldcin;
  cplx beta;
  cplx* part;  // split K: partial products, (split, n, m) with m fastest
  int* err;
};

// Grouped launches: one CTA per 128 x BN tile of any of n independent GEMMs
// C_q = A_q B_q (no split K; the tiles of many products fill the SMs).
struct SplitGroupParams {
  const SplitProblem* probs;  // tile_begin ascending
  int n;
  int* err;
};

template <int BN, bool GROUPED>
__global__ void __launch_bounds__(SP_THREADS, 1) zgemm_split_kernel(SplitGemmParams p, SplitGroupParams gp) {
  constexpr int A_STAGE = SP_PLANES * sp_plane_bytes(SP_BM);
  constexpr int B_STAGE = SP_PLANES * sp_plane_bytes(BN);
  constexpr int STAGE = A_STAGE + B_STAGE;
  constexpr int STAGES = sp_stages(BN);
  constexpr uint32_t TMEM_COLS = 2 * BN;  // Cr in [0, BN), Ci in [BN, 2 BN); 512 = all of TMEM at BN = 256
  extern __shared__ uint8_t smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[SP_STAGES];
  __shared__ __align__(8) uint64_t empty_bar[SP_STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int aborted;

  // 128-byte aligned ring of STAGES stages (the launch adds 128 bytes of slack)
  const uint32_t ring = (smem_u32(smem_dyn) + 127u) & ~127u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int mt, nt, sp, k0, nk;
  if constexpr (GROUPED) {
    // the problem whose tile range holds this CTA (last tile_begin <= blockIdx.x)
    const long long t = blockIdx.x;
    int lo = 0, hi = gp.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (gp.probs[mid].tile_begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const SplitProblem q = gp.probs[lo];
    const long long local = t - q.tile_begin;
    mt = (int)(local % q.mtiles);
    nt = (int)(local / q.mtiles);
    sp = 0;
    k0 = q.k0;
    nk = q.nk > 0 ? q.nk : q.KS - q.k0;
    p.M = q.M;
    p.N = q.N;
    p.KS = q.KS;
    p.Ap = q.Ap;
    p.Bp = q.Bp;
    p.C = q.C;
    p.ldc = q.ldc;
    p.alpha = cmake(1.0, 0.0);
    p.Cin = nullptr;
    p.part = nullptr;
    p.err = gp.err;
  } else {
    mt = blockIdx.x;
    nt = blockIdx.y;
    sp = blockIdx.z;
    k0 = sp * p.ks_per_split;
    nk = min(p.KS - k0, p.ks_per_split);
  }

  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    mbar_init(smem_u32(&done_bar), 1);
    aborted = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (tid == 0) {
    const uint8_t* a_src = p.Ap + ((size_t)mt * p.KS + k0) * A_STAGE;
    const uint8_t* b_src = p.Bp + ((size_t)nt * p.KS + k0) * B_STAGE;
    auto load = [&](int t) {
      const int buf = t % STAGES;
      const uint32_t bar = smem_u32(&full_bar[buf]);
      const uint32_t dst = ring + buf * STAGE;
      mbar_expect_tx(bar, STAGE);
      bulk_g2s(dst, a_src + (size_t)t * A_STAGE, A_STAGE, bar);
      bulk_g2s(dst + A_STAGE, b_src + (size_t)t * B_STAGE, B_STAGE, bar);
    };
    int loaded = min(STAGES, nk);
    for (int t = 0; t < loaded; t++) load(t);
    const uint32_t id_pos = mma_idesc(BN, false), id_neg = mma_idesc(BN, true);
    bool ok = true;
    int kt = 0;
    for (; kt < nk; ++kt) {
      const int buf = kt % STAGES;
      if (!mbar_wait(smem_u32(&full_bar[buf]), (kt / STAGES) & 1)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = ring + buf * STAGE, sb = sa + A_STAGE;
      const uint32_t first = (kt == 0) ? 0u : 1u;
#pragma unroll
      for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j + i < 3; j++) {
          const uint64_t are = smem_desc(sa + i * sp_plane_bytes(SP_BM), SP_BM * 16, 128);
          const uint64_t aim = smem_desc(sa + (3 + i) * sp_plane_bytes(SP_BM), SP_BM * 16, 128);
          const uint64_t bre = smem_desc(sb + j * sp_plane_bytes(BN), BN * 16, 128);
          const uint64_t bim = smem_desc(sb + (3 + j) * sp_plane_bytes(BN), BN * 16, 128);
          const uint32_t acc = (i == 0 && j == 0) ? first : 1u;
          mma_bf16(tmem, are, bre, id_pos, acc);
          mma_bf16(tmem, aim, bim, id_neg, 1u);
          mma_bf16(tmem + BN, are, bim, id_pos, acc);
          mma_bf16(tmem + BN, aim, bre, id_pos, 1u);
        }
      }
      mma_commit(smem_u32(&empty_bar[buf]));
      // refill the stage the previous k-step used once its MMAs are done,
      // keeping this step's MMAs queued behind them
      if (kt >= 1 && kt - 1 + STAGES < nk) {
        const int j = kt - 1;
        if (!mbar_wait(smem_u32(&empty_bar[j % STAGES]), (j / STAGES) & 1)) {
          ok = false;
          ++kt;
          break;
        }
        load(j + STAGES);
        loaded = j + STAGES + 1;
      }
    }
    if (!ok) {
      *(volatile int*)p.err = 1;
      aborted = 1;
      for (int t = kt; t < loaded; t++) mbar_wait(smem_u32(&full_bar[t % STAGES]), (t / STAGES) & 1);
    }
    mma_commit(smem_u32(&done_bar));
  }
  __syncthreads();
  const bool done = mbar_wait(smem_u32(&done_bar), 0);
  if (!done && lane == 0) *(volatile int*)p.err = 1;
  tc_fence_after();
  if (!aborted && __all_sync(0xffffffffu, done)) {
    const int row = mt * SP_BM + warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    const bool direct = (p.part == nullptr);
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      __syncwarp();
      uint32_t vr[32], vi[32];
      tmem_ld32(tl + c, vr);
      tmem_ld32(tl + BN + c, vi);
      tmem_wait_ld();
      if (row < p.M) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int n = nt * BN + c + j;
          if (n < p.N) {
            const cplx v = cmake((double)__uint_as_float(vr[j]), (double)__uint_as_float(vi[j]));
            if (direct) {
              cplx o = cmul(p.alpha, v);
              if (p.Cin) o = cadd(o, cmul(p.beta, p.Cin[row + (long long)n * p.ldcin]));
              p.C[row + (long long)n * p.ldc] = o;
            } else {
              p.part[((long long)sp * p.N + n) * p.M + row] = v;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

__global__ void split_reduce_kernel(int M, int N, int splits, const cplx* __restrict__ part, cplx* C, long long ldc,
                                    cplx alpha, const cplx* Cin, long long ldcin, cplx beta) {
  const long long total = (long long)M * N;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(idx % M);
    const long long n = idx / M;
    cplx s = cmake(0.0, 0.0);
    for (int t = 0; t < splits; t++) s = cadd(s, part[(long long)t * total + idx]);
    cplx o = cmul(alpha, s);
    if (Cin) o = cadd(o, cmul(beta, Cin[m + n * ldcin]));
    C[m + n * ldc] = o;
  }
}

// Grouped sums of partial products (split_reduce_grouped): element t of
// job j (t in [begin_j, begin_{j+1})) is C[m + n ldc] = alpha sum_s part[s M N
// + m + n M] + beta Cin[m + n ldcin], the partials added in order.
__global__ void split_reduce_grouped_kernel(const SplitReduceJob* __restrict__ jobs, int n, long long total) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const SplitReduceJob& jb = jobs[lo];
    const long long e = t - jb.begin, mn = (long long)jb.M * jb.N;
    const int m = (int)(e % jb.M);
    const long long col = e / jb.M;
    cplx s = cmake(0.0, 0.0);
    for (int p = 0; p < jb.nparts; p++) s = cadd(s, jb.part[p * mn + e]);
    cplx o = cmul(jb.alpha, s);
    if (jb.Cin) o = cadd(o, cmul(jb.beta, jb.Cin[m + col * jb.ldcin]));
    jb.C[m + col * jb.ldc] = o;
  }
}

template <int BN>
constexpr int split_smem_bytes() {
  return sp_stages(BN) * (SP_PLANES * sp_plane_bytes(SP_BM) + SP_PLANES * sp_plane_bytes(BN)) + 128;
}

template <int BN, bool GROUPED>
void launch_split(const Stream& st, const SplitGemmParams& p, const SplitGroupParams& gp, dim3 grid) {
  constexpr int smem = split_smem_bytes<BN>();
  static std::atomic<unsigned long long> attr{0};
  if (device_needs_setup(attr)) {
    MPSGPU_CUDA(cudaFuncSetAttribute(zgemm_split_kernel<BN, GROUPED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     smem));
    mark_device_done(attr);
  }
  zgemm_split_kernel<BN, GROUPED><<<grid, SP_THREADS, smem, st.s>>>(p, gp);
  after_launch(st);
}

// Grouped operand preparation: job j covers threads [thread_begin, next);
// every operand is tiled with 128-row tiles.
__global__ void split_prepare_grouped_kernel(const SplitPrepJob* __restrict__ jobs, int n, long long total) {
  constexpr int RT = SP_BM;
  constexpr int groups = RT / 8;
  constexpr int plane = sp_plane_bytes(RT);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].thread_begin <= idx) lo = mid;
      else hi = mid - 1;
    }
    const SplitPrepJob& jb = jobs[lo];
    const long long li = idx - jb.thread_begin;
    const int r = (int)(li & 7);
    long long q = li >> 3;
    const int g = (int)(q % groups);
    q /= groups;
    const int kg = (int)(q & 1);
    q >>= 1;
    const int ks = (int)(q % jb.KS);
    const long long rt = q / jb.KS;
    const long long row = rt * RT + g * 8 + r;
    const int k0 = ks * SP_BK + kg * 8;
    union {
      __nv_bfloat16 h[8];
      uint4 u;
    } pk[SP_PLANES];
#pragma unroll
    for (int kk = 0; kk < 8; kk++) {
      const int k = k0 + kk;
      cplx x = cmake(0.0, 0.0);
      if (row < jb.rows && k < jb.K) x = jb.X[row * jb.rs + (long long)k * jb.ks];
      split3(x.x, pk[0].h[kk], pk[1].h[kk], pk[2].h[kk]);
      split3(x.y, pk[3].h[kk], pk[4].h[kk], pk[5].h[kk]);
    }
    uint8_t* base = jb.out + ((rt * jb.KS + ks) * SP_PLANES) * plane + (long long)kg * (RT * 16) + g * 128 + r * 16;
#pragma unroll
    for (int p = 0; p < SP_PLANES; p++) *reinterpret_cast<uint4*>(base + (long long)p * plane) = pk[p].u;
  }
}

}  // namespace

long long split_operand_bytes(int rows, int K, int RT) {
  const long long tiles = (rows + RT - 1) / RT, ks = (K + SP_BK - 1) / SP_BK;
  return tiles * ks * SP_PLANES * sp_plane_bytes(RT);
}

void split_prepare(const Stream& st, int rows, int K, const cplx* X, long long rs, long long ks, int RT,
                   uint8_t* out) {
  MPSGPU_CHECK(rows > 0 && K > 0 && (RT == 64 || RT == 128 || RT == 256), MPSGPU_INVALID,
               "split_prepare: bad shape");
  MPSGPU_CHECK(((uintptr_t)out & 15) == 0, MPSGPU_INVALID, "split_prepare: output not 16-byte aligned");
  const int KS = (K + SP_BK - 1) / SP_BK;
  const long long total = (long long)((rows + RT - 1) / RT) * KS * 2 * RT;
  const int threads = 256;
  const int blocks = (int)std::min<long long>((total + threads - 1) / threads, 148LL * 16);
  split_prepare_kernel<<<blocks, threads, 0, st.s>>>(rows, K, KS, RT, X, rs, ks, out);
  after_launch(st);
}

SplitPlan split_plan(int M, int N, int K, int nsm) {
  SplitPlan pl;
  pl.M = M;
  pl.N = N;
  pl.K = K;
  pl.KS = (K + SP_BK - 1) / SP_BK;
  pl.mtiles = (M + SP_BM - 1) / SP_BM;
  // 256-column tiles when they alone fill the SMs (half the A traffic and
  // tile overhead per flop), 128 unless that leaves most SMs idle, else 64
  if (pl.mtiles * ((N + 255) / 256) >= nsm) pl.BN = 256;
  else pl.BN = (pl.mtiles * ((N + 127) / 128) >= nsm / 2) ? 128 : 64;
  pl.ntiles = (N + pl.BN - 1) / pl.BN;
  const int tiles = pl.mtiles * pl.ntiles;
  // split K over CTAs while tiles do not fill the SMs, keeping >= 4 k-steps each
  int splits = std::max(1, std::min(nsm / std::max(tiles, 1), pl.KS / 4));
  pl.ks_per_split = (pl.KS + splits - 1) / splits;
  pl.splits = (pl.KS + pl.ks_per_split - 1) / pl.ks_per_split;
  return pl;
}

void zgemm_split_prepared(const Stream& st, const SplitPlan& pl, const uint8_t* Ap, const uint8_t* Bp, cplx* C,
                          long long ldc, cplx alpha, const cplx* Cin, long long ldcin, cplx beta, cplx* part,
                          int* err) {
  MPSGPU_CHECK(((uintptr_t)Ap & 15) == 0 && ((uintptr_t)Bp & 15) == 0, MPSGPU_INVALID,
               "zgemm_split: operands not 16-byte aligned");
  MPSGPU_CHECK(pl.splits == 1 || part != nullptr, MPSGPU_INVALID, "zgemm_split: split K needs a partial buffer");
  // 24 BF16 MMAs (M x N x 16) per complex k-step of 16: 48 M N K tensor flops
  ProfScope ps(st, GemmProfiler::SPLIT, 48.0 * (double)pl.M * pl.N * pl.K);
  SplitGemmParams p;
  p.M = pl.M;
  p.N = pl.N;
  p.KS = pl.KS;
  p.ks_per_split = pl.ks_per_split;
  p.Ap = Ap;
  p.Bp = Bp;
  p.C = C;
  p.ldc = ldc;
  p.alpha = alpha;
  p.Cin = Cin;
  p.ldcin = ldcin;
  p.beta = beta;
  p.part = pl.splits > 1 ? part : nullptr;
  p.err = err;
  const SplitGroupParams none{nullptr, 0, nullptr};
  const dim3 grid(pl.mtiles, pl.ntiles, pl.splits);
  if (pl.BN == 256)
    launch_split<256, false>(st, p, none, grid);
  else if (pl.BN == 128)
    launch_split<128, false>(st, p, none, grid);
  else
    launch_split<64, false>(st, p, none, grid);
  if (pl.splits > 1) {
    const long long total = (long long)pl.M * pl.N;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
    split_reduce_kernel<<<blocks, 256, 0, st.s>>>(pl.M, pl.N, pl.splits, part, C, ldc, alpha, Cin, ldcin, beta);
    after_launch(st);
  }
}

long long split_group_tiles(SplitProblem* probs, int n) {
  long long t = 0;
  for (int i = 0; i < n; i++) {
    SplitProblem& q = probs[i];
    q.KS = (q.K + SP_BK - 1) / SP_BK;
    q.mtiles = (q.M + SP_BM - 1) / SP_BM;
    q.tile_begin = t;
    t += (long long)q.mtiles * ((q.N + SP_GROUP_BN - 1) / SP_GROUP_BN);
  }
  return t;
}

void zgemm_split_grouped(const Stream& st, const SplitProblem* d_probs, int n, long long tiles, int* err) {
  MPSGPU_CHECK(tiles > 0 && tiles < (1LL << 31), MPSGPU_INVALID, "zgemm_split_grouped: tile count");
  SplitGemmParams p{};
  const SplitGroupParams gp{d_probs, n, err};
  launch_split<SP_GROUP_BN, true>(st, p, gp, dim3((unsigned)tiles));
}

long long split_reduce_jobs(SplitReduceJob* jobs, int n) {
  long long t = 0;
  for (int i = 0; i < n; i++) {
    jobs[i].begin = t;
    t += (long long)jobs[i].M * jobs[i].N;
  }
  return t;
}

void split_reduce_grouped(const Stream& st, const SplitReduceJob* d_jobs, int n, long long total) {
  if (total <= 0) return;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
  split_reduce_grouped_kernel<<<blocks, 256, 0, st.s>>>(d_jobs, n, total);
  after_launch(st);
}

long long split_prepare_jobs(SplitPrepJob* jobs, int n) {
  long long t = 0;
  for (int i = 0; i < n; i++) {
    SplitPrepJob& j = jobs[i];
    j.KS = (j.K + SP_BK - 1) / SP_BK;
    j.thread_begin = t;
    t += (long long)((j.rows + SP_BM - 1) / SP_BM) * ((j.K + SP_BK - 1) / SP_BK) * 2 * SP_BM;
  }
  return t;
}

void split_prepare_grouped(const Stream& st, const SplitPrepJob* d_jobs, int n, long long threads) {
  const int blocks = (int)std::min<long long>((threads + 255) / 256, 148LL * 16);
  split_prepare_grouped_kernel<<<blocks, 256, 0, st.s>>>(d_jobs, n, threads);
  after_launch(st);
}

}  // namespace mpsgpu
