// Launchers of the mpsgpu CUDA kernels (host-callable, stream-ordered).
#pragma once

#include "common.cuh"

namespace mpsgpu {

enum { OP_N = 0, OP_C = 1, OP_T = 2 };

// Stream-ordered device buffer that grows on demand (cudaMallocAsync pool).
struct Scratch {
  cudaStream_t stream = nullptr;
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t need) {
    if (need > bytes) {
      if (ptr) cudaFreeAsync(ptr, stream);
      size_t nb = need + need / 4 + 4096;
      cudaError_t e = cudaMallocAsync(&ptr, nb, stream);
      if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        throw Error(MPSGPU_OOM, "scratch allocation failed");
      }
      bytes = nb;
    }
    return ptr;
  }
  void release() {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    bytes = 0;
  }
};

struct GemmArgs {
  int M = 0, N = 0, K = 0, batch = 1;
  const cplx* A = nullptr; long long lda = 0, strideA = 0; int opA = OP_N;
  const cplx* B = nullptr; long long ldb = 0, strideB = 0; int opB = OP_N;
  cplx* C = nullptr; long long ldc = 0, strideC = 0;
  cplx alpha = {1.0, 0.0};
  const cplx* Cin = nullptr; long long ldcin = 0, strideCin = 0;
  cplx beta = {0.0, 0.0};
};

// C = alpha op(A) op(B) + beta Cin  (complex FP64, DMMA tensor pipe)
void zgemm(const Stream& st, const GemmArgs& g, Scratch& scratch);
// Autotuner of zgemm's launch configuration (tile edge, K slices): on by
// default (environment MPSGPU_AUTOTUNE=0 turns it off); entries = shapes tuned.
void set_gemm_autotune(int on);
long long gemm_autotune_entries();
bool gemm_autotune_on();

// One GEMM C = A B (op N, N) of a grouped launch; tile_begin / tiles_m are
// filled by grouped_tiles (64 x 64 tiles).
struct GroupedGemm {
  int M = 0, N = 0, K = 0;
  const cplx* A = nullptr; long long lda = 0;
  const cplx* B = nullptr; long long ldb = 0;
  cplx* C = nullptr; long long ldc = 0;
  long long tile_begin = 0;
  int tiles_m = 0;
};
// Host: assigns tile ranges in order; returns the total number of tiles.
long long grouped_tiles(GroupedGemm* descs, int n);
// All tiles of n GEMMs (descriptors in device memory) in one persistent launch of `ctas` CTAs.
void zgemm_grouped(const Stream& st, const GroupedGemm* d_descs, int n, long long total_tiles, int ctas);

// ---- split-precision complex GEMM (umma.cu): BF16 limbs on tcgen05 ----
// Tiling of C = A B (M x N, inner K): 128-row A tiles, BN-column B tiles,
// k-steps of 16, K split over `splits` CTAs of ks_per_split k-steps each.
struct SplitPlan {
  int M = 0, N = 0, K = 0, KS = 0;
  int BN = 128, mtiles = 0, ntiles = 0;
  int splits = 1, ks_per_split = 0;
};
SplitPlan split_plan(int M, int N, int K, int nsm);
// Bytes of a prepared operand of `rows` rows and inner dimension K, row tile RT.
long long split_operand_bytes(int rows, int K, int RT);
// Six BF16 limb planes of X (rows x K, entry (r, k) at X[r*rs + k*ks]),
// tiled for the tensor cores with row tile RT (128 for A, plan.BN for B,
// whose rows are the columns of C); out is 16-byte aligned.
void split_prepare(const Stream& st, int rows, int K, const cplx* X, long long rs, long long ks, int RT,
                   uint8_t* out);
// C = alpha A B + beta Cin from prepared operands; part holds
// splits * M * N complex partial products when splits > 1; *err is set when
// a bounded wait inside the kernel ran out.
void zgemm_split_prepared(const Stream& st, const SplitPlan& pl, const uint8_t* Ap, const uint8_t* Bp, cplx* C,
                          long long ldc, cplx alpha, const cplx* Cin, long long ldcin, cplx beta, cplx* part,
                          int* err);
// Grouped form: every operand prepared with 128-row tiles (split_prepare
// with RT = 128, or the grouped preparation below); one launch computes all
// C_q = A_q B_q (M_q x N_q, inner K_q), one CTA per 128 x 128 tile.  A
// problem may cover a range of k-steps only (k0, nk; nk = 0: to the end), so
// that a K split is a set of problems writing separate partial products.
struct SplitProblem {
  int M = 0, N = 0, K = 0;
  int KS = 0, mtiles = 0;  // filled by split_group_tiles
  const uint8_t* Ap = nullptr;
  const uint8_t* Bp = nullptr;
  cplx* C = nullptr;
  long long ldc = 0;
  long long tile_begin = 0;
  int k0 = 0, nk = 0;  // k-steps [k0, k0 + nk) of the KS (of 16) the operands hold
};
long long split_group_tiles(SplitProblem* probs, int n);
void zgemm_split_grouped(const Stream& st, const SplitProblem* d_probs, int n, long long tiles, int* err);
// Sum of partial products: C[m + n ldc] = alpha sum_{s < nparts} part[s M N + m + n M]
// + beta Cin[m + n ldcin] for every job, one launch (elements numbered from
// `begin`, filled by split_reduce_jobs).
struct SplitReduceJob {
  int M = 0, N = 0, nparts = 0;
  const cplx* part = nullptr;
  cplx* C = nullptr;
  long long ldc = 0;
  cplx alpha = {1.0, 0.0};
  const cplx* Cin = nullptr;
  long long ldcin = 0;
  cplx beta = {0.0, 0.0};
  long long begin = 0;
};
long long split_reduce_jobs(SplitReduceJob* jobs, int n);
void split_reduce_grouped(const Stream& st, const SplitReduceJob* d_jobs, int n, long long total);
// One preparation job per operand (rows x K, entry (r, k) at X[r*rs + k*ks]).
struct SplitPrepJob {
  int rows = 0, K = 0;
  int KS = 0;  // filled by split_prepare_jobs
  const cplx* X = nullptr;
  long long rs = 0, ks = 0;
  uint8_t* out = nullptr;
  long long thread_begin = 0;  // filled by split_prepare_jobs
};
long long split_prepare_jobs(SplitPrepJob* jobs, int n);
void split_prepare_grouped(const Stream& st, const SplitPrepJob* d_jobs, int n, long long threads);

// ---- grouped effective-Hamiltonian matvec (grouped.cu) ----
// One instance in device layouts: L (Dl, wl, Dl) = (bra, w, ket); W
// (d, wl, d, wr) as the reference stores it; Rt (Dr, wr, Dr) = (ket, w, bra);
// x, y (Dl, d, Dr) with the left bond fastest.
struct HeffInstance {
  int d = 0, wl = 0, wr = 0, Dl = 0, Dr = 0;
  const cplx* L = nullptr;
  const cplx* W = nullptr;
  const cplx* Rt = nullptr;
  const cplx* x = nullptr;
  cplx* y = nullptr;
};
struct DevMem {
  cplx* p = nullptr;
  long long n = 0;
};
inline void dbuf_alloc(const Stream& st, DevMem& m, long long n) {
  MPSGPU_CUDA(cudaMallocAsync((void**)&m.p, std::max<long long>(n, 1) * sizeof(cplx), st.s));
  m.n = n;
}
struct GroupedMatvecPlan {
  int n = 0;
  DevMem t1, t2, wm;
  void* desc = nullptr;
  GroupedGemm* d_g1 = nullptr;
  GroupedGemm* d_g3 = nullptr;
  void* d_wg = nullptr;
  void* d_wp = nullptr;
  long long tiles1 = 0, tiles3 = 0, pixels = 0, wel = 0;
  int maxnin = 1, maxnout = 1, ctas = 148;
  double flops = 0.0;  // algorithmic flops of one grouped product
  // split precision: BF16 limb planes of L, Rt (prepared once by
  // grouped_matvec_prepare_env), x and T2 (prepared in every product)
  bool split = false;
  DevMem sp;                                  // all prepared planes
  void* sdesc = nullptr;                      // device tables below
  SplitProblem* d_s1 = nullptr;               // T1 = L . x
  SplitProblem* d_s3 = nullptr;               // y = T2 . Rt
  SplitPrepJob* d_jenv = nullptr;             // L and Rt, 2n jobs
  SplitPrepJob* d_jx = nullptr;               // x, n jobs
  SplitPrepJob* d_jt = nullptr;               // T2, n jobs
  long long stiles1 = 0, stiles3 = 0, thr_env = 0, thr_x = 0, thr_t = 0;
  int* err = nullptr;                         // set by a tensor-core kernel whose bounded wait ran out
  ~GroupedMatvecPlan();
};
// split = true plans the split-precision form (tcgen05, BF16 limbs).
void grouped_matvec_plan(const Stream& st, const std::vector<HeffInstance>& inst, GroupedMatvecPlan& plan,
                         int nsm, bool split = false);
// Split form: the limb planes of the environments, made once per set of instances.
void grouped_matvec_prepare_env(const Stream& st, GroupedMatvecPlan& plan);
void grouped_matvec_run(const Stream& st, GroupedMatvecPlan& plan);
void grouped_matvec_free(const Stream& st, GroupedMatvecPlan& plan);

// MPO-leg contraction: for every pixel (x, y) in [0,nx) x [0,ny)
//   out[x*ox + y*oy + o0*so0 + o1*so1] =
//       sum_{i0,i1} Wm[(o0 + n_o0*o1) + nout*(i0 + n_i0*i1)] in[x*ix + y*iy + i0*si0 + i1*si1]
// with Wm an (n_o0*n_o1) x (n_i0*n_i1) column-major complex matrix in device memory.
struct WContractArgs {
  int nx = 0, ny = 0;
  const cplx* in = nullptr; long long ix = 0, iy = 0, si0 = 0, si1 = 0; int n_i0 = 0, n_i1 = 0;
  cplx* out = nullptr; long long ox = 0, oy = 0, so0 = 0, so1 = 0; int n_o0 = 0, n_o1 = 0;
  const cplx* Wm = nullptr;
};
void wcontract(const Stream& st, const WContractArgs& a);
// The MPO-leg contraction of n problems in one launch (grouped.cu): problem
// q covers the pixels [pix_begin_q, pix_begin_q + nx ny), pix_begin_q a
// multiple of WC_CHUNK (pixel ranges padded by wcontract_chunked), within
// `pixels`; maxnin and maxnout are the largest n_i0 n_i1 and n_o0 n_o1 (at
// most 32 inputs, 1024 leg entries).  With parts > 1 the input is the sum of
// `parts` arrays part_stride apart (the partial products of a K split), added
// in order.
constexpr int WC_THREADS = 128;
constexpr int WC_CHUNK = 512;
struct WGroup {
  WContractArgs a;
  long long pix_begin = 0;
  int parts = 1;
  long long part_stride = 0;
};
long long wcontract_chunked(long long pixels);
void wcontract_grouped(const Stream& st, const WGroup* d_wg, int n, long long pixels, int maxnin, int maxnout);

// ---- effective-Hamiltonian contractions (heff.cu), grouped ----
constexpr int GEMM_MAXP = 16;  // problems per launch
// T2 = Wm . (A B) per pixel: C = A B with A(row, k) = A[row + k lda],
// B(k, col) = B[k + col ldb]; rows x + X i0 (i0 < n_i0), columns i1 + n_i1 y
// (i1 < n_i1); for every pixel (x < X, y < Y)
//   out[x ox + y oy + o0 so0 + o1 so1] = sum_{i0,i1} Wm[(o0 + n_o0 o1) + nout (i0 + n_i0 i1)] C[(x,i0),(i1,y)]
// (Wm column-major nout x nin in device memory, nin = n_i0 n_i1 <= 1024).
struct Gemm1wDesc {
  const cplx* A = nullptr;
  long long lda = 0;
  const cplx* B = nullptr;
  long long ldb = 0;
  int X = 0, Y = 0, K = 0, n_i0 = 0, n_i1 = 0, n_o0 = 0, n_o1 = 0;
  const cplx* Wm = nullptr;
  cplx* out = nullptr;
  long long ox = 0, oy = 0, so0 = 0, so1 = 0;
  int tiles_x = 0, tiles_y = 0, tile_begin = 0;  // filled by heff_gemm1w
};
struct Gemm1wBatch {
  int n = 0;
  Gemm1wDesc d[GEMM_MAXP];
};
void heff_gemm1w(const Stream& st, Gemm1wBatch& b);
// C = alpha (A1 B1 + A2 B2) + beta Cin, column-major, op N: A1 M x K1,
// B1 K1 x N, and (K2 > 0) A2 M x K2, B2 K2 x N; Cin may be null.
struct Gemm3Desc {
  int M = 0, N = 0, K1 = 0, K2 = 0;
  const cplx* A1 = nullptr;
  long long lda1 = 0;
  const cplx* B1 = nullptr;
  long long ldb1 = 0;
  const cplx* A2 = nullptr;
  long long lda2 = 0;
  const cplx* B2 = nullptr;
  long long ldb2 = 0;
  cplx alpha = {1.0, 0.0}, beta = {0.0, 0.0};
  const cplx* Cin = nullptr;
  long long ldcin = 0;
  cplx* C = nullptr;
  long long ldc = 0;
  int tiles_m = 0, tiles_n = 0, tile_begin = 0;  // filled by heff_gemm3
};
struct Gemm3Batch {
  int n = 0;
  Gemm3Desc d[GEMM_MAXP];
};
void heff_gemm3(const Stream& st, Gemm3Batch& b);

// ---- vector kernels (Lanczos, norms) ----
// dots[j] = sum_i conj(V[i + j*ldv]) w[i], j < k   (two-stage, deterministic)
void cgemv_c(const Stream& st, int n, int k, const cplx* V, long long ldv, const cplx* w,
             cplx* dots, Scratch& scratch);
// w += sign * V h  (h on device, length k; sign = -1 subtracts)
void cgemv_n_sub(const Stream& st, int n, int k, const cplx* V, long long ldv, const cplx* h,
                 cplx* w, double sign = -1.0);
// Lanczos coefficients written by the fused orthogonalisation kernels.
struct LanczosScalars {
  double alpha[256];
  double beta[256];
  cplx loc;    // v_j^H w after the beta_{j-1} v_{j-1} subtraction (local step)
  double nb2;  // |w'|^2 before the first Gram-Schmidt pass
  double ap;   // first-pass Re h_j, while a second pass is pending
  int flag;    // second pass needed
};
// One reorthogonalised Lanczos step (local three-term subtraction, classical
// Gram-Schmidt against the basis with a second pass when the norm drops below
// 1/sqrt(2) of its value, normalisation; an optional projector) for a group
// of independent instances in one cooperative launch (lzstep.cu).  Per instance: w = (H - sigma) v_j on
// entry; on exit sc->alpha[j], sc->beta[j] (and the mirror) are set and, when
// write_next, V[:, j+1] = w / beta_j.  With nu > 0, U (n x nu, ld n) holds the
// projector vectors (sqrt of the penalty folded in) and w += U (U^H v_j)
// first.  Workspaces: part and part2 nrb_total x 256 complex, pn1/pn2
// nrb_total; bar 2 x LZ_MAXI unsigned words that are zero at rest (one pair
// per instance).
constexpr int LZ_THREADS = 256;
constexpr int LZ_MAXI = 16;  // instances per launch
constexpr int LZ_MAXU = 8;   // projector vectors per instance
struct LzInst {
  int n = 0, j = 0, k = 0, nu = 0, write_next = 0;
  int rb0 = 0, nrb = 0;     // row blocks, filled by lanczos_step
  int cta0 = 0, ncta = 0;   // the instance's CTAs, filled by lanczos_step
  double sigma = 0.0;
  cplx* V = nullptr;
  long long ldv = 0;
  cplx* w = nullptr;
  const cplx* U = nullptr;
  LanczosScalars* sc = nullptr;
  LanczosScalars* mirror = nullptr;
};
struct LzBatch {
  int ninst = 0, nrb_total = 0;
  LzInst in[LZ_MAXI];
  cplx* part = nullptr;
  cplx* part2 = nullptr;
  double* pn1 = nullptr;
  double* pn2 = nullptr;
  unsigned* bar = nullptr;
  int* err = nullptr;  // set when a bounded barrier ran out
};
// Rows per row block (the unit of the workspaces' nrb counts).
int lanczos_step_rows_per_block();
void lanczos_step(const Stream& st, LzBatch& b);

// out[0] = ||x||_2 (deterministic two-stage reduction)
void dznrm2(const Stream& st, int n, const cplx* x, double* out, Scratch& scratch);
// y = x / (*nrm)   (device scalar)
void zscal_inv(const Stream& st, int n, const cplx* x, const double* nrm, cplx* y);
// y = a x + b y (host scalars)
void zaxpby(const Stream& st, int n, cplx a, const cplx* x, cplx b, cplx* y);
// y = sum_j s[j] V[:, j]  (s real, device)
void combine_real(const Stream& st, int n, int k, const cplx* V, long long ldv, const double* s,
                  cplx* y);
// dst = src (n complex)
void zcopy(const Stream& st, int n, const cplx* src, cplx* dst);
void zfill(const Stream& st, long long n, cplx v, cplx* dst);

// ---- layout conversions between the reference and the device layout ----
// site: ref A(s, a, r) -> dev X(a, s, r) and back
void site_ref_to_dev(const Stream& st, int d, int Dl, int Dr, const cplx* ref, cplx* dev);
void site_dev_to_ref(const Stream& st, int d, int Dl, int Dr, const cplx* dev, cplx* ref);
// 3-index transpose T(p, q, r) -> U(r, q, p) (used for R environments)
void transpose_pqr_to_rqp(const Stream& st, int p, int q, int r, const cplx* in, cplx* out,
                          bool conj = false);

// Seeded complex Gaussian fill (SplitMix64 counter stream + Box-Muller),
// entry i uses draws 2(offset+i), 2(offset+i)+1; written in the reference
// site order (s fastest) into the device layout (a fastest).
void gaussian_site(const Stream& st, uint64_t seed, long long offset, int d, int Dl, int Dr,
                   cplx* dev);

// Singular values (descending) of the m x n matrix A (device, ld lda) by
// one-sided Jacobi (svd.cu); host-synchronous, A untouched.
std::vector<double> singular_values(const Stream& st, int m, int n, const cplx* A, long long lda,
                                    Scratch& scratch);
// Thin SVD with the cut of wrapper::svd(A, 0, cut): U (m x keep, ld m),
// diag(s) V^H (keep x n, ld keep); all min(m, n) values in sv; returns keep.
int svd_cut(const Stream& st, int m, int n, const cplx* A, long long lda, int cut, cplx* U, cplx* SVh,
            std::vector<double>& sv, Scratch& scratch, bool left_s = false);

// ---- Householder QR (LAPACK zgeqrf/zungqr conventions) ----
// Factor the m x n column-major matrix A (ld = m; overwritten by R above and
// the reflectors below the diagonal).  Q (m x K, ld = ldq) and R (K x n,
// ld = ldr, zero below the diagonal) are written when non-null; K = min(m, n).
void householder_qr_inplace(const Stream& st, int m, int n, cplx* A, cplx* Q, long long ldq,
                            cplx* R, long long ldr, Scratch& scratch);
// Places the fixed scratch array of mpsgpu_qr_device_noalloc on device `dev`
// (current) and sets its kernels' attributes; called when a context is created.
mpsgpu_status noalloc_qr_prepare(int dev);

// Two-level strided view: element (i, j) lives at
//   (i % rd)*r0 + (i / rd)*r1 + (j % cd)*c0 + (j / cd)*c1, optionally conjugated.
struct View2 {
  long long rd = 1, r0 = 1, r1 = 0, cd = 1, c0 = 0, c1 = 0;
  bool conj = false;
};
// dst (m x n, col-major, ld m) = view(src)
void gather2(const Stream& st, int m, int n, const cplx* src, const View2& v, cplx* dst);
// view(dst) = src (m x n, col-major, ld m)
void scatter2(const Stream& st, int m, int n, const cplx* src, cplx* dst, const View2& v);

}  // namespace mpsgpu
