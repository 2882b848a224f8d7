// Host-side engine of the mpsgpu library: device-resident MPO/MPS/environment
// storage and the sweep algorithms of the reference's Contractor, driving the
// CUDA kernels of kernels.h on one stream per context.
#pragma once

#include <array>
#include <atomic>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace mpsgpu {

// Device buffer owned by the engine (stream-ordered allocation).
struct DBuf {
  cplx* p = nullptr;
  long long cap = 0;  // complex elements
};

// Device words of a context (zero at rest): one barrier pair per instance of
// a Lanczos-step launch, from kLzBarrierOffset.
constexpr int kLzBarrierOffset = 0;
constexpr int kCounterWords = 2 * LZ_MAXI;
// Descriptor ring of a context: slots of kDescSlotBytes.
constexpr int kDescSlots = 8;
constexpr size_t kDescSlotBytes = 64 * 1024;

struct Context;

void dbuf_reserve(Context& c, DBuf& b, long long n);
void dbuf_free(Context& c, DBuf& b);

// Workspace of one local eigenproblem (one per concurrent sweep): Krylov
// basis V (N x (m+1)), the product w, the product's temporaries, the thick
// restart's V G and G, and the Lanczos coefficients (device, and a pinned
// host mirror the step writes through its mapping).
struct LzWork {
  DBuf V, w, t2, t3, T, Q;
  DBuf s1, s2, spart, sx, st;  // split-precision products: T1, T2, partials (FP64); x, T2 planes (bytes)
  LanczosScalars* dsc = nullptr;
  LanczosScalars* hsc = nullptr;
  LanczosScalars* hsc_dev = nullptr;
  double* dS = nullptr;
  void init(Context& c);
  void release(Context& c);
};

struct MpoDev {
  int L = 0;
  std::vector<std::array<int, 4>> dims;  // (du, wl, dd, wr)
  std::vector<DBuf> W;      // reference layout (du, wl, dd, wr)
  std::vector<DBuf> Wlr;    // (du*wr) x (wl*dd): out (s', c), in (b, s)   [matvec, left env]
  std::vector<DBuf> Wrl;    // (wl*du) x (dd*wr): out (b, t), in (s, c)   [right env]
  std::vector<DBuf> Wlr_h;  // same as Wlr for the adjoint operator (du == dd only)
  std::vector<DBuf> Wrl_h;
};

struct MpsDev {
  int L = 0;
  std::vector<std::array<int, 3>> dims;  // (d, Dl, Dr)
  std::vector<DBuf> A;                   // device layout X(a, s, r): a fastest
  double normfact = 1.0;
  int gauge = 0;  // enum Gauge of the reference: gNone=0, gLeft=1, gRight=2, gBoth=3
  int bond = 0;
  int max_bond() const;
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  long long launches = 0;
  Scratch scratch;   // short-lived (GEMM split-K partials, reductions)
  Scratch qrws;      // QR T factors
  std::string last_error;
  // reusable workspaces (complex elements)
  DBuf t1, t2, t3, t4, matA, matQ, matR;
  DBuf lzws;           // workspace of the fused Lanczos step (partial dots and norms)
  LzWork lzone;        // eigensolver workspace of single solves
  int* hlz_err = nullptr;  // pinned, mapped: set when a grid barrier of the Lanczos step ran out
  int* dlz_err = nullptr;  // its device address
  // descriptor tables of grouped launches: a ring of pinned host slots copied
  // to device slots in stream order (a slot is rewritten only after its copy
  // has completed, and on the device only by a later copy on the same stream)
  uint8_t* hdesc = nullptr;
  uint8_t* ddesc = nullptr;
  cudaEvent_t desc_ev[kDescSlots] = {};
  int desc_next = 0;
  int* hsplit_err = nullptr;   // pinned, mapped: set by a tensor-core kernel whose bounded wait ran out
  int* dsplit_err = nullptr;   // its device address
  double* dscal = nullptr;     // device scalars (alpha, beta, norms)
  cplx* dcplx = nullptr;       // device complex scalars (dots)
  double* hscal = nullptr;     // pinned host mirror
  cplx* hcplx = nullptr;
  unsigned* dcounter = nullptr;   // kCounterWords device words: the Lanczos step's barrier pairs
  std::vector<cudaEvent_t> iter_ev;  // one per Lanczos iteration in flight
  cudaEvent_t ev = nullptr;
  cudaEvent_t mv0 = nullptr, mv1 = nullptr;
  GemmProfiler prof;
  std::vector<std::unique_ptr<Context>> subs;  // sub-contexts of the sweeps of a batch
  Context* parent = nullptr;                   // a sub-context counts its launches there
  Stream st() { return Stream{stream, parent ? &parent->launches : &launches, parent ? &parent->prof : &prof}; }
};

// Context set-up and release (mpsgpu_create / mpsgpu_destroy), and the i-th
// sub-context of c (created on first use, released with c).
void context_init(Context& c, int device);
void context_release(Context& c);
Context& context_sub(Context& c, int i);

// Environment cache (TmpManager, src/core/cpp/TmpManager.cpp:22-160):
// L[pos] (Dbra, w, Dket) and Rt[pos] (Dket, w, Dbra) (R transposed), with
// validity flags; L[0] = Rt[L-1] = 1.
struct EnvCache {
  int L = 0;
  std::vector<DBuf> Le, Re;
  std::vector<std::array<int, 3>> ldims, rdims;  // ldims (Db, w, Dk); rdims (Dk, w, Db)
  std::vector<char> okL, okR;
  void init(Context& c, int L);
  void release(Context& c);
  void outofdate_l(int l) { if (l > 0) okL[l] = 0; }
  void outofdate_r(int l) { if (l < L - 1) okR[l] = 0; }
};

// Norm caches between the state and one projected level (TmpManagerExc,
// src/core/headers/TmpManagerExc.h:29-45): nL[pos] (Dlevel, Dket), nRt[pos]
// (Dket, Dlevel).
struct NormCache {
  std::vector<DBuf> nL, nR;
  std::vector<std::array<int, 2>> ldims, rdims;
  void init(Context& c, int L);
  void release(Context& c);
};

struct Counters {
  long long site_solves = 0, matvecs = 0, env_updates = 0, qr_calls = 0;
  double flops = 0.0;
  double mv_ms = 0.0;
  int rounds = 0;
  long long split_matvecs = 0;  // products in split precision
  int split_rounds = 0;         // half-sweeps in split precision
  double host_launch_s = 0.0, host_wait_s = 0.0, host_tridiag_s = 0.0;  // eigensolver loop, host side
};

struct SolveOptions {
  double convtol = 1e-5, eigtol = 0.0, excorthtol = 0.0;
  int max_rounds = 1000, max_krylov = 64, verbose = 0;
  // 0: complex FP64 throughout; 1: mixed (split-precision matvec products
  // until the half-sweep energy settles to kSplitSwitchTol, then FP64 to convtol)
  int precision = 0;
  // Raised by another host thread to stop a sweep between two site steps
  // (MPSGPU_CANCELLED); nothing is in flight on the device when it returns.
  const volatile int* cancel = nullptr;
  void check_cancel() const {
    if (cancel && __atomic_load_n(cancel, __ATOMIC_ACQUIRE)) throw Error(MPSGPU_CANCELLED, "solve cancelled");
  }
  // checkpoints (tmpfile, freqSv, maxTime of the reference)
  std::string checkpoint;
  int checkpoint_every = 200;
  double checkpoint_seconds = 0.0;
};

// ---- building blocks (device layout) ----
void mpo_upload(Context& c, MpoDev& m, int L, const int* dims, const double* const* data,
                bool check_edges = true);
void mpo_free(Context& c, MpoDev& m);
void mps_upload(Context& c, MpsDev& s, int L, const int* dims, const double* const* data, double nf);
void mps_random(Context& c, MpsDev& s, int L, int d, int D, uint64_t seed);
void mps_random_state(Context& c, MpsDev& s, int L, int d, int D, uint64_t seed);
void mps_product(Context& c, MpsDev& s, int L, int d, int D);
void mps_copy(Context& c, const MpsDev& src, MpsDev& dst);
void mps_download(Context& c, const MpsDev& s, double* const* data);
void mps_free(Context& c, MpsDev& s);
void mps_gauge_all(Context& c, MpsDev& s, char dir, bool normal, int cutD = 0, double* disc = nullptr);
void mps_approximate(Context& c, const MpsDev& src, MpsDev& dst, int D, double* disc);
void mps_apply_mpo(Context& c, const MpoDev& ops, const MpsDev& src, MpsDev& dst, int cutD, bool dagger, char dir,
                   double* disc);
void mps_gauge_site(Context& c, MpsDev& s, int pos, char dir, bool next, Counters* cnt);
void mps_increase_bond(Context& c, MpsDev& s, int D);

// y = Heff x (+ offset x); environments in device layout.
// Operands of one site's effective Hamiltonian prepared for the split-precision
// products: BF16 limb planes of L (rows Dlb*wl, inner Dlk) and Rt (rows Drb,
// inner Drk*wr), both with 128-row tiles, made once per site solve.
struct SplitMatvec {
  DBuf Lp, Rp;
  bool ready = false;
};
void split_matvec_prepare(Context& c, SplitMatvec& s, const cplx* Le, const std::array<int, 3>& ld,
                          const MpoDev& m, int k, const cplx* Rt, const std::array<int, 3>& rd);
void split_matvec_release(Context& c, SplitMatvec& s);
// y = Heff x + offset x in FP64.
void heff_apply(Context& c, const cplx* Le, const std::array<int, 3>& ld, const MpoDev& m, int k,
                bool adjoint, const cplx* Rt, const std::array<int, 3>& rd, const cplx* x,
                cplx* y, cplx offset, Counters* cnt);
// y = 1/2 (H x + H^dag x) + offset x (TensorMultiplierHermitian) in FP64; Lh,
// Rth the adjoint environments.
void heff_apply_hermitian(Context& c, const cplx* Le, const cplx* Lh, const std::array<int, 3>& ld,
                          const MpoDev& m, int k, const cplx* Rt, const cplx* Rth, const std::array<int, 3>& rd,
                          const cplx* x, cplx* y, cplx offset, Counters* cnt);
// Split-precision products of one lockstep round, run together: for every
// product y = alpha sum_h L_h W_h R_h x + offset x over its one half (the
// plain multiplier, alpha = 1) or two (H and H^dag, alpha = 1/2), as six
// grouped launches for all of them (x planes, T1 = L X on tcgen05, MPO legs,
// T2 planes, T2 Rt on tcgen05 with K split into partial products, and the
// sum of the partials with the offset term).
struct SplitProduct {
  int nh = 1;
  const SplitMatvec* sp[2] = {nullptr, nullptr};
  const cplx* Wm[2] = {nullptr, nullptr};  // MPO leg matrices (du*wr) x (wl*dd)
  int Dlb = 0, Dlk = 0, wl = 0, dd = 0, Drk = 0, du = 0, wr = 0, Drb = 0;
  const cplx* x = nullptr;
  cplx* y = nullptr;
  cplx alpha = {1.0, 0.0}, offset = {0.0, 0.0};
  LzWork* ws = nullptr;  // the product's intermediates
};
struct SplitRound {
  std::vector<SplitProduct> p;
};
// Enqueues the round's products on c's stream and empties the round (the
// K chunks of its two tcgen05 products autotuned per round shape).
void split_round_run(Context& c, SplitRound& r);
long long split_autotune_entries();
// The grouped launches of one Lanczos round that products append to.
struct RoundBatch {
  Gemm1wBatch g1;
  Gemm3Batch g3;
  SplitRound sr;
};
// Descriptors of the two FP64 contractions of one product (heff.cu).
Gemm1wDesc heff_first_desc(const cplx* Le, int Dlb, int Dlk, int wl, const cplx* x, int dd, int Drk, const cplx* Wm,
                           int du, int wr, cplx* t2);
Gemm3Desc heff_last_desc(const cplx* t2, int M, const cplx* Rt, int K, int Drb, cplx* y, const cplx* x,
                         cplx offset);
// Left/right environment update (Operator::contractleftop / contractrightop).
void env_left_update(Context& c, const cplx* Le, const std::array<int, 3>& ld, const MpsDev& ket,
                     const MpoDev* m, int k, const MpsDev& bra, DBuf& out,
                     std::array<int, 3>& od, Counters* cnt);
void env_right_update(Context& c, const cplx* Rt, const std::array<int, 3>& rd, const MpsDev& ket,
                      const MpoDev* m, int k, const MpsDev& bra, DBuf& out,
                      std::array<int, 3>& od, Counters* cnt);

// ---- files in the reference's binary formats (mpsio.cpp) ----
void mps_export_file(Context& c, const MpsDev& s, const std::string& fn);
void mps_import_file(Context& c, const std::string& fn, MpsDev& s);
void mpo_save_file(Context& c, const MpoDev& m, const std::string& fn);
void mpo_load_file(Context& c, const std::string& fn, MpoDev& m);

// ---- local eigensolver (batched thick-restart Lanczos) ----
// One local problem: product(lc, x, y, sigma, rb) must make y = (H - sigma) x
// appear on the stream of lc (the context running the rounds), either by
// appending to the round's grouped launches rb (FP64 descriptors of the two
// contractions, or a split-precision product; the caller launches them in
// the same round) or by launching its own kernels on lc.
struct LzTask {
  int N = 0;
  cplx* x = nullptr;  // start vector in, normalised eigenvector out
  double tol = 1e-12, shift0 = 0.0;
  const cplx* U = nullptr;  // projector vectors (N x nu), sqrt(penalty) folded in
  int nu = 0;
  int max_krylov = 64;
  std::function<void(Context&, const cplx*, cplx*, double, RoundBatch&)> product;
  LzWork* ws = nullptr;
  Counters* cnt = nullptr;
  double theta = 0.0;  // out: lowest Ritz value
  int iters = 0;       // out: products
};
// Lowest eigenpairs of every task, advanced in lockstep rounds of grouped
// launches; returns when all have converged (their x written).
void lanczos_batch(Context& c, std::vector<LzTask*>& tasks);

// ---- algorithms (Contractor) ----
double find_ground_state(Context& c, const MpoDev& ops, int D, MpsDev& init, double offset,
                         const SolveOptions& opt, Counters& cnt);
double find_ground_state_two_site(Context& c, const MpoDev& ops, int D, MpsDev& init, double offset,
                                  const SolveOptions& opt, Counters& cnt, double* max_discarded);
double find_next_excited_state(Context& c, const MpoDev& ops, int D,
                               const std::vector<const MpsDev*>& levels, MpsDev& init,
                               double offset, const SolveOptions& opt, Counters& cnt);
// Several independent solves swept in lockstep on the context's stream: the
// local eigenproblems of all chains at the same site share grouped launches
// (lanczos_batch).  Per-solve results, counters, status and message.
void find_ground_state_batch(Context& c, const std::vector<const MpoDev*>& ops, int D, std::vector<MpsDev*>& inits,
                             double offset, const SolveOptions& opt, std::vector<double>& energies,
                             std::vector<Counters>& cnts, std::vector<int>& status, std::vector<std::string>& err);
void find_next_excited_state_batch(Context& c, const std::vector<const MpoDev*>& ops, int D,
                                   const std::vector<std::vector<const MpsDev*>>& levels, std::vector<MpsDev*>& inits,
                                   double offset, const SolveOptions& opt, std::vector<double>& energies,
                                   std::vector<Counters>& cnts, std::vector<int>& status,
                                   std::vector<std::string>& err);
void optimize(Context& c, const MpoDev& ops, const MpsDev& orig, MpsDev& init, int D,
              const SolveOptions& opt, double* errN, double* errT, Counters& cnt);
// optimizeSum: init ~ sum_k beta_k kets[k] at bond D (Contractor.cpp:2332-2477).
void optimize_sum(Context& c, const std::vector<const MpsDev*>& kets, const std::vector<cplx>& beta, MpsDev& init,
                  int D, const SolveOptions& opt, Counters& cnt);
cplx contract(Context& c, const MpsDev& ket, const MpoDev* ops, const MpsDev& bra);
cplx contract2(Context& c, const MpoDev& ops, const MpsDev& ket, const MpsDev& bra);
void expectation_local(Context& c, const MpsDev& s, const double* op, double* out);
void schmidt_values(Context& c, const MpsDev& s, int pos, std::vector<double>& vals);
double entropy(Context& c, const MpsDev& s, int pos);

}  // namespace mpsgpu
