/*
 * mpsgpu -- C ABI of the B200 DMRG sweep library (sm_100a, complex FP64).
 *
 * This is the drop-in boundary for the single-site DMRG hot path of
 * mcbapo/mpsdyn.  Every entry point takes plain pointers and sizes; tensors
 * cross the boundary in the reference's own layout:
 *
 *   complex128 = two doubles (re, im), interleaved (src/wrapper/complex.h)
 *   all tensors column-major ("Fortran order", src/wrapper/mwArray.cpp:452-470)
 *   site tensor     A(d, Dl, Dr)              (src/core/cpp/Site.cpp:16-21)
 *   MPO tensor      W(du, Dl, dd, Dr)         (src/core/cpp/Operator.cpp:17-24)
 *   environments    L(Dbra, w, Dket), R(Dbra, w, Dket)
 *                                             (src/core/cpp/Operator.cpp:273-387)
 *   local vector    vec(A(d, Dl, Dr))         (src/wrapper/multipliers/TensorMultiplier.h:28)
 *
 * Inside the library the state lives in HBM in its own layout (see the design
 * notes); uploads and downloads convert.  Every function returns an
 * mpsgpu_status; the reference's convention of printing and calling exit()
 * (e.g. exit(212) on an energy increase, Contractor.cpp:1418-1427) becomes a
 * status code, and the C++ facade restores the reference behaviour.
 *
 * Threading: calls on one context are serialised on that context's CUDA
 * stream; different contexts may be used from different host threads.
 */
#ifndef MPSGPU_H
#define MPSGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MPSGPU_OK = 0,
  MPSGPU_BAD_SHAPE = 1,       /* inconsistent or unsupported dimensions */
  MPSGPU_NOT_CONVERGED = 2,   /* eigensolver or sweep limit reached */
  MPSGPU_ENERGY_INCREASE = 3, /* Contractor.cpp:1418-1427 (reference: exit 212) */
  MPSGPU_NAN = 4,             /* non-finite value (Contractor.cpp:954-960: exit 1) */
  MPSGPU_OOM = 5,             /* device allocation failed */
  MPSGPU_CANCELLED = 6,       /* cancel flag raised by the caller */
  MPSGPU_TIMEOUT = 7,         /* bounded device wait gave up */
  MPSGPU_CUDA_ERROR = 8,      /* CUDA runtime error (see mpsgpu_last_error) */
  MPSGPU_INVALID = 9          /* null handle or bad argument */
} mpsgpu_status;

typedef struct mpsgpu_context mpsgpu_context;
typedef struct mpsgpu_mpo mpsgpu_mpo;
typedef struct mpsgpu_mps mpsgpu_mps;

/* Solver options.  Defaults (mpsgpu_default_options) are the reference
 * Contractor's: convtol 1e-5, eigtol 0 (Contractor.cpp:39-42). */
typedef struct {
  double convtol;      /* setConvTol (Contractor.h:213) */
  double eigtol;       /* setEigTol; 0 = 1e-12 relative Lanczos residual
                        * (1e-9 in the final half-sweeps of precision 1
                        * and 2, see below) */
  double excorthtol;   /* setExcOrthTol (Contractor.h:229); 0 = no check */
  int max_rounds;      /* half-sweep cap; 0 = 1000 (MAX_ROUND_EXCTD, Contractor.cpp:26) */
  int max_krylov;      /* Lanczos vectors per restart; 0 = 64 */
  int precision;       /* 0 = complex FP64 throughout; 1 = mixed: the
                        * effective-Hamiltonian products of the single-site
                        * ground- and excited-state sweeps run in split
                        * precision (BF16 limbs on the tensor cores,
                        * eigensolver residual 1e-6) until the half-sweep
                        * energy change falls below 1e-6 relative, then in
                        * FP64 at residual 1e-9 to convtol (at least one
                        * full FP64 round); in optimize (time evolution) 1
                        * computes the local vector L W R x in split
                        * precision throughout (environments stay FP64);
                        * 2 = the schedule of 1 (its
                        * eigensolver tolerances and phases) with FP64
                        * products, which separates what the schedule
                        * saves from what the tensor cores save */
  int verbose;         /* 1 = one line per half-sweep on stdout */
  /* Optional: when *cancel_flag becomes non-zero (set by another host
   * thread), the sweep stops between two site steps with MPSGPU_CANCELLED. */
  const volatile int* cancel_flag;
  /* Checkpoints (the reference's tmpfile / freqSv / maxTime arguments of
   * findGroundState, Contractor.h:255-257, and findNextExcitedState,
   * Contractor.h:309-314): when checkpoint_file is non-null the state is
   * written there in the reference's binary MPS format (MPS::exportMPS).
   * Ground state: at the end of a half-sweep that does not converge, when
   * the half-sweep count is a multiple of checkpoint_every (0 = 200), as
   * Contractor.cpp:1526-1530.  Excited state: at the end of every half-sweep
   * when checkpoint_seconds <= 0, else once at least checkpoint_seconds of
   * wall time have passed since the last save (the reference counts CPU
   * time, Contractor.cpp:2868-2883).  Restart by importing the file
   * (mpsgpu_mps_import) and calling the solver again. */
  const char* checkpoint_file;
  int checkpoint_every;
  double checkpoint_seconds;
} mpsgpu_options;

/* Counters of one solve (host-side; the flop count is algorithmic). */
typedef struct {
  int rounds;                /* half-sweeps */
  long long site_solves;     /* local eigenproblems */
  long long matvecs;         /* effective-Hamiltonian products */
  long long env_updates;     /* environment contractions */
  long long qr_calls;        /* gauge moves */
  double flops;              /* algorithmic flops, all kernels */
  double seconds;            /* wall time of the call */
  double matvec_seconds;     /* device time spent in matvec kernels (events) */
  long long split_matvecs;   /* products run in split precision (precision = 1) */
  int split_rounds;          /* half-sweeps run in split precision */
  /* host time of the local eigensolver's loop: launching the iterations,
   * waiting for their results, solving the projected tridiagonal problem */
  double host_launch_seconds;
  double host_wait_seconds;
  double host_tridiag_seconds;
} mpsgpu_stats;

/* ---- context ------------------------------------------------------------ */
void mpsgpu_default_options(mpsgpu_options* opt);
mpsgpu_status mpsgpu_create(int device, mpsgpu_context** ctx);
mpsgpu_status mpsgpu_destroy(mpsgpu_context* ctx);
const char* mpsgpu_status_string(mpsgpu_status s);
const char* mpsgpu_last_error(mpsgpu_context* ctx);
/* Counts this library's kernel launches on the context (for reporting). */
long long mpsgpu_launch_count(mpsgpu_context* ctx);
mpsgpu_status mpsgpu_synchronize(mpsgpu_context* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time the
 * library's work with their own events on that stream. */
mpsgpu_status mpsgpu_get_stream(mpsgpu_context* ctx, void** stream);
/* Device-time accounting of the tensor-pipe GEMMs: between begin and end,
 * CUDA events bracket one GEMM launch in 32 on the context's stream; end
 * returns the summed device time (ms), algorithmic flops and count of the
 * sampled launches (their ratio is the average per-launch throughput). */
mpsgpu_status mpsgpu_profile_begin(mpsgpu_context* ctx);
mpsgpu_status mpsgpu_profile_end(mpsgpu_context* ctx, double* gemm_ms, double* gemm_flops,
                                 long long* gemm_calls);
/* After mpsgpu_profile_end: the same per kernel class (arrays of
 * MPSGPU_PROFILE_CLASSES entries, each may be null): 0 complex FP64 GEMMs on
 * the DMMA pipe, 1 split-precision GEMMs on tcgen05 (work = BF16 tensor
 * flops), 2 the fused Lanczos step (work = algorithmic bytes), 3 Householder
 * QR (flops), 4 the split products' operand passes (BF16 limb planes, MPO
 * legs, sums of K chunks; work = bytes).  Sampled launches: one in 32 of each
 * class; ms their summed device time, work their summed algorithmic work. */
#define MPSGPU_PROFILE_CLASSES 5
mpsgpu_status mpsgpu_profile_kernels(mpsgpu_context* ctx, double* ms, double* work, long long* calls);

/* ---- MPO (replaces MPO / Operator storage, src/core/headers/MPO.h:33-176) --
 * dims[4k..4k+3] = (du, Dl, dd, Dr) of operator k; data[k] its column-major
 * complex128 tensor (host memory). */
mpsgpu_status mpsgpu_mpo_upload(mpsgpu_context* ctx, int L, const int* dims,
                                const double* const* data, mpsgpu_mpo** out);
mpsgpu_status mpsgpu_mpo_free(mpsgpu_context* ctx, mpsgpu_mpo* mpo);
/* MPO::saveMPO / loadMPO (src/core/cpp/MPO.cpp:214-231, 291-312): the
 * reference's binary MPO file (int length, then every operator as an
 * mwArray: int rank, int dims[rank], column-major complex128 data). */
mpsgpu_status mpsgpu_mpo_save(mpsgpu_context* ctx, const mpsgpu_mpo* mpo, const char* filename);
mpsgpu_status mpsgpu_mpo_load(mpsgpu_context* ctx, const char* filename, mpsgpu_mpo** out);
/* Length and dims[4k..4k+3] = (du, Dl, dd, Dr) of an uploaded MPO (either
 * output may be null), and its tensors back to host buffers (data[k] holds
 * du*Dl*dd*Dr complex128, column-major), as MPO::getOpData returns them. */
mpsgpu_status mpsgpu_mpo_info(mpsgpu_context* ctx, const mpsgpu_mpo* mpo, int* L,
                              int* dims);
mpsgpu_status mpsgpu_mpo_download(mpsgpu_context* ctx, const mpsgpu_mpo* mpo,
                                  double* const* data);
/* Model MPOs built by the library (host tensors as the reference builds
 * them, then uploaded):
 *   IsingHamiltonian(L, 2, J, g, h).getHMPO() (models/cpp/IsingHamiltonian.cpp:70-121)
 *   IsingHamiltonian::getUMPO(mpo, delta, 0, imag, 2)     (IsingHamiltonian.cpp:131-148)
 *   SchwingerHamiltonian(N, mu, x, l0, alpha).getHMPO()    (models/cpp/SchwingerHamiltonian.cpp:13-121) */
mpsgpu_status mpsgpu_mpo_ising(mpsgpu_context* ctx, int L, double J, double g, double h,
                               mpsgpu_mpo** out);
mpsgpu_status mpsgpu_mpo_ising_evolution(mpsgpu_context* ctx, int L, double J, double g,
                                         double h, double delta, int imag, mpsgpu_mpo** out);
mpsgpu_status mpsgpu_mpo_schwinger(mpsgpu_context* ctx, int N, double mu, double x, double l0,
                                   double alpha, mpsgpu_mpo** out);
/* HeisenbergHamiltonian(L, Jx, Jy, Jz, hx, hy, hz, 2, offset).getHMPO()
 * (models/cpp/HeisenbergHamiltonian.cpp:266-331): spin-1/2 XYZ chain with
 * uniform couplings and fields, MPO bond 5. */
mpsgpu_status mpsgpu_mpo_heisenberg(mpsgpu_context* ctx, int L, double Jx, double Jy, double Jz,
                                    double hx, double hy, double hz, double offset,
                                    mpsgpu_mpo** out);
/* BoseHubbardHamiltonian(L, N, t, U, Ntarget, penN, V).getHMPO()
 * (models/cpp/BoseHubbardHamiltonian.cpp:7-17, 73-160): bosons with at most
 * N per site (d = N + 1), H = -t sum (b+_i b_i+1 + h.c.) + U/2 sum n_i(n_i-1)
 * + V sum n_i + penN (sum n_i - Ntarget)^2, MPO bond 5; t >= 0
 * (MPSGPU_INVALID otherwise). */
mpsgpu_status mpsgpu_mpo_bosehubbard(mpsgpu_context* ctx, int L, int N, double t, double U, int Ntarget,
                                     double penN, double V, mpsgpu_mpo** out);

/* ---- MPS (replaces MPS / Site storage, src/core/headers/MPS.h) ------------
 * dims[3k..3k+2] = (d, Dl, Dr) of site k; data[k] column-major complex128. */
mpsgpu_status mpsgpu_mps_upload(mpsgpu_context* ctx, int L, const int* dims,
                                const double* const* data, double normfact,
                                mpsgpu_mps** out);
/* Seeded i.i.d. complex Gaussian MPS on the bond schedule
 * D_k = min(d^k, d^(L-k), D), generated on the device from the SplitMix64
 * counter stream (entry i of the chain uses draws 2i, 2i+1, Box-Muller). */
mpsgpu_status mpsgpu_mps_random(mpsgpu_context* ctx, int L, int d, int D,
                                uint64_t seed, mpsgpu_mps** out);
/* The same sites right-gauged one after another as MPS::setRandomState
 * does (src/core/cpp/MPS.cpp:282-294): a normalised chain of random
 * isometries, safe from overflow at any L (the raw Gaussian chain above
 * grows like (d D)^(L/2)). */
mpsgpu_status mpsgpu_mps_random_state(mpsgpu_context* ctx, int L, int d, int D,
                                      uint64_t seed, mpsgpu_mps** out);
/* MPS(L,D,d) of the reference (src/core/cpp/MPS.cpp:15-35): element (0,0,0)
 * of every site is 1, bonds D (D=1: the product state |0...0>). */
mpsgpu_status mpsgpu_mps_product(mpsgpu_context* ctx, int L, int d, int D,
                                 mpsgpu_mps** out);
mpsgpu_status mpsgpu_mps_copy(mpsgpu_context* ctx, const mpsgpu_mps* src,
                              mpsgpu_mps** out);
mpsgpu_status mpsgpu_mps_info(mpsgpu_context* ctx, const mpsgpu_mps* mps,
                              int* L, int* dims, double* normfact);
mpsgpu_status mpsgpu_mps_download(mpsgpu_context* ctx, const mpsgpu_mps* mps,
                                  double* const* data);
mpsgpu_status mpsgpu_mps_free(mpsgpu_context* ctx, mpsgpu_mps* mps);
/* MPS::exportMPS / importMPS (src/core/cpp/MPS.cpp:442-509): the
 * reference's binary MPS file (int length, int bond, double normfact, int
 * gauge, then per site int pos and the site as an mwArray (d, Dl, Dr)). */
mpsgpu_status mpsgpu_mps_export(mpsgpu_context* ctx, const mpsgpu_mps* mps, const char* filename);
mpsgpu_status mpsgpu_mps_import(mpsgpu_context* ctx, const char* filename, mpsgpu_mps** out);
/* MPS::gaugeCond(dir, normal=true) (src/core/cpp/MPS.cpp:306-364). */
mpsgpu_status mpsgpu_mps_gauge(mpsgpu_context* ctx, mpsgpu_mps* mps, char dir);
/* MPS::gaugeCond(dir, normalize, cutD) (src/core/cpp/MPS.cpp:306-364): QR
 * (cutD = 0) or SVD-cut (cutD > 0, bonds <= cutD) sweep; normalize = 0 keeps
 * the norm in normfact.  discarded (nullable): sum of dropped squares. */
mpsgpu_status mpsgpu_mps_gauge_cond(mpsgpu_context* ctx, mpsgpu_mps* mps, char dir,
                                    int normalize, int cutD, double* discarded);
/* MPS::increaseBondDimension(D) (src/core/cpp/MPS.cpp:650-719): integer bond
 * schedule and zero padding. */
mpsgpu_status mpsgpu_mps_increase_bond(mpsgpu_context* ctx, mpsgpu_mps* mps, int D);
/* The bond field and the gauge tag (0 none, 1 left, 2 right) the reference
 * keeps beside the tensors (MPS::getBond, MPS.h:62-70), and the norm factor
 * setter (MPS::setNormFact). */
mpsgpu_status mpsgpu_mps_bond(mpsgpu_context* ctx, const mpsgpu_mps* mps, int* bond,
                              int* gauge);
mpsgpu_status mpsgpu_mps_set_normfact(mpsgpu_context* ctx, mpsgpu_mps* mps, double normfact);
/* MPS(const MPS& src, int D) (src/core/cpp/MPS.cpp:761-772): a copy cut to
 * bond dimension D by right-to-left SVDs (gaugeCond('L', 0, D), Site::gaugeL
 * with cutD, wrapper::svd with tol 0: zero singular values are dropped too).
 * The norm stays in normfact.  discarded (nullable) receives the sum over
 * the cut bonds of the squares of the dropped singular values, which the
 * reference does not report. */
mpsgpu_status mpsgpu_mps_approximate(mpsgpu_context* ctx, const mpsgpu_mps* src,
                                     int D, mpsgpu_mps** out, double* discarded);
/* MPO applied to an MPS site by site with an SVD gauge move after each site
 * (src/core/cpp/MPS.cpp:858-936, Site::reduceDimLOp/ROp, Site.cpp:303-402):
 * D <= 0 is MPS::applyExactly(ops, dagger, dir) (no cut beyond dropping
 * zero singular values), D > 0 is MPS::truncate(ops, src, D, dagger, dir) /
 * MPS::approximate.  dagger applies ops^dagger; dir 'L' sweeps from the
 * right end (result right-gauged), 'R' from the left end. */
mpsgpu_status mpsgpu_mps_apply_mpo(mpsgpu_context* ctx, const mpsgpu_mpo* ops,
                                   const mpsgpu_mps* src, int D, int dagger,
                                   char dir, mpsgpu_mps** out,
                                   double* discarded);

/* ---- Contractor (src/core/headers/Contractor.h:46-604) ------------------- */
/* findGroundState(ops, D, &lambda, init, offset) (Contractor.cpp:1352-1533). */
mpsgpu_status mpsgpu_find_ground_state(mpsgpu_context* ctx, const mpsgpu_mpo* ops,
                                       int D, double offset,
                                       const mpsgpu_options* opt, mpsgpu_mps* init,
                                       double* lambda, mpsgpu_stats* stats);
/* Two-site DMRG ground state.  No counterpart in the reference (its sweeps
 * are single-site): each bond (k, k+1) is optimised as one two-site tensor
 * with the same thick-restart Lanczos, then split by an SVD cut to at most D
 * (singular values moved in the sweep direction), so bonds grow from the
 * initial state up to D.  Convergence as findGroundState: |E_old - E_new| <
 * convtol |E + offset| at the chain ends.  max_discarded (nullable): the
 * largest relative discarded weight sum_{i>=K} s_i^2 / sum s_i^2 of any cut
 * in the run.  init is overwritten with the result (normalised). */
mpsgpu_status mpsgpu_find_ground_state_two_site(mpsgpu_context* ctx, const mpsgpu_mpo* ops,
                                                int D, double offset,
                                                const mpsgpu_options* opt, mpsgpu_mps* init,
                                                double* lambda, double* max_discarded,
                                                mpsgpu_stats* stats);
/* findNextExcitedState(ops, D, levels, &lambda, init, offset)
 * (Contractor.cpp:2676-2727 -> findGroundStateWithProjectorPenalty :2739-2956). */
mpsgpu_status mpsgpu_find_next_excited_state(mpsgpu_context* ctx,
                                             const mpsgpu_mpo* ops, int D,
                                             const mpsgpu_mps* const* levels,
                                             int nlevels, double offset,
                                             const mpsgpu_options* opt,
                                             mpsgpu_mps* init, double* lambda,
                                             mpsgpu_stats* stats);
/* Batches of independent solves on one context, swept in lockstep: the local
 * eigenproblems of all solves at the same site share grouped launches of the
 * two contractions and of the Lanczos step (the reference runs one
 * findGroundState / findNextExcitedState after another; the result of each
 * solve is the one it has alone).  ops[i], inits[i]: solve i (all with the
 * same length; inits are overwritten by the results); lambdas[i] its energy;
 * status[i] (may be null) its own status, stats[i] (may be null) its
 * counters.  The call returns the first failing solve's status, MPSGPU_OK
 * when all succeed.  Excited states: solve i projects out the nlevels[i]
 * states that follow in `levels` (the lists of all solves concatenated). */
mpsgpu_status mpsgpu_find_ground_state_batch(mpsgpu_context* ctx, int n, const mpsgpu_mpo* const* ops, int D,
                                             double offset, const mpsgpu_options* opt, mpsgpu_mps* const* inits,
                                             double* lambdas, int* status, mpsgpu_stats* stats);
mpsgpu_status mpsgpu_find_next_excited_state_batch(mpsgpu_context* ctx, int n, const mpsgpu_mpo* const* ops, int D,
                                                   const mpsgpu_mps* const* levels, const int* nlevels,
                                                   double offset, const mpsgpu_options* opt,
                                                   mpsgpu_mps* const* inits, double* lambdas, int* status,
                                                   mpsgpu_stats* stats);
/* optimize(ops, orig, init, D, errN, errT) (Contractor.cpp:77-278): the
 * variational MPO.MPS product used for time evolution.  errN (nullable)
 * receives <orig|ops^dag ops|orig> + <init|init> - 2 Re <init|ops|orig> and
 * errT (used only with errN) the first term (Contractor.cpp:263-276). */
mpsgpu_status mpsgpu_optimize(mpsgpu_context* ctx, const mpsgpu_mpo* ops,
                              const mpsgpu_mps* orig, mpsgpu_mps* init, int D,
                              const mpsgpu_options* opt, double* errN,
                              double* errT, mpsgpu_stats* stats);
/* Contractor::optimizeSum (Contractor.cpp:2332-2477): init becomes the best
 * MPS of bond D approximating sum_k beta_k |kets[k]>; beta holds n complex
 * coefficients as (re, im) pairs.  Convergence by opt->convtol on the
 * distance, as optimize.  Replaces the reference's random perturbation of an
 * init without overlap (:2395-2405) by MPSGPU_INVALID. */
mpsgpu_status mpsgpu_optimize_sum(mpsgpu_context* ctx, int n, const mpsgpu_mps* const* kets,
                                  const double* beta, mpsgpu_mps* init, int D,
                                  const mpsgpu_options* opt, mpsgpu_stats* stats);
/* Contractor::optimizeMPS (Contractor.cpp:2319-2329): optimizeSum of one ket
 * with beta = 1; err (may be null) = <ket|ket> + <init|init> - 2 Re <init|ket>. */
mpsgpu_status mpsgpu_optimize_mps(mpsgpu_context* ctx, const mpsgpu_mps* ket, mpsgpu_mps* init,
                                  int D, const mpsgpu_options* opt, double* err,
                                  mpsgpu_stats* stats);
/* contract(ket, ops, bra) = <bra|ops|ket> (Contractor.cpp:528-556); ops may be
 * null for contract(ket, bra) (Contractor.cpp:467-499). */
mpsgpu_status mpsgpu_contract(mpsgpu_context* ctx, const mpsgpu_mps* ket,
                              const mpsgpu_mpo* ops, const mpsgpu_mps* bra,
                              double* re, double* im);
/* contract2(bra, ops, ket) = <bra|ops^dag ops|ket> (Contractor.cpp:634-718);
 * bra may be null for contract2(ops, ket) = <ket|ops^dag ops|ket>. */
mpsgpu_status mpsgpu_contract2(mpsgpu_context* ctx, const mpsgpu_mpo* ops,
                               const mpsgpu_mps* ket, const mpsgpu_mps* bra,
                               double* re, double* im);
/* <op_k> / <psi|psi> for every site k, op a d x d column-major matrix
 * (programs/banulsm/curved/flatIsing.cpp:258-282). out has L entries. */
mpsgpu_status mpsgpu_expectation_local(mpsgpu_context* ctx, const mpsgpu_mps* mps,
                                       const double* op, double* out);
/* getEntropy(state, pos) (Contractor.cpp:2045-2076). */
mpsgpu_status mpsgpu_entropy(mpsgpu_context* ctx, const mpsgpu_mps* mps, int pos,
                             double* entropy);
/* getSchmidtValues(state, lambdas, pos) (Contractor.cpp:2243-2270); writes at
 * most cap values (ascending), the count into *n. */
mpsgpu_status mpsgpu_schmidt_values(mpsgpu_context* ctx, const mpsgpu_mps* mps,
                                    int pos, double* values, int cap, int* n);

/* ---- solve server (continuous batching of independent requests) ---------
 * Requests are ground-state solves of model chains or time evolutions of
 * Ising chains.  The server owns `slots` worker threads, each with its own
 * context (CUDA stream); a request starts when a slot is free and its HBM
 * footprint fits in what the running requests leave of `hbm_budget_bytes`.
 * Admission is first fit in arrival order: the oldest queued request that
 * fits starts, so one large request does not hold free slots idle, and a
 * request that has been passed over 32 times is admitted before any later
 * one (no starvation).  Requests that arrive while others run are admitted
 * as slots and memory free up, and their device work overlaps.  State (MPO,
 * MPS, environments, Lanczos basis) stays on the device for the whole
 * request; the final state can be written to a file. */
typedef struct mpsgpu_server mpsgpu_server;

typedef enum { MPSGPU_MODEL_ISING = 0, MPSGPU_MODEL_SCHWINGER = 1 } mpsgpu_model;
typedef enum { MPSGPU_REQUEST_GROUND_STATE = 0, MPSGPU_REQUEST_TIME_EVOLUTION = 1 } mpsgpu_request_kind;

typedef struct {
  int model;         /* mpsgpu_model */
  int L;             /* sites */
  int D;             /* bond dimension (the maximum for a time evolution) */
  double p0, p1, p2; /* Ising: J, g, h.  Schwinger: mu, x, alpha (l0 = 0) */
  uint64_t seed;     /* initial MPS: mpsgpu_mps_random_state(L, 2, D, seed) */
  double convtol;    /* 0 = 1e-10 */
  int precision;     /* mpsgpu_options.precision: 0 FP64, 1 mixed */
  /* ---- fields below: zero-initialise for a ground-state request ---- */
  int kind;          /* mpsgpu_request_kind */
  /* Time evolution (Ising only): `steps` steps of the second-order Trotter
   * MPO of IsingHamiltonian::getUMPO (IsingHamiltonian.cpp:131-148) with
   * time step dt, imaginary time when imag != 0, each applied by
   * Contractor::optimize at bond D (Contractor.cpp:77-278), starting from
   * the product state |0...0> (seed unused).  After every step
   * obs_sx[step] = <sigma_x> on site L/2 and obs_entropy[step] = the
   * entropy of the bond L/2 when those caller-owned arrays (length steps)
   * are non-null; they must stay valid until the result is polled.  The
   * result's energy is <H> of the final state. */
  int steps;
  double dt;
  int imag;
  double* obs_sx;
  double* obs_entropy;
  /* Non-null: the final state is written there (reference binary MPS format,
   * MPS::exportMPS) before the result is reported; copied at submission. */
  const char* result_file;
} mpsgpu_request;

typedef struct {
  uint64_t id;
  int status;                /* mpsgpu_status */
  double energy;
  int rounds;
  long long matvecs;
  double flops;
  double t_submit, t_start, t_end;  /* seconds since the server was created */
  long long footprint_bytes;
} mpsgpu_result;

mpsgpu_status mpsgpu_server_create(int device, int slots, long long hbm_budget_bytes,
                                   mpsgpu_server** out);
mpsgpu_status mpsgpu_server_submit(mpsgpu_server* srv, const mpsgpu_request* req, uint64_t* id);
/* Moves up to cap finished results into out (in completion order). */
mpsgpu_status mpsgpu_server_poll(mpsgpu_server* srv, mpsgpu_result* out, int cap, int* n);
/* Cancels a queued request, or stops a running one between two site steps. */
mpsgpu_status mpsgpu_server_cancel(mpsgpu_server* srv, uint64_t id);
/* Waits until no request is queued or running (timeout_s <= 0: no limit). */
mpsgpu_status mpsgpu_server_drain(mpsgpu_server* srv, double timeout_s);
/* Estimated device footprint of a request (the admission criterion). */
long long mpsgpu_request_footprint(const mpsgpu_request* req);
mpsgpu_status mpsgpu_server_destroy(mpsgpu_server* srv);

/* ---- kernel-level entry points (host buffers, reference layouts) ---------
 * TensorMultiplier(Offset)::product (TensorMultiplier.cpp:61-93,
 * TensorMultiplierOffset.cpp:14-17); hermitian!=0 gives
 * TensorMultiplierHermitian(Offset)::product (TensorMultiplierHermitian.cpp:37-70).
 * ldims = (Dlb, wl, Dlk), wdims = (du, wl, dd, wr), rdims = (Drb, wr, Drk);
 * x has dd*Dlk*Drk entries, y gets du*Dlb*Drb. */
mpsgpu_status mpsgpu_heff_matvec(mpsgpu_context* ctx, const int* ldims,
                                 const double* L, const int* wdims,
                                 const double* W, const int* rdims,
                                 const double* R, const double* x, double* y,
                                 double offset, int hermitian);
/* Grouped matvec over many independent instances (the batched form of
 * TensorMultiplier::product), all operands already on the device in the
 * library's layouts:
 *   L  (Dl, wl, Dl)  left environment (bra, w, ket), as the reference stores it
 *   W  (d, wl, d, wr) MPO tensor, as the reference stores it
 *   Rt (Dr, wr, Dr)  right environment in (ket, w, bra) order
 *   x, y (Dl, d, Dr) site vector with the left bond fastest
 * The three grouped launches (GEMM, MPO-leg contraction, GEMM) run once; with
 * repeats > 0 they are captured in a CUDA graph and replayed `repeats` times,
 * and *ms_per_run gets the device time per product (CUDA events).  *flops
 * gets the algorithmic flops of one grouped product. */
typedef struct {
  int d, wl, wr, Dl, Dr;
  const double* L;
  const double* W;
  const double* Rt;
  const double* x;
  double* y;
} mpsgpu_heff_instance;
mpsgpu_status mpsgpu_heff_matvec_grouped(mpsgpu_context* ctx, int n, const mpsgpu_heff_instance* inst,
                                         int repeats, double* ms_per_run, double* flops);
/* The same with a precision choice: 0 = complex FP64 (as above); 1 = split
 * precision, both GEMMs of every instance on the tcgen05 tensor cores with
 * BF16 limbs (about 1e-7 relative error).  In split precision the limb
 * planes of L and Rt are made once before the products (the environments
 * of an eigensolve do not change between its products); *ms_prepare gets
 * that device time, and every product prepares x and the intermediate. */
mpsgpu_status mpsgpu_heff_matvec_grouped_ex(mpsgpu_context* ctx, int n, const mpsgpu_heff_instance* inst,
                                            int precision, int repeats, double* ms_per_run, double* flops,
                                            double* ms_prepare);

/* Autotuner of the complex FP64 GEMM's launch configuration (tile edge
 * 32 or 64, 1 to 16 K slices), and of the K chunks (1-4 and 1-8) of the two
 * tcgen05 products of a lockstep round's split-precision products.  The
 * first GEMM of each shape (M, N, K, batch, ops, epilogue), and the first
 * round of each shape signature (every product's dimensions), times every
 * candidate on its own operands and the fastest is used from then on, for
 * all contexts of the process; no tuning while a stream is captured into a
 * graph.  On by default (MPSGPU_AUTOTUNE=0 in the environment turns it off
 * before the first GEMM); results of different configurations differ only
 * by the order of the K-slice sums.  entries = shapes tuned so far. */
void mpsgpu_set_autotune(int on);
long long mpsgpu_autotune_entries(void);

/* Split-precision complex GEMM C = A B (column-major, complex interleaved,
 * host buffers; m x k times k x n) on the tcgen05 tensor cores: every FP64
 * real is split into three BF16 limbs and the limb products with combined
 * order <= 2 are accumulated in FP32, so C carries about 1e-7 relative error
 * of |A||B| entrywise.  No counterpart in the reference (which multiplies in
 * complex FP64 through zgemm, wrapper.cpp); it is the product the
 * split-precision sweep mode runs on.  With repeats > 0, *ms_total gets the
 * device time of operand preparation plus product and *ms_mma the product
 * alone, each averaged over `repeats` runs. */
mpsgpu_status mpsgpu_zgemm_split(mpsgpu_context* ctx, int m, int n, int k, const double* A, int lda,
                                 const double* B, int ldb, double* C, int ldc, int repeats,
                                 double* ms_total, double* ms_mma);

/* Operator::contractL / contractR (Operator.cpp:273-398): out gets
 * (Dr_bra, wr, Dr_ket) resp. (Dl_bra, wl, Dl_ket). */
mpsgpu_status mpsgpu_env_left(mpsgpu_context* ctx, const int* tdims,
                              const double* T, const int* kdims,
                              const double* ket, const int* wdims,
                              const double* W, const int* bdims,
                              const double* bra, double* out);
mpsgpu_status mpsgpu_env_right(mpsgpu_context* ctx, const int* tdims,
                               const double* T, const int* kdims,
                               const double* ket, const int* wdims,
                               const double* W, const int* bdims,
                               const double* bra, double* out);
/* wrapper::qr / wrapper::lq (src/wrapper/qr.cpp:33-188): Householder with
 * the LAPACK zgeqrf/zungqr conventions; K = min(m, n); Q is m x K and R is
 * K x n (qr), L is m x K and Q is K x n (lq). */
mpsgpu_status mpsgpu_qr(mpsgpu_context* ctx, int m, int n, const double* A,
                        double* Q, double* R);
mpsgpu_status mpsgpu_lq(mpsgpu_context* ctx, int m, int n, const double* A,
                        double* Lf, double* Q);

/* QR of a device-resident m x n matrix that allocates nothing.  No
 * counterpart in the reference: it is a variant of mpsgpu_qr for callers that
 * cannot allocate device memory when they need a gauge move (a serving
 * process whose allocator owns the whole HBM, a loop that must not fail on
 * an allocation half way through a sweep).
 *   A: m x n column-major complex128 on the device (read only);
 *   Q: m x K (ld m), R: K x n (ld K), K = min(m, n), on the device; either may
 *      be null.  Same results as mpsgpu_qr (LAPACK zgeqrf/zungqr conventions).
 *   stream: the cudaStream_t to run on (null = default stream); the call is
 *      asynchronous on it and returns after enqueueing.
 * Limit: m, n <= 640 and m*n <= 131072; larger sizes return MPSGPU_BAD_SHAPE.
 * Working memory is one fixed 2.1 MiB device array inside the library.  CUDA
 * places it on a GPU when the library's code is first loaded there:
 * mpsgpu_create does that for its device (so create a context on the GPU,
 * while allocation is still allowed, before relying on this call); it is then
 * held until the process exits.  The first call on a device also looks up the
 * array's address (cudaGetSymbolAddress) unless a context did it already:
 * make that first call before any stream capture.  All calls share the
 * array, so calls that overlap on the GPU (different streams, or concurrent
 * host threads) race; serialise them on one stream. */
mpsgpu_status mpsgpu_qr_device_noalloc(int m, int n, const double* A, double* Q,
                                       double* R, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MPSGPU_H */
