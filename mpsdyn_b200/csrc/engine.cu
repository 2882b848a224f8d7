// Sweep engine: the reference Contractor's single-site algorithms
// (src/core/cpp/Contractor.cpp) on device-resident tensors.
//
// Device layout of a site tensor: X(a, s, r) with the left bond fastest, so
// that the first GEMM of every contraction reads it as a plain (Dl x d*Dr)
// matrix.  Left environments are stored as the reference stores them,
// L(bra, w, ket); right environments transposed, Rt(ket, w, bra), so that the
// last GEMM of the matvec reads them as a plain ((Dr*w) x Dr) matrix.  With
// these layouts every step of
//   y[s',a',r'] = sum L[a',b,a] W[s',b,s,c] R[r',c,r] x[s,a,r]
// is one GEMM or one MPO-leg contraction; none of the explicit permutes of
// TensorMultiplier::product (TensorMultiplier.cpp:61-93) remain.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"
#include "tridiag.h"

namespace mpsgpu {

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------

void dbuf_reserve(Context& c, DBuf& b, long long n) {
  if (n <= b.cap) return;
  if (b.p) MPSGPU_CUDA(cudaFreeAsync(b.p, c.stream));
  b.p = nullptr;
  b.cap = 0;
  long long nn = std::max<long long>(n, 1);
  MPSGPU_CUDA(cudaMallocAsync((void**)&b.p, nn * sizeof(cplx), c.stream));
  b.cap = nn;
}

void dbuf_free(Context& c, DBuf& b) {
  if (b.p) cudaFreeAsync(b.p, c.stream);
  b.p = nullptr;
  b.cap = 0;
}

int MpsDev::max_bond() const {
  int m = 1;
  for (auto& d : dims) m = std::max(m, std::max(d[1], d[2]));
  return m;
}

static inline long long nel(const std::array<int, 3>& d) { return (long long)d[0] * d[1] * d[2]; }

// ---------------------------------------------------------------------------
// MPO upload: reference tensors plus the small leg matrices of each operator
// ---------------------------------------------------------------------------

void mpo_upload(Context& c, MpoDev& m, int L, const int* dims, const double* const* data,
                bool check_edges) {
  MPSGPU_CHECK(L >= 1, MPSGPU_BAD_SHAPE, "mpo: L < 1");
  m.L = L;
  m.dims.resize(L);
  m.W.assign(L, DBuf());
  m.Wlr.assign(L, DBuf());
  m.Wrl.assign(L, DBuf());
  m.Wlr_h.assign(L, DBuf());
  m.Wrl_h.assign(L, DBuf());
  for (int k = 0; k < L; k++) {
    const int du = dims[4 * k], wl = dims[4 * k + 1], dd = dims[4 * k + 2], wr = dims[4 * k + 3];
    MPSGPU_CHECK(du > 0 && wl > 0 && dd > 0 && wr > 0, MPSGPU_BAD_SHAPE, "mpo: non-positive dimension");
    MPSGPU_CHECK(du * wr <= 64 && wl * dd <= 64 && wl * du <= 64 && dd * wr <= 64, MPSGPU_BAD_SHAPE,
                 "mpo: d*w must not exceed 64");
    if (k > 0) MPSGPU_CHECK(m.dims[k - 1][3] == wl, MPSGPU_BAD_SHAPE, "mpo: bond mismatch");
    m.dims[k] = {du, wl, dd, wr};
    const long long n = (long long)du * wl * dd * wr;
    const cplx* W = reinterpret_cast<const cplx*>(data[k]);
    auto at = [&](int sp, int b, int s, int cc) { return W[sp + du * (b + wl * (s + dd * cc))]; };
    std::vector<cplx> lr(n), rl(n), lrh(n), rlh(n);
    const int nout_lr = du * wr, nout_rl = wl * du;
    for (int sp = 0; sp < du; sp++)
      for (int b = 0; b < wl; b++)
        for (int s = 0; s < dd; s++)
          for (int cc = 0; cc < wr; cc++) {
            cplx w = at(sp, b, s, cc);
            lr[(sp + du * cc) + (long long)nout_lr * (b + wl * s)] = w;
            rl[(b + wl * sp) + (long long)nout_rl * (s + dd * cc)] = w;
            if (du == dd) {
              // adjoint operator W^dag[s', b, s, c] = conj(W[s, b, s', c])
              cplx wa = at(s, b, sp, cc);
              wa.y = -wa.y;
              lrh[(sp + du * cc) + (long long)nout_lr * (b + wl * s)] = wa;
              rlh[(b + wl * sp) + (long long)nout_rl * (s + dd * cc)] = wa;
            }
          }
    dbuf_reserve(c, m.W[k], n);
    dbuf_reserve(c, m.Wlr[k], n);
    dbuf_reserve(c, m.Wrl[k], n);
    MPSGPU_CUDA(cudaMemcpyAsync(m.W[k].p, W, n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
    MPSGPU_CUDA(cudaMemcpyAsync(m.Wlr[k].p, lr.data(), n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
    MPSGPU_CUDA(cudaMemcpyAsync(m.Wrl[k].p, rl.data(), n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
    if (du == dd) {
      dbuf_reserve(c, m.Wlr_h[k], n);
      dbuf_reserve(c, m.Wrl_h[k], n);
      MPSGPU_CUDA(cudaMemcpyAsync(m.Wlr_h[k].p, lrh.data(), n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
      MPSGPU_CUDA(cudaMemcpyAsync(m.Wrl_h[k].p, rlh.data(), n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
    }
    // host vectors must outlive the async copies
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  }
  if (check_edges)
    MPSGPU_CHECK(m.dims[0][1] == 1 && m.dims[L - 1][3] == 1, MPSGPU_BAD_SHAPE,
                 "mpo: edge bonds must be 1");
}

void mpo_free(Context& c, MpoDev& m) {
  for (auto* v : {&m.W, &m.Wlr, &m.Wrl, &m.Wlr_h, &m.Wrl_h})
    for (auto& b : *v) dbuf_free(c, b);
  m.L = 0;
}

// ---------------------------------------------------------------------------
// MPS storage
// ---------------------------------------------------------------------------

void mps_upload(Context& c, MpsDev& s, int L, const int* dims, const double* const* data, double nf) {
  MPSGPU_CHECK(L >= 1, MPSGPU_BAD_SHAPE, "mps: L < 1");
  s.L = L;
  s.dims.resize(L);
  s.A.resize(L);
  long long maxn = 0;
  for (int k = 0; k < L; k++) {
    s.dims[k] = {dims[3 * k], dims[3 * k + 1], dims[3 * k + 2]};
    MPSGPU_CHECK(s.dims[k][0] > 0 && s.dims[k][1] > 0 && s.dims[k][2] > 0, MPSGPU_BAD_SHAPE,
                 "mps: non-positive dimension");
    if (k > 0) MPSGPU_CHECK(s.dims[k - 1][2] == s.dims[k][1], MPSGPU_BAD_SHAPE, "mps: bond mismatch");
    maxn = std::max(maxn, nel(s.dims[k]));
  }
  MPSGPU_CHECK(s.dims[0][1] == 1 && s.dims[L - 1][2] == 1, MPSGPU_BAD_SHAPE, "mps: edge bonds must be 1");
  dbuf_reserve(c, c.t1, maxn);
  for (int k = 0; k < L; k++) {
    long long n = nel(s.dims[k]);
    dbuf_reserve(c, s.A[k], n);
    MPSGPU_CUDA(cudaMemcpyAsync(c.t1.p, data[k], n * sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
    site_ref_to_dev(c.st(), s.dims[k][0], s.dims[k][1], s.dims[k][2], c.t1.p, s.A[k].p);
  }
  s.normfact = nf;
  s.gauge = 0;
  s.bond = s.max_bond();
}

void mps_random(Context& c, MpsDev& s, int L, int d, int D, uint64_t seed) {
  MPSGPU_CHECK(L >= 2 && d >= 1 && D >= 1, MPSGPU_BAD_SHAPE, "mps_random: bad sizes");
  s.L = L;
  s.dims.resize(L);
  s.A.resize(L);
  std::vector<int> bonds(L + 1);
  for (int k = 0; k <= L; k++) {
    double lk = std::min(k, L - k) * std::log((double)d);
    bonds[k] = lk > std::log((double)D) ? D : std::min<long long>(D, (long long)std::llround(std::pow((double)d, std::min(k, L - k))));
  }
  long long off = 0;
  for (int k = 0; k < L; k++) {
    s.dims[k] = {d, bonds[k], bonds[k + 1]};
    dbuf_reserve(c, s.A[k], nel(s.dims[k]));
    gaussian_site(c.st(), seed, off, d, bonds[k], bonds[k + 1], s.A[k].p);
    off += nel(s.dims[k]);
  }
  s.normfact = 1.0;
  s.gauge = 0;
  s.bond = s.max_bond();
}

// MPS::setRandomState (src/core/cpp/MPS.cpp:282-294): random sites, each
// right-gauged in turn; the R factor moves on only where the bond shrinks,
// so the state is a chain of random isometries with norm 1 whatever L.
void mps_random_state(Context& c, MpsDev& s, int L, int d, int D, uint64_t seed) {
  mps_random(c, s, L, d, D, seed);
  for (int k = 0; k < L; k++) mps_gauge_site(c, s, k, 'R', false, nullptr);
  s.normfact = 1.0;
  s.gauge = 2;
}

void mps_product(Context& c, MpsDev& s, int L, int d, int D) {
  s.L = L;
  s.dims.resize(L);
  s.A.resize(L);
  for (int k = 0; k < L; k++) {
    int dl = k == 0 ? 1 : D, dr = k == L - 1 ? 1 : D;
    s.dims[k] = {d, dl, dr};
    dbuf_reserve(c, s.A[k], nel(s.dims[k]));
    zfill(c.st(), nel(s.dims[k]), make_double2(0.0, 0.0), s.A[k].p);
    cplx one = make_double2(1.0, 0.0);
    MPSGPU_CUDA(cudaMemcpyAsync(s.A[k].p, &one, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
  }
  MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  s.normfact = 1.0;
  s.gauge = 0;
  s.bond = D;
}

void mps_copy(Context& c, const MpsDev& src, MpsDev& dst) {
  if (&src == &dst) return;
  dst.L = src.L;
  dst.dims = src.dims;
  dst.A.resize(src.L);
  for (int k = 0; k < src.L; k++) {
    dbuf_reserve(c, dst.A[k], nel(src.dims[k]));
    zcopy(c.st(), (int)nel(src.dims[k]), src.A[k].p, dst.A[k].p);
  }
  dst.normfact = src.normfact;
  dst.gauge = src.gauge;
  dst.bond = src.bond;
}

void mps_download(Context& c, const MpsDev& s, double* const* data) {
  long long maxn = 0;
  for (int k = 0; k < s.L; k++) maxn = std::max(maxn, nel(s.dims[k]));
  dbuf_reserve(c, c.t1, maxn);
  for (int k = 0; k < s.L; k++) {
    long long n = nel(s.dims[k]);
    site_dev_to_ref(c.st(), s.dims[k][0], s.dims[k][1], s.dims[k][2], s.A[k].p, c.t1.p);
    MPSGPU_CUDA(cudaMemcpyAsync(data[k], c.t1.p, n * sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  }
}

void mps_free(Context& c, MpsDev& s) {
  for (auto& b : s.A) dbuf_free(c, b);
  s.A.clear();
  s.dims.clear();
  s.L = 0;
}

// ---------------------------------------------------------------------------
// Gauge moves (Site::gaugeR / gaugeL, src/core/cpp/Site.cpp:179-283;
// MPS::gaugeCond, src/core/cpp/MPS.cpp:306-419)
// ---------------------------------------------------------------------------

// Move the norm of site pos into a factor: dir 'R' -> site = Q (left
// isometry), factor R (K x Dr) left in c.matR (ld K); dir 'L' -> site = Q^H
// rows (right isometry), factor R' (K x Dl) with L = R'^H.  Returns K.
// cutD > 0 replaces the QR by the SVD cut of Site::gaugeR/gaugeL with cutD
// (Site.cpp:186-193, :218-224): Q = U[:, :K], R = diag(s) V^H, K = the
// number of values > 0 among the cutD largest; the sum of the squares of
// the dropped values is added to *disc.
static int site_factor(Context& c, MpsDev& s, int pos, char dir, cplx* r00, int cutD = 0,
                       double* disc = nullptr) {
  const int d = s.dims[pos][0], Dl = s.dims[pos][1], Dr = s.dims[pos][2];
  int m, n;
  View2 v;
  if (dir == 'R') {
    m = d * Dl; n = Dr;
    // row i = s + d a  (reference order), column r
    v.rd = d; v.r0 = Dl; v.r1 = 1; v.cd = 1; v.c0 = 0; v.c1 = (long long)Dl * d;
  } else {
    // QR of M^H, M = X viewed as (Dl x d*Dr): B(i, j) = conj(X[j + Dl i])
    m = d * Dr; n = Dl;
    v.rd = 1; v.r0 = 0; v.r1 = Dl; v.cd = 1; v.c0 = 0; v.c1 = 1; v.conj = true;
  }
  int K = std::min(m, n);
  dbuf_reserve(c, c.matA, (long long)m * n);
  dbuf_reserve(c, c.matQ, (long long)m * K);
  dbuf_reserve(c, c.matR, (long long)K * n);
  gather2(c.st(), m, n, s.A[pos].p, v, c.matA.p);
  if (cutD > 0) {
    std::vector<double> sv;
    K = svd_cut(c.st(), m, n, c.matA.p, m, cutD, c.matQ.p, c.matR.p, sv, c.scratch);
    if (disc)
      for (size_t j = K; j < sv.size(); j++) *disc += sv[j] * sv[j];
  } else {
    householder_qr_inplace(c.st(), m, n, c.matA.p, c.matQ.p, m, c.matR.p, K, c.qrws);
  }
  // write the isometry back into the site
  View2 w;
  if (dir == 'R') {
    s.dims[pos] = {d, Dl, K};
    w.rd = d; w.r0 = Dl; w.r1 = 1; w.cd = 1; w.c0 = 0; w.c1 = (long long)Dl * d;
  } else {
    s.dims[pos] = {d, K, Dr};
    // site X'(k, s, r) at k + K (s + d r) = conj(Q'(c = s + d r, k))
    w.rd = 1; w.r0 = 0; w.r1 = K; w.cd = 1; w.c0 = 0; w.c1 = 1; w.conj = true;
  }
  scatter2(c.st(), m, K, c.matQ.p, s.A[pos].p, w);
  if (r00 && K == 1 && n == 1) {
    MPSGPU_CUDA(cudaMemcpyAsync(r00, c.matR.p, sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  }
  return K;
}

// Single-element phase handling of Site::gaugeR/gaugeL on the last/first site.
static double edge_phase(Context& c, MpsDev& s, int pos, char dir, cplx aux) {
  double a = std::sqrt(cabs2(aux));
  if (dir == 'L') aux.y = -aux.y;  // L = R'^H
  cplx phase = a > 0 ? make_double2(aux.x / a, aux.y / a) : make_double2(1.0, 0.0);
  zaxpby(c.st(), (int)nel(s.dims[pos]), phase, s.A[pos].p, make_double2(0.0, 0.0), s.A[pos].p);
  return a;
}

// A_next <- R * A_next on its left bond (Site::reduceDimR); A_prev <- A_prev * L
// on its right bond (Site::reduceDimL) with L = R'^H.
static void absorb(Context& c, MpsDev& s, int target, char dir, int K, int n) {
  const int d = s.dims[target][0], Dl = s.dims[target][1], Dr = s.dims[target][2];
  GemmArgs g;
  if (dir == 'R') {
    MPSGPU_CHECK(Dl == n, MPSGPU_BAD_SHAPE, "absorb R: bond mismatch");
    dbuf_reserve(c, c.t3, (long long)K * d * Dr);
    g.M = K; g.N = d * Dr; g.K = Dl;
    g.A = c.matR.p; g.lda = K; g.opA = OP_N;
    g.B = s.A[target].p; g.ldb = Dl; g.opB = OP_N;
    g.C = c.t3.p; g.ldc = K;
    zgemm(c.st(), g, c.scratch);
    s.dims[target] = {d, K, Dr};
  } else {
    MPSGPU_CHECK(Dr == n, MPSGPU_BAD_SHAPE, "absorb L: bond mismatch");
    dbuf_reserve(c, c.t3, (long long)Dl * d * K);
    g.M = Dl * d; g.N = K; g.K = Dr;
    g.A = s.A[target].p; g.lda = (long long)Dl * d; g.opA = OP_N;
    g.B = c.matR.p; g.ldb = K; g.opB = OP_C;  // (R')^H : Dr x K
    g.C = c.t3.p; g.ldc = (long long)Dl * d;
    zgemm(c.st(), g, c.scratch);
    s.dims[target] = {d, Dl, K};
  }
  dbuf_reserve(c, s.A[target], nel(s.dims[target]));
  zcopy(c.st(), (int)nel(s.dims[target]), c.t3.p, s.A[target].p);
}

// QR/LQ of site pos; when the factor is the 1x1 of a bond of dimension 1
// the phase goes into the site and |factor| is returned (else -1, factor
// left in c.matR).  Site::gaugeR / gaugeL, Site.cpp:199-207 and :229-237.
static int gauge_factor(Context& c, MpsDev& s, int pos, char dir, double* scalar, Counters* cnt, int cutD = 0,
                        double* disc = nullptr) {
  const auto old = s.dims[pos];
  const int n = dir == 'R' ? old[2] : old[1];
  cplx r00 = make_double2(0.0, 0.0);
  const int K = site_factor(c, s, pos, dir, &r00, cutD, disc);
  *scalar = -1.0;
  if (K == 1 && n == 1) *scalar = edge_phase(c, s, pos, dir, r00);
  if (cnt) {
    cnt->qr_calls++;
    const double m = dir == 'R' ? (double)old[0] * old[1] : (double)old[0] * old[2];
    const double kk = K;
    cnt->flops += 8.0 * 2.0 * (2.0 * m * n * kk - (m + n) * kk * kk + 2.0 * kk * kk * kk / 3.0);
  }
  return K;
}

// Site::reduceDimR / reduceDimL with the factor of gauge_factor.
static void pass_factor(Context& c, MpsDev& s, int target, char dir, int K, int n, double scalar) {
  if (scalar >= 0.0) {
    zaxpby(c.st(), (int)nel(s.dims[target]), make_double2(scalar, 0.0), s.A[target].p,
           make_double2(0.0, 0.0), s.A[target].p);
  } else {
    absorb(c, s, target, dir, K, n);
  }
}

// MPS::gaugeCond(pos, dir, next) (MPS.cpp:366-419).
void mps_gauge_site(Context& c, MpsDev& s, int pos, char dir, bool next, Counters* cnt) {
  const auto old = s.dims[pos];
  const int n = dir == 'R' ? old[2] : old[1];
  double scalar = -1.0;
  const int K = gauge_factor(c, s, pos, dir, &scalar, cnt);
  if (dir == 'L') {
    if ((s.dims[pos][1] != old[1] || next) && pos > 0) pass_factor(c, s, pos - 1, 'L', K, n, scalar);
    if (pos == 0 && next) {
      MPSGPU_CHECK(scalar >= 0.0, MPSGPU_BAD_SHAPE, "gaugeL on site 0: factor is not a scalar");
      s.normfact *= scalar;
    }
  } else {
    if (pos < s.L - 1 && (s.dims[pos][2] != old[2] || next)) pass_factor(c, s, pos + 1, 'R', K, n, scalar);
    if (next && pos == s.L - 1) {
      MPSGPU_CHECK(scalar >= 0.0, MPSGPU_BAD_SHAPE, "gaugeR on the last site: factor is not a scalar");
      s.normfact *= scalar;
    }
  }
  s.gauge = 0;
}

// MPS::gaugeCond(dir, normal, cutD) (MPS.cpp:306-364): a full QR (or LQ)
// sweep carrying the factor along, or with cutD > 0 an SVD sweep that cuts
// every bond to at most cutD; the final scalar becomes the norm factor.
void mps_gauge_all(Context& c, MpsDev& s, char dir, bool normal, int cutD, double* disc) {
  double last = 1.0;
  if (dir == 'R') {
    for (int pos = 0; pos < s.L; pos++) {
      const int n = s.dims[pos][2];
      double scalar = -1.0;
      const int K = gauge_factor(c, s, pos, 'R', &scalar, nullptr, cutD, disc);
      if (pos < s.L - 1) pass_factor(c, s, pos + 1, 'R', K, n, scalar);
      else last = scalar;
    }
    s.gauge = 2;
  } else {
    for (int pos = s.L - 1; pos >= 0; pos--) {
      const int n = s.dims[pos][1];
      double scalar = -1.0;
      const int K = gauge_factor(c, s, pos, 'L', &scalar, nullptr, cutD, disc);
      if (pos > 0) pass_factor(c, s, pos - 1, 'L', K, n, scalar);
      else last = scalar;
    }
    s.gauge = 1;
  }
  s.bond = std::min(s.bond > 0 ? s.bond : 1 << 30, s.max_bond());
  if (normal) s.normfact = 1.0;
  else s.normfact *= last;
}

// MPS::increaseBondDimensionWithNoise(D, 0) (MPS.cpp:654-719): integer bond
// schedule, zero padding of every site.
void mps_increase_bond(Context& c, MpsDev& s, int D) {
  if (D <= s.bond) return;
  const int L = s.L;
  long long cumd = 1, cumdr_last = 1;
  int boundR = L - 1;
  bool done = false;
  while (!done && boundR > 0) {
    int dim = s.dims[boundR][0];
    if (cumdr_last * dim < D) { boundR--; cumdr_last *= dim; }
    else done = true;
  }
  long long cumdr = boundR > 0 ? D : cumdr_last * s.dims[0][0];
  int maxbond = 1;
  for (int k = 0; k < L; k++) {
    auto old = s.dims[k];
    long long newDl, newDr;
    if (k == 0) newDl = old[1];
    else newDl = (cumd < D || cumdr < D) ? std::min(cumd, cumdr) : D;
    int posd = s.dims[k][0];
    if (cumd < D) cumd *= posd;
    if (k == boundR) cumdr = cumdr_last;
    else if (k > boundR) cumdr = cumdr / posd;
    if (k == L - 1) newDr = old[2];
    else newDr = (cumd < D || cumdr < D) ? std::min(cumd, cumdr) : D;
    std::array<int, 3> nd = {old[0], (int)newDl, (int)newDr};
    // zero-padded copy: X'(a, s, r) = X(a, s, r) inside the old box
    DBuf nb;
    dbuf_reserve(c, nb, nel(nd));
    zfill(c.st(), nel(nd), make_double2(0.0, 0.0), nb.p);
    const int m1 = std::min(old[1], nd[1]), m2 = std::min(old[2], nd[2]);
    // rows = (a, s) with a < m1, columns r < m2
    const int rows = m1 * old[0];
    View2 vi; vi.rd = m1; vi.r0 = 1; vi.r1 = old[1]; vi.cd = 1; vi.c0 = 0; vi.c1 = (long long)old[1] * old[0];
    View2 vo; vo.rd = m1; vo.r0 = 1; vo.r1 = nd[1]; vo.cd = 1; vo.c0 = 0; vo.c1 = (long long)nd[1] * nd[0];
    dbuf_reserve(c, c.t3, (long long)rows * m2);
    gather2(c.st(), rows, m2, s.A[k].p, vi, c.t3.p);
    scatter2(c.st(), rows, m2, c.t3.p, nb.p, vo);
    dbuf_free(c, s.A[k]);
    s.A[k] = nb;
    s.dims[k] = nd;
    maxbond = std::max(maxbond, (int)std::max(newDl, newDr));
  }
  s.bond = maxbond;
  s.gauge = 0;
}

// ---------------------------------------------------------------------------
// Contractions
// ---------------------------------------------------------------------------

static double mv_flops(int d, int w1, int w2, int dl, int dr) {
  // complex MACs of the three steps, 8 real flops each
  double a = (double)dl * w1 * dl * d * dr;       // L . X
  double b = (double)dl * d * d * w1 * w2 * dr;   // W
  double cc = (double)dl * d * dr * w2 * dr;      // . R
  return 8.0 * (a + b + cc);
}

// Mixed-precision sweep: the split phase ends at the first half-sweep whose
// energy change is below kSplitSwitchTol (relative); its Lanczos residual
// tolerance and energy-increase margin sit above the products' error.
constexpr double kSplitSwitchTol = 1e-6;
constexpr double kSplitEigTol = 1e-6;
// The first FP64 half-sweep after the split phase cannot end the solve (it is
// compared with a split-phase energy), so its site solves stop at a residual
// of 1e-9: the energy error is quadratic in the residual, and the half-sweeps
// that decide convergence run at the full tolerance.
constexpr double kFirst64EigTol = 1e-9;
// The schedule forms (precision 1 and 2) end at an eigensolver residual of
// 1e-9 of the spectrum's scale instead of the reference's 1e-12: an energy
// error is quadratic in the residual, (1e-9 |theta|)^2 / gap, which for the
// headline chain (|theta| ~ 6e3, gap ~ 10) is 4e-12 absolute, 6e-16 relative,
// far inside the 1e-10 the solve converges to; measured on the headline
// workload the energies stay within 1e-13 of the reference's.
constexpr double kScheduleEigTol = 1e-9;
// Products per set of split-round launches.
constexpr int kSplitRoundMax = 16;
// optimize with split-precision local vectors: relative distance tolerance
// (its noise floor is the products' error)
constexpr double kSplitOptimizeTol = 1e-6;
constexpr double kSplitIncreaseTol = 1e-5;

static int device_sms(Context& c) {
  int v = 148;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, c.device) != cudaSuccess) v = 148;
  return v;
}

static uint8_t* bytes_reserve(Context& c, DBuf& b, long long bytes) {
  dbuf_reserve(c, b, (bytes + (long long)sizeof(cplx) - 1) / (long long)sizeof(cplx));
  return reinterpret_cast<uint8_t*>(b.p);
}

void split_matvec_prepare(Context& c, SplitMatvec& s, const cplx* Le, const std::array<int, 3>& ld,
                          const MpoDev& m, int k, const cplx* Rt, const std::array<int, 3>& rd) {
  const auto& wd = m.dims[k];
  const int wl = wd[1], wr = wd[3];
  const int Dlb = ld[0], Dlk = ld[2], Drk = rd[0], Drb = rd[2];
  const Stream st = c.st();
  // L as the A operand of T1 = L . X: rows Dlb*wl, inner Dlk, column-major
  split_prepare(st, Dlb * wl, Dlk, Le, 1, (long long)Dlb * wl, 128,
                bytes_reserve(c, s.Lp, split_operand_bytes(Dlb * wl, Dlk, 128)));
  // Rt as the B operand of Y = T2 . Rt: its columns (Drb) are the prepared rows
  split_prepare(st, Drb, Drk * wr, Rt, (long long)Drk * wr, 1, 128,
                bytes_reserve(c, s.Rp, split_operand_bytes(Drb, Drk * wr, 128)));
  s.ready = true;
}

// First contraction of the matvec: T2[a', s', r, c] = sum_{a,b,s} W[s',b,s,c]
// L[a',b,a] X[a,s,r] with L (Dlb, w, Dlk), X (Dlk, d, Drk) in device layout
// and T2 (Dlb, du, Drk, wr) (a' fastest), the operand of the last product.
Gemm1wDesc heff_first_desc(const cplx* Le, int Dlb, int Dlk, int wl, const cplx* x, int dd, int Drk, const cplx* Wm,
                           int du, int wr, cplx* t2) {
  Gemm1wDesc d;
  d.A = Le; d.lda = (long long)Dlb * wl;
  d.B = x; d.ldb = Dlk;
  d.X = Dlb; d.Y = Drk; d.K = Dlk;
  d.n_i0 = wl; d.n_i1 = dd; d.n_o0 = du; d.n_o1 = wr;
  d.Wm = Wm;
  d.out = t2; d.ox = 1; d.oy = (long long)Dlb * du; d.so0 = Dlb; d.so1 = (long long)Dlb * du * Drk;
  return d;
}

// Last contraction: Y[(a',s'), r'] = T2((Dlb du) x (Drk wr)) . Rt((Drk wr) x Drb) + offset X.
Gemm3Desc heff_last_desc(const cplx* t2, int M, const cplx* Rt, int K, int Drb, cplx* y, const cplx* x,
                         cplx offset) {
  Gemm3Desc d;
  d.M = M; d.N = Drb; d.K1 = K;
  d.A1 = t2; d.lda1 = M;
  d.B1 = Rt; d.ldb1 = K;
  d.C = y; d.ldc = M;
  if (offset.x != 0.0 || offset.y != 0.0) {
    d.Cin = x; d.ldcin = M; d.beta = offset;
  }
  return d;
}

void split_matvec_release(Context& c, SplitMatvec& s) {
  dbuf_free(c, s.Lp);
  dbuf_free(c, s.Rp);
  s.ready = false;
}

void heff_apply(Context& c, const cplx* Le, const std::array<int, 3>& ld, const MpoDev& m, int k,
                bool adjoint, const cplx* Rt, const std::array<int, 3>& rd, const cplx* x, cplx* y,
                cplx offset, Counters* cnt) {
  const auto& wd = m.dims[k];
  const int du = wd[0], wl = wd[1], dd = wd[2], wr = wd[3];
  const int Dlb = ld[0], Dlk = ld[2], Drk = rd[0], Drb = rd[2];
  MPSGPU_CHECK(ld[1] == wl && rd[1] == wr, MPSGPU_BAD_SHAPE, "heff: MPO bond mismatch");
  // steps 1 and 2 in one kernel (the MPO legs applied in the epilogue of
  // L . X), step 3 with the offset in the epilogue
  const cplx* Wm = adjoint ? m.Wlr_h[k].p : m.Wlr[k].p;
  MPSGPU_CHECK(Wm != nullptr, MPSGPU_BAD_SHAPE, "heff: adjoint needs du == dd");
  dbuf_reserve(c, c.t2, (long long)Dlb * du * Drk * wr);
  Gemm1wBatch g1;
  g1.n = 1;
  g1.d[0] = heff_first_desc(Le, Dlb, Dlk, wl, x, dd, Drk, Wm, du, wr, c.t2.p);
  heff_gemm1w(c.st(), g1);
  Gemm3Batch g3;
  g3.n = 1;
  g3.d[0] = heff_last_desc(c.t2.p, Dlb * du, Rt, Drk * wr, Drb, y, x, offset);
  heff_gemm3(c.st(), g3);
  if (cnt) {
    cnt->matvecs++;
    cnt->flops += mv_flops(dd, wl, wr, Dlb, Drb);
  }
}

// Hermitian part of the effective Hamiltonian, TensorMultiplierHermitian
// (TensorMultiplierHermitian.cpp:37-70): y = 1/2 (H x + H^dag x) + offset x,
// with H^dag from the adjoint environments (Lh, Rth) and MPO legs: both
// first contractions in one grouped launch, the two last ones as one product
// with the two sources concatenated along K.
void heff_apply_hermitian(Context& c, const cplx* Le, const cplx* Lh, const std::array<int, 3>& ld,
                          const MpoDev& m, int k, const cplx* Rt, const cplx* Rth, const std::array<int, 3>& rd,
                          const cplx* x, cplx* y, cplx offset, Counters* cnt) {
  const auto& wd = m.dims[k];
  const int du = wd[0], wl = wd[1], dd = wd[2], wr = wd[3];
  const int Dlb = ld[0], Dlk = ld[2], Drk = rd[0], Drb = rd[2];
  MPSGPU_CHECK(m.Wlr_h[k].p != nullptr, MPSGPU_BAD_SHAPE, "heff: adjoint needs du == dd");
  MPSGPU_CHECK(ld[1] == wl && rd[1] == wr, MPSGPU_BAD_SHAPE, "heff: MPO bond mismatch");
  const long long n2 = (long long)Dlb * du * Drk * wr;
  dbuf_reserve(c, c.t2, n2);
  dbuf_reserve(c, c.t3, n2);
  Gemm1wBatch g1;
  g1.n = 2;
  g1.d[0] = heff_first_desc(Le, Dlb, Dlk, wl, x, dd, Drk, m.Wlr[k].p, du, wr, c.t2.p);
  g1.d[1] = heff_first_desc(Lh, Dlb, Dlk, wl, x, dd, Drk, m.Wlr_h[k].p, du, wr, c.t3.p);
  heff_gemm1w(c.st(), g1);
  Gemm3Batch g3;
  g3.n = 1;
  g3.d[0] = heff_last_desc(c.t2.p, Dlb * du, Rt, Drk * wr, Drb, y, x, offset);
  g3.d[0].K2 = Drk * wr;
  g3.d[0].A2 = c.t3.p;
  g3.d[0].lda2 = (long long)Dlb * du;
  g3.d[0].B2 = Rth;
  g3.d[0].ldb2 = (long long)Drk * wr;
  g3.d[0].alpha = make_double2(0.5, 0.0);
  heff_gemm3(c.st(), g3);
  if (cnt) {
    cnt->matvecs++;
    cnt->flops += 2.0 * mv_flops(dd, wl, wr, Dlb, Drb);
  }
}

// Copies a descriptor blob into the next slot of the context's ring and
// returns the slot's device address (the copy is ordered on c's stream before
// the launches that read it).
static uint8_t* desc_upload(Context& c, const std::vector<uint8_t>& blob) {
  MPSGPU_CHECK(blob.size() <= kDescSlotBytes, MPSGPU_BAD_SHAPE, "grouped launch: descriptor tables too large");
  const int s = c.desc_next;
  c.desc_next = (s + 1) % kDescSlots;
  MPSGPU_CUDA(cudaEventSynchronize(c.desc_ev[s]));  // the slot's previous copy has completed
  uint8_t* h = c.hdesc + (size_t)s * kDescSlotBytes;
  uint8_t* d = c.ddesc + (size_t)s * kDescSlotBytes;
  std::memcpy(h, blob.data(), blob.size());
  MPSGPU_CUDA(cudaMemcpyAsync(d, h, blob.size(), cudaMemcpyHostToDevice, c.stream));
  MPSGPU_CUDA(cudaEventRecord(c.desc_ev[s], c.stream));
  return d;
}

template <class T>
static size_t blob_put(std::vector<uint8_t>& blob, const std::vector<T>& v) {
  const size_t off = (blob.size() + 15) & ~size_t(15);
  blob.resize(off + v.size() * sizeof(T));
  if (!v.empty()) std::memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

// The launches of a split round with the K of the first product cut into S1
// chunks and that of the last into S (each chunk at least one k-step of 16).
static void split_round_launch(Context& c, const SplitRound& r, int S1, int S, bool profile) {
  Stream st = c.st();
  if (!profile) st.prof = nullptr;
  std::vector<SplitPrepJob> jx, jt;
  std::vector<SplitProblem> g1, g3;
  std::vector<WGroup> wg;
  std::vector<SplitReduceJob> red;
  long long pix = 0;
  int maxnin = 1, maxnout = 1;
  // algorithmic work per launch: BF16 tensor flops of the two GEMMs, bytes
  // of the operand passes (FP64 read 16 B, limb planes written 12 B per entry)
  double f1 = 0.0, f3 = 0.0, bx = 0.0, bw = 0.0, bt = 0.0, br = 0.0;
  for (const SplitProduct& q : r.p) {
    const int M1 = q.Dlb * q.wl, N1 = q.dd * q.Drk, K1 = q.Dlk;
    const int M3 = q.Dlb * q.du, N3 = q.Drb, K3 = q.Drk * q.wr;
    const long long n1 = (long long)M1 * N1, n2 = (long long)M3 * K3, n3 = (long long)M3 * N3;
    const int KS3 = ceil_div(K3, 16), kps = ceil_div(KS3, S), nch = ceil_div(KS3, kps);
    const int KS1 = ceil_div(K1, 16), kps1 = ceil_div(KS1, S1), nch1 = ceil_div(KS1, kps1);
    LzWork& w = *q.ws;
    dbuf_reserve(c, w.s1, (long long)q.nh * nch1 * n1);
    dbuf_reserve(c, w.s2, q.nh * n2);
    dbuf_reserve(c, w.spart, (long long)q.nh * nch * n3);
    const long long xb = split_operand_bytes(N1, K1, 128), tb = split_operand_bytes(M3, K3, 128);
    uint8_t* xp = bytes_reserve(c, w.sx, xb);
    uint8_t* tp = bytes_reserve(c, w.st, q.nh * tb);
    // x as the B operand of T1 = L . X: its columns (dd*Drk) are the prepared rows
    jx.push_back(SplitPrepJob{N1, K1, 0, q.x, K1, 1, xp, 0});
    for (int h = 0; h < q.nh; h++) {
      MPSGPU_CHECK(q.sp[h] && q.sp[h]->ready && q.Wm[h], MPSGPU_INVALID, "split round: operands not prepared");
      cplx* T1 = w.s1.p + (long long)h * nch1 * n1;  // nch1 partial products, n1 apart
      cplx* T2 = w.s2.p + h * n2;
      uint8_t* th = tp + h * tb;
      for (int s1 = 0; s1 < nch1; s1++) {
        SplitProblem a;
        a.M = M1; a.N = N1; a.K = K1;
        a.Ap = reinterpret_cast<const uint8_t*>(q.sp[h]->Lp.p);
        a.Bp = xp;
        a.C = T1 + s1 * n1; a.ldc = M1;
        a.k0 = s1 * kps1;
        a.nk = std::min(kps1, KS1 - s1 * kps1);
        g1.push_back(a);
      }
      // T2[a', s', r, c] = sum_{b,s} W[s',b,s,c] T1[a',b,s,r], T1 the sum of its partials
      WGroup W;
      W.parts = nch1;
      W.part_stride = n1;
      WContractArgs& wa = W.a;
      wa.nx = q.Dlb; wa.ny = q.Drk;
      wa.in = T1; wa.ix = 1; wa.iy = (long long)q.Dlb * q.wl * q.dd; wa.si0 = q.Dlb; wa.si1 = (long long)q.Dlb * q.wl;
      wa.n_i0 = q.wl; wa.n_i1 = q.dd;
      wa.out = T2; wa.ox = 1; wa.oy = (long long)q.Dlb * q.du; wa.so0 = q.Dlb; wa.so1 = (long long)q.Dlb * q.du * q.Drk;
      wa.n_o0 = q.du; wa.n_o1 = q.wr;
      wa.Wm = q.Wm[h];
      W.pix_begin = pix;
      pix += wcontract_chunked((long long)q.Dlb * q.Drk);
      wg.push_back(W);
      maxnin = std::max(maxnin, q.wl * q.dd);
      maxnout = std::max(maxnout, q.du * q.wr);
      // T2 ((Dlb du) x (Drk wr), column-major) as the A operand
      jt.push_back(SplitPrepJob{M3, K3, 0, T2, 1, M3, th, 0});
      for (int s = 0; s < nch; s++) {
        SplitProblem b;
        b.M = M3; b.N = N3; b.K = K3;
        b.Ap = th;
        b.Bp = reinterpret_cast<const uint8_t*>(q.sp[h]->Rp.p);
        b.C = w.spart.p + (h * nch + s) * n3; b.ldc = M3;
        b.k0 = s * kps;
        b.nk = std::min(kps, KS3 - s * kps);
        g3.push_back(b);
      }
      f1 += 48.0 * (double)M1 * N1 * K1;
      f3 += 48.0 * (double)M3 * N3 * K3;
      bw += 16.0 * ((double)nch1 * n1 + (double)n2);
      bt += 28.0 * (double)n2;
    }
    bx += 28.0 * (double)N1 * K1;
    br += 16.0 * ((double)q.nh * nch * n3 + 2.0 * n3);
    SplitReduceJob rj;
    rj.M = M3; rj.N = N3; rj.nparts = q.nh * nch;
    rj.part = w.spart.p;
    rj.C = q.y; rj.ldc = M3;
    rj.alpha = q.alpha;
    if (q.offset.x != 0.0 || q.offset.y != 0.0) {
      rj.Cin = q.x; rj.ldcin = M3; rj.beta = q.offset;
    }
    red.push_back(rj);
  }
  const long long thr_x = split_prepare_jobs(jx.data(), (int)jx.size());
  const long long t1 = split_group_tiles(g1.data(), (int)g1.size());
  const long long thr_t = split_prepare_jobs(jt.data(), (int)jt.size());
  const long long t3 = split_group_tiles(g3.data(), (int)g3.size());
  const long long rtot = split_reduce_jobs(red.data(), (int)red.size());
  std::vector<uint8_t> blob;
  const size_t ox = blob_put(blob, jx), o1 = blob_put(blob, g1), ow = blob_put(blob, wg), ot = blob_put(blob, jt),
               o3 = blob_put(blob, g3), orr = blob_put(blob, red);
  uint8_t* d = desc_upload(c, blob);
  {
    ProfScope ps(st, GemmProfiler::SPLITOPS, bx);
    split_prepare_grouped(st, reinterpret_cast<const SplitPrepJob*>(d + ox), (int)jx.size(), thr_x);
  }
  {
    ProfScope ps(st, GemmProfiler::SPLIT, f1);
    zgemm_split_grouped(st, reinterpret_cast<const SplitProblem*>(d + o1), (int)g1.size(), t1, c.dsplit_err);
  }
  {
    ProfScope ps(st, GemmProfiler::SPLITOPS, bw);
    wcontract_grouped(st, reinterpret_cast<const WGroup*>(d + ow), (int)wg.size(), pix, maxnin, maxnout);
  }
  {
    ProfScope ps(st, GemmProfiler::SPLITOPS, bt);
    split_prepare_grouped(st, reinterpret_cast<const SplitPrepJob*>(d + ot), (int)jt.size(), thr_t);
  }
  {
    ProfScope ps(st, GemmProfiler::SPLIT, f3);
    zgemm_split_grouped(st, reinterpret_cast<const SplitProblem*>(d + o3), (int)g3.size(), t3, c.dsplit_err);
  }
  {
    ProfScope ps(st, GemmProfiler::SPLITOPS, br);
    split_reduce_grouped(st, reinterpret_cast<const SplitReduceJob*>(d + orr), (int)red.size(), rtot);
  }
}

// Autotuner of the split round's K chunks: the first round of each shape
// signature (device; every product's dimensions and halves) times the
// candidate chunk counts on its own operands (a round only reads its inputs
// and overwrites its intermediates and outputs, so running it again is
// harmless) and keeps the fastest for every later round of that signature,
// for all contexts of the process.  Off with mpsgpu_set_autotune(0) (or
// MPSGPU_AUTOTUNE=0), and while the stream is captured into a graph; then
// the heuristic: about one CTA per SM over the round's tiles.
namespace {
std::mutex g_split_tune_mu;
std::map<std::vector<int>, std::pair<int, int>> g_split_tune;
}  // namespace

long long split_autotune_entries() {
  std::lock_guard<std::mutex> lk(g_split_tune_mu);
  return (long long)g_split_tune.size();
}

void split_round_run(Context& c, SplitRound& r) {
  const int n = (int)r.p.size();
  if (n == 0) return;
  // at most 16 products per set of launches (the descriptor tables of one
  // set fit one slot of the context's ring)
  if (n > kSplitRoundMax) {
    for (int i0 = 0; i0 < n; i0 += kSplitRoundMax) {
      SplitRound part;
      part.p.assign(r.p.begin() + i0, r.p.begin() + std::min(n, i0 + kSplitRoundMax));
      split_round_run(c, part);
    }
    r.p.clear();
    return;
  }
  const int nsm = device_sms(c);
  long long tiles1 = 0, tiles3 = 0;
  int ks1 = 1, ks3 = 1;
  std::vector<int> key{c.device};
  for (const SplitProduct& q : r.p) {
    tiles1 += (long long)q.nh * ceil_div(q.Dlb * q.wl, 128) * ceil_div(q.dd * q.Drk, 128);
    tiles3 += (long long)q.nh * ceil_div(q.Dlb * q.du, 128) * ceil_div(q.Drb, 128);
    ks1 = std::max(ks1, ceil_div(q.Dlk, 16));
    ks3 = std::max(ks3, ceil_div(q.Drk * q.wr, 16));
    key.insert(key.end(), {q.nh, q.Dlb, q.Dlk, q.wl, q.dd, q.Drk, q.du, q.wr, q.Drb});
  }
  // heuristic: chunks of at least four k-steps, about one CTA per SM over the
  // round's tiles, at most 4 for the first product (the MPO-leg kernel adds
  // its chunks) and 8 for the last
  auto chunks = [&](long long tiles, int ks, int cap) {
    const int s = (int)std::min<long long>(cap, std::max<long long>(1, (nsm + tiles - 1) / std::max<long long>(1, tiles)));
    return std::max(1, std::min(s, ks / 4));
  };
  int S1 = chunks(tiles1, ks1, 4), S = chunks(tiles3, ks3, 8);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool tune = gemm_autotune_on() && cudaStreamIsCapturing(c.stream, &cs) == cudaSuccess &&
                    cs == cudaStreamCaptureStatusNone;
  bool found = false;
  if (tune) {
    std::lock_guard<std::mutex> lk(g_split_tune_mu);
    auto it = g_split_tune.find(key);
    if (it != g_split_tune.end()) {
      S1 = it->second.first;
      S = it->second.second;
      found = true;
    }
  }
  if (tune && !found) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MPSGPU_CUDA(cudaEventCreate(&e0));
    MPSGPU_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int b1 = S1, b3 = S;
    try {
      for (int s1 : {1, 2, 4}) {
        if (s1 > 1 && s1 > ks1 / 2) continue;
        for (int s3 : {1, 2, 4, 8}) {
          if (s3 > 1 && s3 > ks3 / 2) continue;
          split_round_launch(c, r, s1, s3, false);  // warm (buffers, descriptor slots)
          MPSGPU_CUDA(cudaEventRecord(e0, c.stream));
          for (int rep = 0; rep < 2; rep++) split_round_launch(c, r, s1, s3, false);
          MPSGPU_CUDA(cudaEventRecord(e1, c.stream));
          MPSGPU_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          MPSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if (ms < best) {
            best = ms;
            b1 = s1;
            b3 = s3;
          }
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    S1 = b1;
    S = b3;
    std::lock_guard<std::mutex> lk(g_split_tune_mu);
    g_split_tune[key] = {S1, S};
  }
  split_round_launch(c, r, S1, S, true);
  r.p.clear();
}

void env_left_update(Context& c, const cplx* Le, const std::array<int, 3>& ld, const MpsDev& ket,
                     const MpoDev* m, int k, const MpsDev& bra, DBuf& out, std::array<int, 3>& od,
                     Counters* cnt) {
  const auto& kd = ket.dims[k];
  const auto& bd = bra.dims[k];
  const int dd = kd[0], Dlk = kd[1], Drk = kd[2];
  const int du = bd[0], Dlb = bd[1], Drb = bd[2];
  const int wl = m ? m->dims[k][1] : 1, wr = m ? m->dims[k][3] : 1;
  MPSGPU_CHECK(ld[0] == Dlb && ld[2] == Dlk && ld[1] == wl, MPSGPU_BAD_SHAPE, "envL: dims");
  const cplx* T2 = nullptr;
  if (m) {
    // T2[a', t, c, r'] = sum_{a,b,s} W[t,b,s,c] L[a',b,a] X_ket[a,s,r'] (one kernel)
    dbuf_reserve(c, c.t2, (long long)Dlb * du * wr * Drk);
    Gemm1wBatch g1;
    g1.n = 1;
    Gemm1wDesc& d = g1.d[0];
    d.A = Le; d.lda = (long long)Dlb * wl;
    d.B = ket.A[k].p; d.ldb = Dlk;
    d.X = Dlb; d.Y = Drk; d.K = Dlk;
    d.n_i0 = wl; d.n_i1 = dd; d.n_o0 = du; d.n_o1 = wr;
    d.Wm = m->Wlr[k].p;
    d.out = c.t2.p; d.ox = 1; d.oy = (long long)Dlb * du * wr; d.so0 = Dlb; d.so1 = (long long)Dlb * du;
    heff_gemm1w(c.st(), g1);
    T2 = c.t2.p;
  } else {
    // T1 = L . X_ket  -> [a', s, r'] (w = 1)
    dbuf_reserve(c, c.t1, (long long)Dlb * wl * dd * Drk);
    GemmArgs g;
    g.M = Dlb * wl; g.N = dd * Drk; g.K = Dlk;
    g.A = Le; g.lda = (long long)Dlb * wl;
    g.B = ket.A[k].p; g.ldb = Dlk;
    g.C = c.t1.p; g.ldc = (long long)Dlb * wl;
    zgemm(c.st(), g, c.scratch);
    T2 = c.t1.p;
  }
  // Lnew[r, (c, r')] = X_bra^H . T2
  od = {Drb, wr, Drk};
  dbuf_reserve(c, out, (long long)Drb * wr * Drk);
  GemmArgs h;
  h.M = Drb; h.N = wr * Drk; h.K = Dlb * du;
  h.A = bra.A[k].p; h.lda = (long long)Dlb * du; h.opA = OP_C;
  h.B = T2; h.ldb = (long long)Dlb * du;
  h.C = out.p; h.ldc = Drb;
  zgemm(c.st(), h, c.scratch);
  if (cnt) {
    cnt->env_updates++;
    cnt->flops += mv_flops(dd, wl, wr, Dlb, Drb);
  }
}

void env_right_update(Context& c, const cplx* Rt, const std::array<int, 3>& rd, const MpsDev& ket,
                      const MpoDev* m, int k, const MpsDev& bra, DBuf& out, std::array<int, 3>& od,
                      Counters* cnt) {
  const auto& kd = ket.dims[k];
  const auto& bd = bra.dims[k];
  const int dd = kd[0], Dlk = kd[1], Drk = kd[2];
  const int du = bd[0], Dlb = bd[1], Drb = bd[2];
  const int wl = m ? m->dims[k][1] : 1, wr = m ? m->dims[k][3] : 1;
  MPSGPU_CHECK(rd[0] == Drk && rd[2] == Drb && rd[1] == wr, MPSGPU_BAD_SHAPE, "envR: dims");
  const cplx* T2 = nullptr;
  if (m) {
    // T2[l', b, t, r] = sum_{s,c,r''} W[t,b,s,c] X_ket[l',s,r''] Rt[r'',c,r] (one kernel)
    dbuf_reserve(c, c.t2, (long long)Dlk * wl * du * Drb);
    Gemm1wBatch g1;
    g1.n = 1;
    Gemm1wDesc& d = g1.d[0];
    d.A = ket.A[k].p; d.lda = (long long)Dlk * dd;
    d.B = Rt; d.ldb = Drk;
    d.X = Dlk; d.Y = Drb; d.K = Drk;
    d.n_i0 = dd; d.n_i1 = wr; d.n_o0 = wl; d.n_o1 = du;
    d.Wm = m->Wrl[k].p;
    d.out = c.t2.p; d.ox = 1; d.oy = (long long)Dlk * wl * du; d.so0 = Dlk; d.so1 = (long long)Dlk * wl;
    heff_gemm1w(c.st(), g1);
    T2 = c.t2.p;
  } else {
    // T1[(l', s), r] = X_ket((Dlk*dd) x Drk) . Rt(Drk x Drb)  (w = 1)
    dbuf_reserve(c, c.t1, (long long)Dlk * dd * wr * Drb);
    GemmArgs g;
    g.M = Dlk * dd; g.N = wr * Drb; g.K = Drk;
    g.A = ket.A[k].p; g.lda = (long long)Dlk * dd;
    g.B = Rt; g.ldb = Drk;
    g.C = c.t1.p; g.ldc = (long long)Dlk * dd;
    zgemm(c.st(), g, c.scratch);
    T2 = c.t1.p;
  }
  // Rt_new[(l', b), l] = T2((Dlk*wl) x (du*Drb)) . X_bra^H  (X_bra as Dlb x (du*Drb))
  od = {Dlk, wl, Dlb};
  dbuf_reserve(c, out, (long long)Dlk * wl * Dlb);
  GemmArgs h;
  h.M = Dlk * wl; h.N = Dlb; h.K = du * Drb;
  h.A = T2; h.lda = (long long)Dlk * wl;
  h.B = bra.A[k].p; h.ldb = Dlb; h.opB = OP_C;
  h.C = out.p; h.ldc = (long long)Dlk * wl;
  zgemm(c.st(), h, c.scratch);
  if (cnt) {
    cnt->env_updates++;
    cnt->flops += mv_flops(dd, wl, wr, Dlb, Drb);
  }
}

void EnvCache::init(Context& c, int L_) {
  L = L_;
  Le.assign(L, DBuf());
  Re.assign(L, DBuf());
  ldims.assign(L, {1, 1, 1});
  rdims.assign(L, {1, 1, 1});
  okL.assign(L, 0);
  okR.assign(L, 0);
  cplx one = make_double2(1.0, 0.0);
  dbuf_reserve(c, Le[0], 1);
  dbuf_reserve(c, Re[L - 1], 1);
  MPSGPU_CUDA(cudaMemcpyAsync(Le[0].p, &one, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
  MPSGPU_CUDA(cudaMemcpyAsync(Re[L - 1].p, &one, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
  MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  okL[0] = 1;
  okR[L - 1] = 1;
}

void EnvCache::release(Context& c) {
  for (auto& b : Le) dbuf_free(c, b);
  for (auto& b : Re) dbuf_free(c, b);
}

// Contractor::calculateL / calculateR (Contractor.cpp:723-764)
static void calc_left(Context& c, EnvCache& E, int pos, const MpoDev* ops, const MpsDev& ket,
                      const MpsDev& bra, Counters* cnt) {
  if (E.okL[pos]) return;
  calc_left(c, E, pos - 1, ops, ket, bra, cnt);
  env_left_update(c, E.Le[pos - 1].p, E.ldims[pos - 1], ket, ops, pos - 1, bra, E.Le[pos], E.ldims[pos], cnt);
  E.okL[pos] = 1;
}

static void calc_right(Context& c, EnvCache& E, int pos, const MpoDev* ops, const MpsDev& ket,
                       const MpsDev& bra, Counters* cnt) {
  if (E.okR[pos]) return;
  calc_right(c, E, pos + 1, ops, ket, bra, cnt);
  env_right_update(c, E.Re[pos + 1].p, E.rdims[pos + 1], ket, ops, pos + 1, bra, E.Re[pos], E.rdims[pos], cnt);
  E.okR[pos] = 1;
}

// Contractor::contract(ket, ops, bra) (Contractor.cpp:467-556)
cplx contract(Context& c, const MpsDev& ket, const MpoDev* ops, const MpsDev& bra) {
  MPSGPU_CHECK(ket.L == bra.L && (!ops || ops->L == ket.L), MPSGPU_BAD_SHAPE, "contract: lengths");
  DBuf a, b;
  std::array<int, 3> ad = {1, 1, 1}, bd;
  dbuf_reserve(c, a, 1);
  cplx one = make_double2(1.0, 0.0);
  MPSGPU_CUDA(cudaMemcpyAsync(a.p, &one, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
  for (int k = 0; k < ket.L; k++) {
    env_left_update(c, a.p, ad, ket, ops, k, bra, b, bd, nullptr);
    std::swap(a, b);
    ad = bd;
  }
  cplx r;
  MPSGPU_CUDA(cudaMemcpyAsync(&r, a.p, sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
  MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  dbuf_free(c, a);
  dbuf_free(c, b);
  return cscale(r, ket.normfact * bra.normfact);
}

// Contractor::contract2(bra, ops, ket) = <bra|ops^dag ops|ket>
// (Contractor.cpp:634-718, Operator::contractL2): the doubled operator
// (O^dag O)(s', b1 b2, s, c1 c2) = sum_t conj(O(t, b1, s', c1)) O(t, b2, s, c2)
// (bond index b1 + wl b2) is formed on the host from the device copy of O
// and contracted like any MPO.
cplx contract2(Context& c, const MpoDev& ops, const MpsDev& ket, const MpsDev& bra) {
  const int L = ops.L;
  MPSGPU_CHECK(ket.L == L && bra.L == L, MPSGPU_BAD_SHAPE, "contract2: lengths");
  std::vector<std::vector<cplx>> dbl(L);
  std::vector<int> dims(4 * L);
  std::vector<const double*> ptrs(L);
  for (int k = 0; k < L; k++) {
    const auto& w = ops.dims[k];
    const int du = w[0], wl = w[1], dd = w[2], wr = w[3];
    std::vector<cplx> W((size_t)du * wl * dd * wr);
    MPSGPU_CUDA(cudaMemcpyAsync(W.data(), ops.W[k].p, W.size() * sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    auto at = [&](int t, int b, int s, int cc) { return W[t + du * (b + wl * (s + dd * cc))]; };
    const int WL = wl * wl, WR = wr * wr;
    dbl[k].assign((size_t)dd * WL * dd * WR, make_double2(0.0, 0.0));
    for (int sp = 0; sp < dd; sp++)
      for (int b1 = 0; b1 < wl; b1++)
        for (int b2 = 0; b2 < wl; b2++)
          for (int s = 0; s < dd; s++)
            for (int c1 = 0; c1 < wr; c1++)
              for (int c2 = 0; c2 < wr; c2++) {
                cplx acc = make_double2(0.0, 0.0);
                for (int t = 0; t < du; t++) acc = cadd(acc, ccmul(at(t, b1, sp, c1), at(t, b2, s, c2)));
                dbl[k][sp + dd * ((b1 + wl * b2) + WL * (s + dd * (c1 + wr * c2)))] = acc;
              }
    dims[4 * k] = dd; dims[4 * k + 1] = WL; dims[4 * k + 2] = dd; dims[4 * k + 3] = WR;
    ptrs[k] = reinterpret_cast<const double*>(dbl[k].data());
  }
  MpoDev two;
  mpo_upload(c, two, L, dims.data(), ptrs.data(), false);
  cplx r;
  try {
    r = contract(c, ket, &two, bra);
  } catch (...) {
    mpo_free(c, two);
    throw;
  }
  mpo_free(c, two);
  return r;
}

// ---------------------------------------------------------------------------
// Lanczos for the lowest eigenpair (replaces the PRIMME call of
// Contractor::solveEigs, Contractor.cpp:3067-3138; and its dense branch),
// for a batch of independent local problems advanced in lockstep.
// Thick-restarted Lanczos with full reorthogonalisation, FP64; convergence
// ||r|| <= tol * max|Ritz|.  Every task's product computes y = (H - sigma) x
// (the excited-state multiplier without its projector); sigma follows the
// task's latest Ritz value (shift0 before the first one is known), which
// keeps the Gram-Schmidt passes well conditioned.  With nu > 0, U (N x nu)
// holds the projector vectors with the square roots of the penalties folded
// in, and the step adds U (U^H v_j) to every product
// (TensorMultiplierProjMulti.cpp:81-90).
//
// One round = one iteration of every active task: FP64 products are
// appended to grouped launches of the two contractions (heff.cu), the
// products of tasks in their split-precision phase to one split round
// (split_round_run: six grouped launches for all of them), then one
// cooperative launch of the Lanczos step (lzstep.cu) serves all tasks and
// writes each task's alpha_j, beta_j into its mapped host mirror.  The host
// enqueues round r+1 before it waits for round r, so the convergence tests
// (tridiagonal eigenpairs on the host) overlap the device work; a
// speculative iteration after convergence is discarded (it only writes the
// task's V[:, j+2], w and the coefficients of step j+1).  Tasks converge,
// restart and leave the batch independently; the arithmetic of a task is
// the same whatever else runs in its rounds.
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Contexts: one stream with its own workspaces; a batch of sweeps gives each
// sweep a sub-context so that their gauge moves and environment updates
// overlap on the GPU while their Lanczos rounds share grouped launches.
// ---------------------------------------------------------------------------

void context_init(Context& c, int device) {
  c.device = device;
  MPSGPU_CUDA(cudaSetDevice(device));
  // the no-allocation QR's fixed array is placed now, while allocation is
  // still allowed, not at that entry point's first call
  {
    const mpsgpu_status ns = noalloc_qr_prepare(device);
    MPSGPU_CHECK(ns == MPSGPU_OK, ns, "create: placing the no-allocation QR scratch failed");
  }
  MPSGPU_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  c.scratch.stream = c.stream;
  c.qrws.stream = c.stream;
  // keep freed pool memory cached across calls
  cudaMemPool_t pool;
  MPSGPU_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t thresh = UINT64_MAX;
  MPSGPU_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
  MPSGPU_CUDA(cudaMalloc((void**)&c.dscal, 1024 * sizeof(double)));
  MPSGPU_CUDA(cudaMalloc((void**)&c.dcplx, 1024 * sizeof(cplx)));
  MPSGPU_CUDA(cudaMallocHost((void**)&c.hscal, 1024 * sizeof(double)));
  MPSGPU_CUDA(cudaMallocHost((void**)&c.hcplx, 1024 * sizeof(cplx)));
  MPSGPU_CUDA(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming));
  MPSGPU_CUDA(cudaEventCreate(&c.mv0));
  MPSGPU_CUDA(cudaEventCreate(&c.mv1));
  MPSGPU_CUDA(cudaHostAlloc((void**)&c.hsplit_err, sizeof(int), cudaHostAllocMapped));
  MPSGPU_CUDA(cudaHostGetDevicePointer((void**)&c.dsplit_err, c.hsplit_err, 0));
  *c.hsplit_err = 0;
  MPSGPU_CUDA(cudaHostAlloc((void**)&c.hlz_err, sizeof(int), cudaHostAllocMapped));
  MPSGPU_CUDA(cudaHostGetDevicePointer((void**)&c.dlz_err, c.hlz_err, 0));
  *c.hlz_err = 0;
  MPSGPU_CUDA(cudaMalloc((void**)&c.dcounter, kCounterWords * sizeof(unsigned)));
  MPSGPU_CUDA(cudaMemset(c.dcounter, 0, kCounterWords * sizeof(unsigned)));
  c.iter_ev.resize(257);
  for (auto& e : c.iter_ev) MPSGPU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  MPSGPU_CUDA(cudaMallocHost((void**)&c.hdesc, kDescSlots * kDescSlotBytes));
  MPSGPU_CUDA(cudaMalloc((void**)&c.ddesc, kDescSlots * kDescSlotBytes));
  for (auto& e : c.desc_ev) MPSGPU_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

void context_release(Context& c) {
  cudaSetDevice(c.device);
  for (auto& sc : c.subs) context_release(*sc);
  c.subs.clear();
  for (DBuf* b : {&c.t1, &c.t2, &c.t3, &c.t4, &c.matA, &c.matQ, &c.matR, &c.lzws}) dbuf_free(c, *b);
  c.scratch.release();
  c.qrws.release();
  c.lzone.release(c);
  if (c.stream) cudaStreamSynchronize(c.stream);
  cudaFree(c.dscal);
  cudaFree(c.dcplx);
  cudaFreeHost(c.hscal);
  cudaFreeHost(c.hcplx);
  if (c.ev) cudaEventDestroy(c.ev);
  if (c.mv0) cudaEventDestroy(c.mv0);
  if (c.mv1) cudaEventDestroy(c.mv1);
  for (auto e : c.iter_ev)
    if (e) cudaEventDestroy(e);
  if (c.hsplit_err) cudaFreeHost(c.hsplit_err);
  if (c.hlz_err) cudaFreeHost(c.hlz_err);
  cudaFree(c.dcounter);
  for (auto e : c.desc_ev)
    if (e) cudaEventDestroy(e);
  if (c.hdesc) cudaFreeHost(c.hdesc);
  cudaFree(c.ddesc);
  c.hdesc = nullptr;
  c.ddesc = nullptr;
  if (c.stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
}

Context& context_sub(Context& c, int i) {
  while ((int)c.subs.size() <= i) {
    c.subs.emplace_back(new Context());
    context_init(*c.subs.back(), c.device);
    c.subs.back()->parent = &c;
  }
  return *c.subs[i];
}

void LzWork::init(Context& c) {
  if (dsc) return;
  MPSGPU_CUDA(cudaMalloc((void**)&dsc, sizeof(LanczosScalars)));
  MPSGPU_CUDA(cudaMemsetAsync(dsc, 0, sizeof(LanczosScalars), c.stream));
  MPSGPU_CUDA(cudaHostAlloc((void**)&hsc, sizeof(LanczosScalars), cudaHostAllocMapped));
  MPSGPU_CUDA(cudaHostGetDevicePointer((void**)&hsc_dev, hsc, 0));
  MPSGPU_CUDA(cudaMalloc((void**)&dS, 256 * sizeof(double)));
}

void LzWork::release(Context& c) {
  for (DBuf* b : {&V, &w, &t2, &t3, &T, &Q, &s1, &s2, &spart, &sx, &st}) dbuf_free(c, *b);
  if (dsc) {
    cudaStreamSynchronize(c.stream);
    cudaFree(dsc);
    cudaFreeHost(hsc);
    cudaFree(dS);
  }
  dsc = nullptr;
  hsc = hsc_dev = nullptr;
  dS = nullptr;
}

namespace {

struct LzState {
  LzTask* t = nullptr;
  int m = 0, keep = 0, max_restarts = 0, restart = 0;
  int j0 = 0;        // first iteration of the current cycle
  int jq = -1;       // last iteration enqueued
  int jr = -1;       // last iteration whose result was read
  bool done = false;
  bool pending_restart = false;  // next round starts a new cycle at j0
  std::vector<double> a, b, s, gq;
  std::vector<cplx> gqc;
  double theta = 0.0, step_hint = 0.0, sigma = 0.0;
  bool have_theta = false;
  TridiagLowest tri;
  ThickRestart thick;
};

}  // namespace

void lanczos_batch(Context& c, std::vector<LzTask*>& tasks) {
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  const Stream st = c.st();
  const int nt = (int)tasks.size();
  if (nt == 0) return;
  std::vector<LzState> S(nt);
  long long nrb_total = 0;
  double* d_tmp = c.dscal + 512;
  for (int q = 0; q < nt; q++) {
    LzTask& t = *tasks[q];
    LzState& z = S[q];
    z.t = &t;
    MPSGPU_CHECK(t.ws != nullptr && t.N > 0, MPSGPU_INVALID, "lanczos: task without workspace");
    MPSGPU_CHECK(t.nu <= LZ_MAXU, MPSGPU_BAD_SHAPE, "lanczos: at most 8 projector vectors");
    LzWork& ws = *t.ws;
    ws.init(c);
    const int N = t.N;
    z.m = std::min(N, std::max(2, std::min(t.max_krylov, 200)));
    z.keep = std::max(1, z.m / 2);
    // budget of about 3840 products (60 cycles of a 64-vector space), whatever m
    z.max_restarts = std::max(60, 3840 / std::max(1, z.m - z.keep));
    z.sigma = std::isfinite(t.shift0) ? t.shift0 : 0.0;
    dbuf_reserve(c, ws.V, (long long)N * (z.m + 1));
    dbuf_reserve(c, ws.w, N);
    nrb_total += ceil_div(N, lanczos_step_rows_per_block());
    // v0 = x / ||x|| (a zero or non-finite start becomes the flat vector)
    dznrm2(st, N, t.x, d_tmp, c.scratch);
    MPSGPU_CUDA(cudaMemcpyAsync(c.hscal, d_tmp, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    if (!(c.hscal[0] > 0.0) || !std::isfinite(c.hscal[0])) {
      zfill(st, N, make_double2(1.0 / std::sqrt((double)N), 0.0), t.x);
      dznrm2(st, N, t.x, d_tmp, c.scratch);
    }
    zscal_inv(st, N, t.x, d_tmp, ws.V.p);
    t.iters = 0;
  }
  // workspace of the step, shared by the instances of a launch: partial dots
  // (row blocks x 256), two partial-norm arrays, the coefficients h, h2
  dbuf_reserve(c, c.lzws, 2 * nrb_total * 256 + nrb_total + 8);
  cplx* part = c.lzws.p;
  cplx* part2 = part + nrb_total * 256;
  double* pn1 = reinterpret_cast<double*>(part2 + nrb_total * 256);
  double* pn2 = pn1 + nrb_total;

  auto check_step = [&]() {
    if (*c.hlz_err) {
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
      MPSGPU_CUDA(cudaMemsetAsync(c.dcounter + kLzBarrierOffset, 0, 2 * LZ_MAXI * sizeof(unsigned), c.stream));
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
      *c.hlz_err = 0;
      throw Error(MPSGPU_TIMEOUT, "lanczos: a bounded grid barrier of the Lanczos step ran out");
    }
  };

  // Enqueue one round: iteration it[q] of every listed task.
  std::vector<std::pair<int, int>> round;  // (task, iteration)
  auto launch_round = [&](const std::vector<std::pair<int, int>>& items, cudaEvent_t ev) {
    const auto t0 = clk::now();
    RoundBatch rb;
    auto flush = [&]() {
      if (rb.g1.n) heff_gemm1w(st, rb.g1);
      if (rb.g3.n) heff_gemm3(st, rb.g3);
      rb.g1.n = rb.g3.n = 0;
    };
    for (auto& it : items) {
      LzState& z = S[it.first];
      LzTask& t = *z.t;
      if (rb.g1.n + 2 > GEMM_MAXP || rb.g3.n + 1 > GEMM_MAXP) flush();
      t.product(c, t.ws->V.p + (long long)it.second * t.N, t.ws->w.p, z.sigma, rb);
    }
    flush();
    split_round_run(c, rb.sr);
    for (size_t i0 = 0; i0 < items.size(); i0 += LZ_MAXI) {
      LzBatch b;
      b.ninst = (int)std::min<size_t>(LZ_MAXI, items.size() - i0);
      b.part = part;
      b.part2 = part2;
      b.pn1 = pn1;
      b.pn2 = pn2;
      b.bar = c.dcounter + kLzBarrierOffset;
      b.err = c.dlz_err;
      for (int i = 0; i < b.ninst; i++) {
        LzState& z = S[items[i0 + i].first];
        LzTask& t = *z.t;
        const int j = items[i0 + i].second;
        LzInst& in = b.in[i];
        in.n = t.N;
        in.j = j;
        in.k = j + 1;
        in.nu = t.nu;
        in.U = t.U;
        in.write_next = j + 1 < z.m ? 1 : 0;
        in.sigma = z.sigma;
        in.V = t.ws->V.p;
        in.ldv = t.N;
        in.w = t.ws->w.p;
        in.sc = t.ws->dsc;
        in.mirror = t.ws->hsc_dev;
      }
      lanczos_step(st, b);
    }
    MPSGPU_CUDA(cudaEventRecord(ev, c.stream));
    for (auto& it : items) {
      S[it.first].jq = it.second;
      S[it.first].t->iters++;
    }
    const double dt = secs(t0, clk::now()) / items.size();
    for (auto& it : items)
      if (S[it.first].t->cnt) S[it.first].t->cnt->host_launch_s += dt;
  };

  // Ritz vector of a task's tridiagonal (k x k) into its x, normalised (enqueued)
  auto ritz_vector = [&](LzState& z, int k) {
    LzTask& t = *z.t;
    MPSGPU_CUDA(cudaMemcpyAsync(t.ws->dS, z.s.data(), k * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    combine_real(st, t.N, k, t.ws->V.p, t.N, t.ws->dS, t.x);
    dznrm2(st, t.N, t.x, d_tmp, c.scratch);
    zscal_inv(st, t.N, t.x, d_tmp, t.x);
    t.theta = z.theta;
    z.done = true;
  };

  // compress after a cycle without convergence (ThickRestart); true when
  // the kept space already holds the converged pair
  auto compress = [&](LzState& z) -> bool {
    LzTask& t = *z.t;
    const int m = z.m, N = t.N;
    if (z.keep >= m) {
      // no room to keep more than one vector: restart from the Ritz vector
      ritz_vector(z, m);
      z.done = false;
      zcopy(st, N, t.x, t.ws->V.p);
      z.a.clear();
      z.b.clear();
      z.j0 = 0;
      return false;
    }
    // V[:, 0..r) <- V G; V[:, r] = f / |f| with f = w, the orthogonalised
    // (not normalised) residual of step m-1
    const double fnorm = z.b[m - 1];
    const int r = z.thick.compress(z.a, z.b, m, z.keep, fnorm, z.gq);
    z.gqc.resize(z.gq.size());
    for (size_t i = 0; i < z.gq.size(); i++) z.gqc[i] = make_double2(z.gq[i], 0.0);
    dbuf_reserve(c, t.ws->Q, (long long)z.gqc.size());
    dbuf_reserve(c, t.ws->T, (long long)N * r);
    MPSGPU_CUDA(cudaMemcpyAsync(t.ws->Q.p, z.gqc.data(), z.gqc.size() * sizeof(cplx), cudaMemcpyHostToDevice,
                                c.stream));
    GemmArgs g;
    g.M = N; g.N = r; g.K = m;
    g.A = t.ws->V.p; g.lda = N;
    g.B = t.ws->Q.p; g.ldb = m;
    g.C = t.ws->T.p; g.ldc = N;
    zgemm(st, g, c.scratch);
    MPSGPU_CUDA(cudaMemcpyAsync(t.ws->V.p, t.ws->T.p, (size_t)N * r * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                c.stream));
    double normT = 0.0;
    z.tri.solve(z.a, z.b, r, z.theta, z.s, normT);
    const double scale = std::max(normT, std::fabs(z.theta));
    if (z.b[r - 1] * std::fabs(z.s[r - 1]) <= t.tol * scale || z.b[r - 1] <= 1e-14 * scale) {
      ritz_vector(z, r);  // converged within the kept space
      return true;
    }
    zscal_inv(st, N, t.ws->w.p, &t.ws->dsc->beta[m - 1], t.ws->V.p + (long long)r * N);  // beta[m-1] = |f|
    // the coupling of V[:, r-1] to the new V[:, r], used by the next step
    MPSGPU_CUDA(cudaMemcpyAsync(&t.ws->dsc->beta[r - 1], &z.b[r - 1], sizeof(double), cudaMemcpyHostToDevice,
                                c.stream));
    z.sigma = z.theta;
    z.j0 = r;
    return false;
  };

  int rid = 0;
  auto next_event = [&]() { return c.iter_ev[(rid++) % c.iter_ev.size()]; };
  // round 0: the first iteration of every task
  std::vector<std::pair<int, int>> cur;
  for (int q = 0; q < nt; q++) cur.push_back({q, 0});
  cudaEvent_t cur_ev = next_event();
  launch_round(cur, cur_ev);
  while (!cur.empty()) {
    // speculative next round: every task of this round that continues its cycle,
    // plus tasks restarting a cycle
    std::vector<std::pair<int, int>> nxt;
    for (int q = 0; q < nt; q++) {
      LzState& z = S[q];
      if (z.done) continue;
      if (z.pending_restart) {
        nxt.push_back({q, z.j0});
        z.pending_restart = false;
      } else if (z.jq >= 0 && z.jq + 1 < z.m && z.jq == z.jr + 1) {
        nxt.push_back({q, z.jq + 1});
      }
    }
    cudaEvent_t nxt_ev = nullptr;
    if (!nxt.empty()) {
      nxt_ev = next_event();
      launch_round(nxt, nxt_ev);
    }
    const auto tw = clk::now();
    MPSGPU_CUDA(cudaEventSynchronize(cur_ev));
    check_step();
    const auto tt = clk::now();
    for (auto& it : cur) {
      LzState& z = S[it.first];
      LzTask& t = *z.t;
      if (t.cnt) t.cnt->host_wait_s += secs(tw, tt) / cur.size();
      if (z.done) continue;  // a speculative iteration after convergence
      const int j = it.second;
      z.jr = j;
      const auto t0 = clk::now();
      const double alpha = t.ws->hsc->alpha[j];
      const double beta = t.ws->hsc->beta[j];
      MPSGPU_CHECK(std::isfinite(alpha) && std::isfinite(beta), MPSGPU_NAN, "lanczos: non-finite value");
      z.a.push_back(alpha);
      z.b.push_back(beta);
      double normT = 0.0;
      const double th_old = z.theta;
      if (z.have_theta)
        z.tri.solve_from(z.a, z.b, (int)z.a.size(), th_old, 4.0 * z.step_hint, z.theta, z.s, normT);
      else
        z.tri.solve(z.a, z.b, (int)z.a.size(), z.theta, z.s, normT);
      z.step_hint = z.have_theta ? std::fabs(th_old - z.theta) : 0.0;
      z.have_theta = true;
      z.sigma = z.theta;
      const double res = beta * std::fabs(z.s[j]);
      const double scale = std::max(normT, std::fabs(z.theta));
      if (res <= t.tol * scale || beta <= 1e-14 * scale || j + 1 == t.N) {
        ritz_vector(z, j + 1);
      } else if (j + 1 == z.m) {
        if (++z.restart >= z.max_restarts) throw Error(MPSGPU_NOT_CONVERGED, "lanczos: no convergence");
        if (!compress(z)) {
          z.pending_restart = true;
          z.jq = z.jr = z.j0 - 1;
        }
      }
      if (t.cnt) t.cnt->host_tridiag_s += secs(t0, clk::now());
    }
    cur = std::move(nxt);
    cur_ev = nxt_ev;
    // tasks that restarted (or stopped speculating) and are not in the round
    // just launched start their next round after it
    if (cur.empty()) {
      for (int q = 0; q < nt; q++) {
        LzState& z = S[q];
        if (z.done) continue;
        std::vector<std::pair<int, int>> one;
        if (z.pending_restart) {
          cur.push_back({q, z.j0});
          z.pending_restart = false;
        } else if (z.jq + 1 < z.m && z.jq == z.jr) {
          cur.push_back({q, z.jq + 1});
        }
      }
      if (!cur.empty()) {
        cur_ev = next_event();
        launch_round(cur, cur_ev);
      }
    }
  }
  for (auto& z : S) MPSGPU_CHECK(z.done, MPSGPU_NOT_CONVERGED, "lanczos: a task left the batch unfinished");
  MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
  check_step();
}

// One local problem with a product that launches its own kernels (the
// two-site sweep), as a batch of one.
template <class Op>
static double lanczos_lowest(Context& c, int N, Op apply, cplx* x, double tol, int max_krylov, int* iters,
                             double shift0, Counters* cnt = nullptr) {
  LzWork& ws = c.lzone;
  LzTask t;
  t.N = N;
  t.x = x;
  t.tol = tol;
  t.shift0 = shift0;
  t.max_krylov = max_krylov;
  t.ws = &ws;
  t.cnt = cnt;
  t.product = [&](Context&, const cplx* xin, cplx* yout, double sigma, RoundBatch&) { apply(xin, yout, sigma); };
  std::vector<LzTask*> v{&t};
  lanczos_batch(c, v);
  if (iters) *iters = t.iters;
  return t.theta;
}

// ---------------------------------------------------------------------------
// findGroundState (Contractor.cpp:1352-1533)
// ---------------------------------------------------------------------------

// MPS(const MPS&, int D) (MPS.cpp:761-772): copy, then gaugeCond('L', 0, D),
// right-to-left SVD cuts to at most D that keep the norm in normfact.
void mps_approximate(Context& c, const MpsDev& src, MpsDev& dst, int D, double* disc) {
  MPSGPU_CHECK(D > 0, MPSGPU_INVALID, "approximate: D must be positive");
  mps_copy(c, src, dst);
  if (disc) *disc = 0.0;
  mps_gauge_all(c, dst, 'L', false, D, disc);
  dst.bond = dst.max_bond();
}

// MPO applied exactly to an MPS, site by site, with an SVD gauge move after
// every site: MPS::applyExactly (cutD <= 0: no cut beyond dropping zero
// singular values) and MPS::truncate / approximate (cutD > 0), MPS.cpp:
// 858-936, with Site::reduceDimLOp / reduceDimROp (Site.cpp:303-402).
// dir 'L' sweeps L-1 -> 0 (right-isometric result), 'R' sweeps 0 -> L-1.
// The carried factor ("link") is kept as (r, w, beta) with r fastest for
// 'L' and as (beta, w, a) with beta fastest for 'R', which is the layout
// the factor of the gauge move comes out in.
void mps_apply_mpo(Context& c, const MpoDev& ops, const MpsDev& src, MpsDev& dst, int cutD, bool dagger, char dir,
                   double* disc) {
  const int L = src.L;
  MPSGPU_CHECK(ops.L == L, MPSGPU_BAD_SHAPE, "apply MPO: lengths differ");
  MPSGPU_CHECK(dir == 'L' || dir == 'R', MPSGPU_INVALID, "apply MPO: direction must be 'L' or 'R'");
  for (int k = 0; k < L; k++) {
    const auto& w = ops.dims[k];
    MPSGPU_CHECK(src.dims[k][0] == (dagger ? w[0] : w[2]), MPSGPU_BAD_SHAPE, "apply MPO: physical dimensions");
  }
  MPSGPU_CHECK(ops.dims[0][1] == 1 && ops.dims[L - 1][3] == 1, MPSGPU_BAD_SHAPE, "apply MPO: open boundary bonds");
  mps_copy(c, src, dst);
  if (disc) *disc = 0.0;
  DBuf link, nlink, Wt;
  int lr = 1, lw = 1, lb = 1;  // link dims: 'L' (r, w, beta), 'R' (beta, w, a)
  dbuf_reserve(c, link, 1);
  const cplx one = make_double2(1.0, 0.0);
  MPSGPU_CUDA(cudaMemcpyAsync(link.p, &one, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
  double last = 1.0;
  try {
    for (int step = 0; step < L; step++) {
      const int pos = dir == 'L' ? L - 1 - step : step;
      const auto od = dst.dims[pos];
      const int d = od[0], Dl = od[1], Dr = od[2];
      const auto& w4 = ops.dims[pos];
      const int du = dagger ? w4[2] : w4[0], wl = w4[1], wr = w4[3];
      // operator as the matrices the two directions need, conjugate-transposed
      // on the physical legs when dagger (W^dag(u, b, s, c) = conj(W(s, b, u, c)))
      const cplx* Wsrc = ops.W[pos].p;
      const long long su = 1, sb = w4[0], ss = (long long)w4[0] * wl, sc = (long long)w4[0] * wl * w4[2];
      const long long s_u = dagger ? ss : su, s_s = dagger ? su : ss;  // strides of (u, s) in W
      View2 v;
      v.conj = dagger;
      GemmArgs g;
      if (dir == 'L') {
        MPSGPU_CHECK(lr == Dr && lw == wr, MPSGPU_BAD_SHAPE, "apply MPO: link mismatch");
        // T1(a, s, c, beta) = X(a s x r) . link(r x c beta)
        dbuf_reserve(c, c.t1, (long long)Dl * d * wr * lb);
        g = GemmArgs();
        g.M = Dl * d; g.N = wr * lb; g.K = Dr;
        g.A = dst.A[pos].p; g.lda = (long long)Dl * d;
        g.B = link.p; g.ldb = Dr;
        g.C = c.t1.p; g.ldc = (long long)Dl * d;
        zgemm(c.st(), g, c.scratch);
        // P(s, c, a, beta)
        dbuf_reserve(c, c.t2, (long long)d * wr * Dl * lb);
        View2 p;
        p.rd = d; p.r0 = Dl; p.r1 = (long long)Dl * d; p.cd = Dl; p.c0 = 1; p.c1 = (long long)Dl * d * wr;
        gather2(c.st(), d * wr, Dl * lb, c.t1.p, p, c.t2.p);
        // Wm(u b x s c)
        dbuf_reserve(c, Wt, (long long)du * wl * d * wr);
        v.rd = du; v.r0 = s_u; v.r1 = sb; v.cd = d; v.c0 = s_s; v.c1 = sc;
        gather2(c.st(), du * wl, d * wr, Wsrc, v, Wt.p);
        // T2(u, b, a, beta) = Wm . P
        dbuf_reserve(c, c.t4, (long long)du * wl * Dl * lb);
        g = GemmArgs();
        g.M = du * wl; g.N = Dl * lb; g.K = d * wr;
        g.A = Wt.p; g.lda = (long long)du * wl;
        g.B = c.t2.p; g.ldb = (long long)d * wr;
        g.C = c.t4.p; g.ldc = (long long)du * wl;
        zgemm(c.st(), g, c.scratch);
        // new site X'(b a, u, beta): left bond b + wl a
        dst.dims[pos] = {du, wl * Dl, lb};
        dbuf_reserve(c, dst.A[pos], nel(dst.dims[pos]));
        View2 q;
        q.rd = wl; q.r0 = du; q.r1 = (long long)du * wl; q.cd = du; q.c0 = 1; q.c1 = (long long)du * wl * Dl;
        gather2(c.st(), wl * Dl, du * lb, c.t4.p, q, dst.A[pos].p);
        const int n = wl * Dl;
        double scalar = -1.0;
        const int K = gauge_factor(c, dst, pos, 'L', &scalar, nullptr, cutD > 0 ? cutD : Dl * wl, disc);
        if (scalar >= 0.0) {
          const cplx sc1 = make_double2(scalar, 0.0);
          dbuf_reserve(c, nlink, 1);
          MPSGPU_CUDA(cudaMemcpyAsync(nlink.p, &sc1, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
          MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
          last = scalar;
          lr = 1; lw = 1; lb = 1;
        } else {
          // link'(a, b, k) = conj(R'(k, b + wl a)), R' in c.matR (ld K)
          dbuf_reserve(c, nlink, (long long)n * K);
          View2 r;
          r.rd = Dl; r.r0 = (long long)K * wl; r.r1 = K; r.cd = 1; r.c0 = 0; r.c1 = 1; r.conj = true;
          gather2(c.st(), n, K, c.matR.p, r, nlink.p);
          lr = Dl; lw = wl; lb = K;
        }
      } else {
        MPSGPU_CHECK(lr == Dl && lw == wl, MPSGPU_BAD_SHAPE, "apply MPO: link mismatch");
        // T1(beta, b, s, r) = link(beta b x a) . X(a x s r)
        dbuf_reserve(c, c.t1, (long long)lb * wl * d * Dr);
        g = GemmArgs();
        g.M = lb * wl; g.N = d * Dr; g.K = Dl;
        g.A = link.p; g.lda = (long long)lb * wl;
        g.B = dst.A[pos].p; g.ldb = Dl;
        g.C = c.t1.p; g.ldc = (long long)lb * wl;
        zgemm(c.st(), g, c.scratch);
        // P(b, s, beta, r)
        dbuf_reserve(c, c.t2, (long long)wl * d * lb * Dr);
        View2 p;
        p.rd = wl; p.r0 = lb; p.r1 = (long long)lb * wl; p.cd = lb; p.c0 = 1; p.c1 = (long long)lb * wl * d;
        gather2(c.st(), wl * d, lb * Dr, c.t1.p, p, c.t2.p);
        // Wm(u c x b s)
        dbuf_reserve(c, Wt, (long long)du * wr * wl * d);
        v.rd = du; v.r0 = s_u; v.r1 = sc; v.cd = wl; v.c0 = sb; v.c1 = s_s;
        gather2(c.st(), du * wr, wl * d, Wsrc, v, Wt.p);
        // T2(u, c, beta, r) = Wm . P
        dbuf_reserve(c, c.t4, (long long)du * wr * lb * Dr);
        g = GemmArgs();
        g.M = du * wr; g.N = lb * Dr; g.K = wl * d;
        g.A = Wt.p; g.lda = (long long)du * wr;
        g.B = c.t2.p; g.ldb = (long long)wl * d;
        g.C = c.t4.p; g.ldc = (long long)du * wr;
        zgemm(c.st(), g, c.scratch);
        // new site X'(beta, u, c r): right bond c + wr r
        dst.dims[pos] = {du, lb, wr * Dr};
        dbuf_reserve(c, dst.A[pos], nel(dst.dims[pos]));
        View2 q;
        q.rd = lb; q.r0 = (long long)du * wr; q.r1 = 1; q.cd = wr; q.c0 = du; q.c1 = (long long)du * wr * lb;
        gather2(c.st(), lb * du, wr * Dr, c.t4.p, q, dst.A[pos].p);
        const int n = wr * Dr;
        double scalar = -1.0;
        const int K = gauge_factor(c, dst, pos, 'R', &scalar, nullptr, cutD > 0 ? cutD : Dr * wr, disc);
        if (scalar >= 0.0) {
          const cplx sc1 = make_double2(scalar, 0.0);
          dbuf_reserve(c, nlink, 1);
          MPSGPU_CUDA(cudaMemcpyAsync(nlink.p, &sc1, sizeof(cplx), cudaMemcpyHostToDevice, c.stream));
          MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
          last = scalar;
          lr = 1; lw = 1; lb = 1;
        } else {
          // link'(k, c, r) = R(k, c + wr r): the factor as it stands
          dbuf_reserve(c, nlink, (long long)K * n);
          zcopy(c.st(), K * n, c.matR.p, nlink.p);
          lr = Dr; lw = wr; lb = K;
        }
      }
      std::swap(link, nlink);
    }
    MPSGPU_CHECK(lr == 1 && lw == 1 && lb == 1, MPSGPU_BAD_SHAPE, "apply MPO: final factor is not a scalar");
  } catch (...) {
    dbuf_free(c, link);
    dbuf_free(c, nlink);
    dbuf_free(c, Wt);
    throw;
  }
  dbuf_free(c, link);
  dbuf_free(c, nlink);
  dbuf_free(c, Wt);
  dst.normfact = src.normfact * last;
  dst.gauge = dir == 'L' ? 1 : 2;
  // applyExactly leaves the bond field alone; truncate lowers it to the
  // largest bond present (MPS.cpp:919,934)
  if (cutD > 0) dst.bond = std::min(src.bond > 0 ? src.bond : dst.max_bond(), dst.max_bond());
}

// Prologue of findGroundState / optimize (Contractor.cpp:1362-1373): pad the
// bonds up to D, or cut the state down to D (init = MPS(init, D)), then
// gauge to the right and back to the left.
static void prepare_init(Context& c, MpsDev& init, int D) {
  if (D > 0) {
    if (D > init.bond) {
      mps_increase_bond(c, init, D);
    } else if (D < init.bond) {
      mps_gauge_all(c, init, 'L', false, D, nullptr);
      init.bond = init.max_bond();
    }
  }
  mps_gauge_all(c, init, 'R', true);
  mps_gauge_all(c, init, 'L', true);
}

namespace {

// The single-site ground-state sweep of Contractor::findGroundState
// (Contractor.cpp:1352-1533) as a state machine: prepare() builds the local
// eigenproblem of the current site (environments, and the product that
// effective Hamiltonian applies), finish() takes its lowest eigenvalue and
// moves on (energy-increase guard, gauge move, convergence at the chain
// ends), so that the sweeps of several chains at the same site can share
// the launches of their local eigensolvers (lanczos_batch).
//
// Mixed precision (opt.precision == 1): split-precision products while the
// sweep is far from convergence, FP64 from the half-sweep after the energy
// change first falls below kSplitSwitchTol; the FP64 phase ends by the
// reference's test, after at least one full FP64 round.  Energies in the
// split phase carry the products' error (about 1e-7 relative), so its
// eigensolver tolerance and energy-increase margin are set at that level,
// and the first FP64 round is not tested for an increase.  precision 2:
// the same schedule of tolerances with FP64 products (to separate what the
// schedule saves from what the tensor cores save).
struct GsSweep {
  Context& c;         // the sweep's own work (environments, gauge moves)
  Context* mc = &c;   // the context running the batch's Lanczos rounds
  const MpoDev& ops;
  MpsDev& init;
  const SolveOptions& opt;
  Counters& cnt;
  LzWork& ws;
  int D = 0, L = 0;
  double offset = 0.0, tol = 1e-12;
  EnvCache E;
  double energy = 0.0, val = 0.0;
  bool right = true, done = false;
  int pos = 0, round = 0;
  bool split_phase = false, split_products = false, first64 = false;
  SplitMatvec smv;
  // the current site
  const cplx* Le = nullptr;
  const cplx* Rt = nullptr;
  std::array<int, 3> ld{}, rd{};

  GsSweep(Context& c_, const MpoDev& ops_, int D_, MpsDev& init_, double offset_, const SolveOptions& opt_,
          Counters& cnt_, LzWork& ws_)
      : c(c_), ops(ops_), init(init_), opt(opt_), cnt(cnt_), ws(ws_), D(D_), L(ops_.L), offset(offset_) {}

  void begin() {
    MPSGPU_CHECK(init.L == L, MPSGPU_BAD_SHAPE, "findGroundState: lengths differ");
    for (int k = 0; k < L; k++)
      MPSGPU_CHECK(init.dims[k][0] == ops.dims[k][2] && ops.dims[k][0] == ops.dims[k][2], MPSGPU_BAD_SHAPE,
                   "findGroundState: physical dimensions differ");
    prepare_init(c, init, D);
    E.init(c, L);
    energy = contract(c, init, &ops, init).x;
    val = energy;
    tol = opt.eigtol > 0 ? opt.eigtol : (opt.precision == 1 || opt.precision == 2) ? kScheduleEigTol : 1e-12;
    split_phase = (opt.precision == 1 || opt.precision == 2);
    split_products = (opt.precision == 1);
    if (split_phase) *c.hsplit_err = *mc->hsplit_err = 0;
  }

  void prepare(LzTask& t) {
    opt.check_cancel();
    calc_left(c, E, pos, &ops, init, init, &cnt);
    calc_right(c, E, pos, &ops, init, init, &cnt);
    Le = E.Le[pos].p;
    Rt = E.Re[pos].p;
    ld = E.ldims[pos];
    rd = E.rdims[pos];
    smv.ready = false;
    if (split_phase && split_products) split_matvec_prepare(c, smv, Le, ld, ops, pos, Rt, rd);
    t = LzTask();
    t.N = (int)nel(init.dims[pos]);
    t.x = init.A[pos].p;
    t.tol = split_phase ? std::max(tol, kSplitEigTol) : first64 ? std::max(tol, kFirst64EigTol) : tol;
    t.shift0 = val + offset;
    t.max_krylov = opt.max_krylov;
    t.ws = &ws;
    t.cnt = &cnt;
    t.product = [this](Context& lc, const cplx* xin, cplx* yout, double sg, RoundBatch& rb) {
      const cplx o = make_double2(offset - sg, 0.0);
      const auto& wd = ops.dims[pos];
      const int du = wd[0], wl = wd[1], dd = wd[2], wr = wd[3];
      const int Dlb = ld[0], Dlk = ld[2], Drk = rd[0], Drb = rd[2];
      MPSGPU_CHECK(ld[1] == wl && rd[1] == wr, MPSGPU_BAD_SHAPE, "heff: MPO bond mismatch");
      cnt.matvecs++;
      cnt.flops += mv_flops(dd, wl, wr, Dlb, Drb);
      if (split_phase && split_products) {
        SplitProduct p;
        p.nh = 1;
        p.sp[0] = &smv;
        p.Wm[0] = ops.Wlr[pos].p;
        p.Dlb = Dlb; p.Dlk = Dlk; p.wl = wl; p.dd = dd; p.Drk = Drk; p.du = du; p.wr = wr; p.Drb = Drb;
        p.x = xin;
        p.y = yout;
        p.offset = o;
        p.ws = &ws;
        rb.sr.p.push_back(p);
        cnt.split_matvecs++;
        return;
      }
      dbuf_reserve(lc, ws.t2, (long long)Dlb * du * Drk * wr);
      rb.g1.d[rb.g1.n++] = heff_first_desc(Le, Dlb, Dlk, wl, xin, dd, Drk, ops.Wlr[pos].p, du, wr, ws.t2.p);
      rb.g3.d[rb.g3.n++] = heff_last_desc(ws.t2.p, Dlb * du, Rt, Drk * wr, Drb, yout, xin, o);
    };
  }

  void finish(double theta) {
    cnt.site_solves++;
    if (split_phase && (*c.hsplit_err || *mc->hsplit_err))
      throw Error(MPSGPU_TIMEOUT, "findGroundState: a bounded wait in the tensor-core kernel ran out");
    val = theta - offset;
    if (!first64 && (val - energy > 1e-8) && (val - energy > std::fabs(energy + offset) * 1e-10)) {
      const double margin = split_phase ? std::max(opt.convtol, kSplitIncreaseTol) : opt.convtol;
      if (val - energy > std::fabs(energy + offset) * margin)
        throw Error(MPSGPU_ENERGY_INCREASE, "findGroundState: energy increasing");
    }
    mps_gauge_site(c, init, pos, right ? 'R' : 'L', true, &cnt);
    for (int l = pos + 1; l < L; l++) E.outofdate_l(l);
    for (int l = pos - 1; l >= 0; l--) E.outofdate_r(l);
    const bool at_end = right ? (pos == L - 1) : (pos == 0);
    if (at_end) {
      const double change = std::fabs(energy - val);
      const bool was_split = split_phase;
      done = change < opt.convtol * std::fabs(energy + offset);
      if (!done && std::fabs(val) < 1e-13) done = true;
      if (split_phase) {
        cnt.split_rounds++;
        if (change < std::max(opt.convtol, kSplitSwitchTol) * std::fabs(energy + offset)) {
          split_phase = false;
          first64 = true;
        }
        done = false;
      } else if (first64) {
        // the first FP64 half-sweep was compared with a split-phase energy
        first64 = false;
        done = false;
      }
      energy = val;
      if (opt.verbose) printf("mpsgpu: round %d energy %.15g%s\n", round, val, was_split ? " (split)" : "");
      if (!done) {
        mps_gauge_site(c, init, pos, right ? 'L' : 'R', true, &cnt);
        pos += right ? -1 : 1;
      }
      right = !right;
      round++;
      // intermediate result every checkpoint_every half-sweeps (Contractor.cpp:1526-1530)
      if (!done && !opt.checkpoint.empty() && round % std::max(1, opt.checkpoint_every) == 0)
        mps_export_file(c, init, opt.checkpoint);
    } else {
      pos += right ? 1 : -1;
    }
    if (!done && round >= opt.max_rounds) throw Error(MPSGPU_NOT_CONVERGED, "findGroundState: round limit reached");
  }

  void release() {
    E.release(c);
    split_matvec_release(c, smv);
    cnt.rounds += round;
  }
};

// Drives sweeps that share the same site positions: each round of site
// steps prepares every live sweep, solves all their local problems in one
// lanczos_batch and lets each sweep finish its step.  A sweep that fails
// stops with its own status; the others go on.
template <class Sweep>
void run_sweeps(Context& c, std::vector<Sweep*>& sw, std::vector<int>& status, std::vector<std::string>& err) {
  // c runs the Lanczos rounds; a sweep on a sub-context hands its prepared
  // site over through an event on its stream
  const int n = (int)sw.size();
  status.assign(n, MPSGPU_OK);
  err.assign(n, std::string());
  auto fail = [&](int i, const Error& e) {
    status[i] = e.status;
    err[i] = e.what();
  };
  std::vector<char> live(n, 1);
  for (int i = 0; i < n; i++) {
    try {
      sw[i]->begin();
    } catch (const Error& e) {
      fail(i, e);
      live[i] = 0;
    }
  }
  std::vector<LzTask> tasks(n);
  for (;;) {
    std::vector<LzTask*> tp;
    std::vector<int> idx;
    for (int i = 0; i < n; i++) {
      if (!live[i] || sw[i]->done) continue;
      try {
        sw[i]->prepare(tasks[i]);
        tp.push_back(&tasks[i]);
        idx.push_back(i);
      } catch (const Error& e) {
        fail(i, e);
        live[i] = 0;
      }
    }
    if (tp.empty()) break;
    for (int i : idx) {
      Context& sc = sw[i]->c;
      if (&sc == &c) continue;
      MPSGPU_CUDA(cudaEventRecord(sc.ev, sc.stream));
      MPSGPU_CUDA(cudaStreamWaitEvent(c.stream, sc.ev, 0));
    }
    try {
      lanczos_batch(c, tp);
    } catch (const Error& e) {
      // the round's local problems are lost: every sweep in it stops
      for (int i : idx) {
        fail(i, e);
        live[i] = 0;
      }
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
      continue;
    }
    for (size_t q = 0; q < idx.size(); q++) {
      const int i = idx[q];
      try {
        sw[i]->finish(tasks[i].theta);
      } catch (const Error& e) {
        fail(i, e);
        live[i] = 0;
      }
    }
  }
  for (int i = 0; i < n; i++) sw[i]->release();
}

}  // namespace

double find_ground_state(Context& c, const MpoDev& ops, int D, MpsDev& init, double offset,
                         const SolveOptions& opt, Counters& cnt) {
  GsSweep s(c, ops, D, init, offset, opt, cnt, c.lzone);
  std::vector<GsSweep*> sw{&s};
  std::vector<int> status;
  std::vector<std::string> err;
  run_sweeps(c, sw, status, err);
  if (status[0] != MPSGPU_OK) throw Error((mpsgpu_status)status[0], err[0]);
  return s.energy;
}

void find_ground_state_batch(Context& c, const std::vector<const MpoDev*>& ops, int D, std::vector<MpsDev*>& inits,
                             double offset, const SolveOptions& opt, std::vector<double>& energies,
                             std::vector<Counters>& cnts, std::vector<int>& status, std::vector<std::string>& err) {
  const int n = (int)inits.size();
  MPSGPU_CHECK(n >= 1 && (int)ops.size() == n, MPSGPU_INVALID, "findGroundState batch: sizes");
  cnts.assign(n, Counters());
  std::vector<LzWork> ws(n);
  std::vector<std::unique_ptr<GsSweep>> own;
  std::vector<GsSweep*> sw;
  for (int i = 0; i < n; i++) {
    // each sweep's environments and gauge moves on its own stream
    Context& sc = n > 1 ? context_sub(c, i) : c;
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    own.emplace_back(new GsSweep(sc, *ops[i], D, *inits[i], offset, opt, cnts[i], ws[i]));
    own.back()->mc = &c;
    sw.push_back(own.back().get());
  }
  try {
    run_sweeps(c, sw, status, err);
  } catch (...) {
    for (auto& w : ws) w.release(c);
    throw;
  }
  energies.assign(n, 0.0);
  for (int i = 0; i < n; i++) energies[i] = sw[i]->energy;
  for (auto* x : sw) MPSGPU_CUDA(cudaStreamSynchronize(x->c.stream));  // the states are read on c next
  for (auto& w : ws) w.release(c);
}

// ---------------------------------------------------------------------------
// Two-site DMRG (no counterpart in the reference, whose sweeps are single
// site): the bond between sites k and k+1 is optimised as one tensor
// Theta(a, s1, s2, r) and split by a cut SVD, so bonds grow up to D and the
// discarded weight of every cut is known.
// ---------------------------------------------------------------------------

// y = L W_k W_{k+1} R x for x = Theta (device layout a, s1, s2, r):
//   T1[(a',b),(s1,s2,r)] = L . X                          GEMM
//   T2[a',s1',c,(s2,r)]  = sum_{b,s1} W_k[s1',b,s1,c] T1    leg kernel
//   T3[(a',s1'),s2',r,e] = sum_{c,s2} W_k+1[s2',c,s2,e] T2  leg kernel
//   Y[(a',s1',s2'),r']   = T3 . Rt + offset X              GEMM
static void heff2_apply(Context& c, const cplx* Le, const std::array<int, 3>& ld, const MpoDev& m, int k,
                        const cplx* Rt, const std::array<int, 3>& rd, const cplx* x, cplx* y, cplx offset,
                        Counters* cnt) {
  const auto& w1 = m.dims[k];
  const auto& w2 = m.dims[k + 1];
  const int du1 = w1[0], wl = w1[1], d1 = w1[2], wc = w1[3];
  const int du2 = w2[0], d2 = w2[2], we = w2[3];
  const int Dlb = ld[0], Dlk = ld[2], Drk = rd[0], Drb = rd[2];
  MPSGPU_CHECK(ld[1] == wl && rd[1] == we && w2[1] == wc, MPSGPU_BAD_SHAPE, "heff2: MPO bond mismatch");
  dbuf_reserve(c, c.t1, (long long)Dlb * wl * d1 * d2 * Drk);
  GemmArgs g;
  g.M = Dlb * wl; g.N = d1 * d2 * Drk; g.K = Dlk;
  g.A = Le; g.lda = (long long)Dlb * wl;
  g.B = x; g.ldb = Dlk;
  g.C = c.t1.p; g.ldc = (long long)Dlb * wl;
  zgemm(c.st(), g, c.scratch);
  dbuf_reserve(c, c.t2, (long long)Dlb * du1 * wc * d2 * Drk);
  WContractArgs a1;
  a1.nx = Dlb; a1.ny = d2 * Drk;
  a1.in = c.t1.p; a1.ix = 1; a1.iy = (long long)Dlb * wl * d1; a1.si0 = Dlb; a1.si1 = (long long)Dlb * wl;
  a1.n_i0 = wl; a1.n_i1 = d1;
  a1.out = c.t2.p; a1.ox = 1; a1.oy = (long long)Dlb * du1 * wc; a1.so0 = Dlb; a1.so1 = (long long)Dlb * du1;
  a1.n_o0 = du1; a1.n_o1 = wc;
  a1.Wm = m.Wlr[k].p;
  wcontract(c.st(), a1);
  dbuf_reserve(c, c.t3, (long long)Dlb * du1 * du2 * Drk * we);
  WContractArgs a2;
  a2.nx = Dlb * du1; a2.ny = Drk;
  a2.in = c.t2.p; a2.ix = 1; a2.iy = (long long)Dlb * du1 * wc * d2;
  a2.si0 = (long long)Dlb * du1; a2.si1 = (long long)Dlb * du1 * wc;
  a2.n_i0 = wc; a2.n_i1 = d2;
  a2.out = c.t3.p; a2.ox = 1; a2.oy = (long long)Dlb * du1 * du2;
  a2.so0 = (long long)Dlb * du1; a2.so1 = (long long)Dlb * du1 * du2 * Drk;
  a2.n_o0 = du2; a2.n_o1 = we;
  a2.Wm = m.Wlr[k + 1].p;
  wcontract(c.st(), a2);
  GemmArgs h;
  h.M = Dlb * du1 * du2; h.N = Drb; h.K = Drk * we;
  h.A = c.t3.p; h.lda = (long long)Dlb * du1 * du2;
  h.B = Rt; h.ldb = (long long)Drk * we;
  h.C = y; h.ldc = (long long)Dlb * du1 * du2;
  if (offset.x != 0.0 || offset.y != 0.0) {
    h.Cin = x; h.ldcin = (long long)Dlb * du1 * du2; h.beta = offset;
  }
  zgemm(c.st(), h, c.scratch);
  if (cnt) {
    cnt->matvecs++;
    cnt->flops += 8.0 * ((double)Dlb * wl * Dlk * d1 * d2 * Drk + (double)Dlb * du1 * wc * wl * d1 * d2 * Drk +
                         (double)Dlb * du1 * du2 * we * wc * d2 * Drk + (double)Dlb * du1 * du2 * Drk * we * Drb);
  }
}

double find_ground_state_two_site(Context& c, const MpoDev& ops, int D, MpsDev& init, double offset,
                                  const SolveOptions& opt, Counters& cnt, double* max_discarded) {
  const int L = ops.L;
  MPSGPU_CHECK(L >= 2 && init.L == L, MPSGPU_BAD_SHAPE, "two-site DMRG: lengths");
  MPSGPU_CHECK(D > 0, MPSGPU_INVALID, "two-site DMRG: D must be positive");
  for (int k = 0; k < L; k++)
    MPSGPU_CHECK(init.dims[k][0] == ops.dims[k][2] && ops.dims[k][0] == ops.dims[k][2], MPSGPU_BAD_SHAPE,
                 "two-site DMRG: physical dimensions differ");
  // start from a normalised right-canonical state; the cut SVDs set the bonds
  if (init.bond > D) {
    mps_gauge_all(c, init, 'L', false, D, nullptr);
    init.bond = init.max_bond();
  }
  mps_gauge_all(c, init, 'R', true);
  mps_gauge_all(c, init, 'L', true);
  EnvCache E;
  E.init(c, L);
  DBuf th;
  double energy = contract(c, init, &ops, init).x;
  double val = energy, dmax = 0.0;
  bool right = true, done = false;
  int pos = 0, round = 0;
  const double tol = opt.eigtol > 0 ? opt.eigtol : 1e-12;
  const cplx off = make_double2(offset, 0.0);
  try {
    while (!done) {
      opt.check_cancel();
      calc_left(c, E, pos, &ops, init, init, &cnt);
      calc_right(c, E, pos + 1, &ops, init, init, &cnt);
      const auto da = init.dims[pos], db = init.dims[pos + 1];
      const int Dl = da[1], d1 = da[0], mid = da[2], d2 = db[0], Dr = db[2];
      MPSGPU_CHECK(db[1] == mid, MPSGPU_BAD_SHAPE, "two-site DMRG: bond mismatch");
      const long long N = (long long)Dl * d1 * d2 * Dr;
      dbuf_reserve(c, th, N);
      GemmArgs g;
      g.M = Dl * d1; g.N = d2 * Dr; g.K = mid;
      g.A = init.A[pos].p; g.lda = (long long)Dl * d1;
      g.B = init.A[pos + 1].p; g.ldb = mid;
      g.C = th.p; g.ldc = (long long)Dl * d1;
      zgemm(c.st(), g, c.scratch);
      const cplx* Le = E.Le[pos].p;
      const cplx* Rt = E.Re[pos + 1].p;
      const auto ld = E.ldims[pos];
      const auto rd = E.rdims[pos + 1];
      auto apply = [&](const cplx* xin, cplx* yout, double sg) {
        heff2_apply(c, Le, ld, ops, pos, Rt, rd, xin, yout, make_double2(off.x - sg, off.y), &cnt);
      };
      int its = 0;
      const double theta = lanczos_lowest(c, (int)N, apply, th.p, tol, opt.max_krylov, &its, val + offset, &cnt);
      cnt.site_solves++;
      val = theta - offset;
      // split Theta (Dl d1 x d2 Dr) = U S V^H, cut to D; the singular values
      // go right on a right move and left on a left move
      const int m = Dl * d1, n = d2 * Dr;
      const int Kmax = std::min(m, n);
      dbuf_reserve(c, c.matQ, (long long)m * Kmax);
      dbuf_reserve(c, c.matR, (long long)Kmax * n);
      std::vector<double> sv;
      const int K = svd_cut(c.st(), m, n, th.p, m, D, c.matQ.p, c.matR.p, sv, c.scratch, !right);
      double dw = 0.0, tot = 0.0;
      for (size_t j = 0; j < sv.size(); j++) {
        tot += sv[j] * sv[j];
        if ((int)j >= K) dw += sv[j] * sv[j];
      }
      if (tot > 0) dmax = std::max(dmax, dw / tot);
      init.dims[pos] = {d1, Dl, K};
      init.dims[pos + 1] = {d2, K, Dr};
      dbuf_reserve(c, init.A[pos], (long long)m * K);
      dbuf_reserve(c, init.A[pos + 1], (long long)K * n);
      zcopy(c.st(), m * K, c.matQ.p, init.A[pos].p);
      zcopy(c.st(), K * n, c.matR.p, init.A[pos + 1].p);
      for (int l = pos + 1; l < L; l++) E.outofdate_l(l);
      for (int l = pos; l >= 0; l--) E.outofdate_r(l);
      const bool at_end = (right && pos == L - 2) || (!right && pos == 0);
      if (at_end) {
        done = std::fabs(energy - val) < opt.convtol * std::fabs(energy + offset);
        if (!done && std::fabs(val) < 1e-13) done = true;
        energy = val;
        if (opt.verbose) printf("mpsgpu: two-site round %d energy %.15g max discarded %.3g\n", round, val, dmax);
        right = !right;  // the same bond is solved again in the new direction
        round++;
        if (!done && round >= opt.max_rounds)
          throw Error(MPSGPU_NOT_CONVERGED, "two-site DMRG: round limit reached");
      } else {
        pos += right ? 1 : -1;
      }
    }
  } catch (...) {
    E.release(c);
    dbuf_free(c, th);
    throw;
  }
  E.release(c);
  dbuf_free(c, th);
  init.bond = init.max_bond();
  init.gauge = 0;
  init.normfact = 1.0;
  cnt.rounds += round;
  if (max_discarded) *max_discarded = dmax;
  return energy;
}

}  // namespace mpsgpu

namespace mpsgpu {

// ---------------------------------------------------------------------------
// Excited states: findNextExcitedState (Contractor.cpp:2676-2727) and
// findGroundStateWithProjectorPenalty (:2739-2956) with the Hermitian,
// projected multiplier TensorMultiplierProjMulti(hermitian=true)
// (TensorMultiplierProjMulti.cpp:81-90):
//   y = 1/2 (H x + H^dag x) + sum_k pen_k u_k (u_k^H x) + offset x,
// u_k = the level-k state contracted with the norm environments
// (Contractor::contractMbraId, Contractor.cpp:880-903).
// ---------------------------------------------------------------------------

namespace {

constexpr int MAX_ROUND_EXCTD = 1000;  // Contractor.cpp:26

struct LevelCache {
  EnvCache n;  // w = 1 environments between init (ket) and the level (bra)
};

}  // namespace

namespace {

// findGroundStateWithProjectorPenalty (Contractor.cpp:2739-2956) as a state
// machine (see GsSweep), with the Hermitian, projected multiplier
// TensorMultiplierProjMulti(hermitian=true) (TensorMultiplierProjMulti.cpp:
// 81-90).  Mixed precision as in GsSweep: split-precision products of both
// halves of the Hermitian multiplier until the half-sweep energy settles,
// then FP64 (at least one full round).
struct ExcSweep {
  Context& c;         // the sweep's own work (environments, gauge moves)
  Context* mc = &c;   // the context running the batch's Lanczos rounds
  const MpoDev& ops;
  MpsDev& init;
  const SolveOptions& opt;
  Counters& cnt;
  LzWork& ws;
  std::vector<double> pens;
  std::vector<const MpsDev*> levels;
  int D = 0, L = 0, nk = 0;
  double offset = 0.0, tol = 1e-12;
  EnvCache E;
  std::vector<EnvCache> NC;
  DBuf Lh, Rth, U;
  double energy = 0.0, val = 0.0;
  bool right = true, done = false;
  int pos = 0, round = 0;
  bool split_phase = false, split_products = false, first64 = false;
  SplitMatvec smv, smvh;
  std::chrono::steady_clock::time_point last_saved;
  const cplx* Le = nullptr;
  const cplx* Rt = nullptr;
  std::array<int, 3> ld{}, rd{};

  ExcSweep(Context& c_, const MpoDev& ops_, int D_, const std::vector<double>& pens_,
           const std::vector<const MpsDev*>& levels_, MpsDev& init_, double offset_, const SolveOptions& opt_,
           Counters& cnt_, LzWork& ws_)
      : c(c_), ops(ops_), init(init_), opt(opt_), cnt(cnt_), ws(ws_), pens(pens_), levels(levels_), D(D_),
        L(ops_.L), nk((int)levels_.size()), offset(offset_) {}

  void begin() {
    MPSGPU_CHECK(nk <= LZ_MAXU, MPSGPU_BAD_SHAPE, "findNextExcitedState: at most 8 computed levels");
    prepare_init(c, init, D);
    energy = contract(c, init, &ops, init).x + offset;
    for (int k = 0; k < nk; k++) {
      cplx ov = contract(c, init, nullptr, *levels[k]);
      energy += pens[k] * cabs2(ov);
    }
    energy -= offset;
    E.init(c, L);
    NC.resize(nk);
    for (auto& n : NC) n.init(c, L);
    val = energy;
    tol = opt.eigtol > 0 ? opt.eigtol : (opt.precision == 1 || opt.precision == 2) ? kScheduleEigTol : 1e-12;
    split_phase = (opt.precision == 1 || opt.precision == 2);
    split_products = (opt.precision == 1);
    if (split_phase) *c.hsplit_err = *mc->hsplit_err = 0;
    last_saved = std::chrono::steady_clock::now();
  }

  void prepare(LzTask& t) {
    opt.check_cancel();
    // calculateLexck / calculateRexck (Contractor.cpp:2958-2988): one set of flags
    {
      std::vector<int> needL, needR;
      int p = pos;
      while (!E.okL[p]) needL.push_back(p--);
      for (int q = (int)needL.size() - 1; q >= 0; q--) {
        const int pp = needL[q];
        env_left_update(c, E.Le[pp - 1].p, E.ldims[pp - 1], init, &ops, pp - 1, init, E.Le[pp], E.ldims[pp], &cnt);
        for (int k = 0; k < nk; k++)
          env_left_update(c, NC[k].Le[pp - 1].p, NC[k].ldims[pp - 1], init, nullptr, pp - 1, *levels[k],
                          NC[k].Le[pp], NC[k].ldims[pp], &cnt);
        E.okL[pp] = 1;
      }
      p = pos;
      while (!E.okR[p]) needR.push_back(p++);
      for (int q = (int)needR.size() - 1; q >= 0; q--) {
        const int pp = needR[q];
        env_right_update(c, E.Re[pp + 1].p, E.rdims[pp + 1], init, &ops, pp + 1, init, E.Re[pp], E.rdims[pp], &cnt);
        for (int k = 0; k < nk; k++)
          env_right_update(c, NC[k].Re[pp + 1].p, NC[k].rdims[pp + 1], init, nullptr, pp + 1, *levels[k],
                           NC[k].Re[pp], NC[k].rdims[pp], &cnt);
        E.okR[pp] = 1;
      }
    }
    const auto dims = init.dims[pos];
    const int N = (int)nel(dims);
    const int Dlk = dims[1], d = dims[0], Drk = dims[2];
    ld = E.ldims[pos];
    rd = E.rdims[pos];
    // adjoint environments: L^dag(bra,w,ket) = conj(L(ket,w,bra)), Rt^dag likewise
    dbuf_reserve(c, Lh, nel(ld));
    dbuf_reserve(c, Rth, nel(rd));
    transpose_pqr_to_rqp(c.st(), ld[0], ld[1], ld[2], E.Le[pos].p, Lh.p, true);
    transpose_pqr_to_rqp(c.st(), rd[0], rd[1], rd[2], E.Re[pos].p, Rth.p, true);
    // projector vectors u_k (sqrt(pen_k) folded in), columns of U (N x nk)
    // (Contractor::contractMbraId, Contractor.cpp:880-903)
    dbuf_reserve(c, U, (long long)N * nk);
    for (int k = 0; k < nk; k++) {
      const MpsDev& lv = *levels[k];
      const auto bd = lv.dims[pos];
      const auto nl = NC[k].ldims[pos];  // (Dlb, 1, Dlk)
      const auto nr = NC[k].rdims[pos];  // (Drk, 1, Drb)
      dbuf_reserve(c, c.t3, (long long)Dlk * d * bd[2]);
      GemmArgs g1;
      g1.M = Dlk; g1.N = d * bd[2]; g1.K = nl[0];
      g1.A = NC[k].Le[pos].p; g1.lda = nl[0]; g1.opA = OP_C;
      g1.B = lv.A[pos].p; g1.ldb = bd[1];
      g1.C = c.t3.p; g1.ldc = Dlk;
      zgemm(c.st(), g1, c.scratch);
      GemmArgs g2;
      g2.M = Dlk * d; g2.N = Drk; g2.K = bd[2];
      g2.A = c.t3.p; g2.lda = (long long)Dlk * d;
      g2.B = NC[k].Re[pos].p; g2.ldb = nr[0]; g2.opB = OP_C;
      g2.C = U.p + (long long)k * N; g2.ldc = (long long)Dlk * d;
      g2.alpha = make_double2(std::sqrt(pens[k]), 0.0);
      zgemm(c.st(), g2, c.scratch);
    }
    Le = E.Le[pos].p;
    Rt = E.Re[pos].p;
    smv.ready = smvh.ready = false;
    if (split_phase && split_products) {
      split_matvec_prepare(c, smv, Le, ld, ops, pos, Rt, rd);
      split_matvec_prepare(c, smvh, Lh.p, ld, ops, pos, Rth.p, rd);
    }
    t = LzTask();
    t.N = N;
    t.x = init.A[pos].p;
    t.tol = split_phase ? std::max(tol, kSplitEigTol) : first64 ? std::max(tol, kFirst64EigTol) : tol;
    t.shift0 = val + offset;
    t.max_krylov = opt.max_krylov;
    t.U = U.p;
    t.nu = nk;
    t.ws = &ws;
    t.cnt = &cnt;
    // 1/2 (H + H^dag) x + (offset - sigma) x; the projector term
    // sum_k pen_k u_k (u_k^H x) is added by the Lanczos step
    t.product = [this](Context& lc, const cplx* xin, cplx* yout, double sg, RoundBatch& rb) {
      const cplx o = make_double2(offset - sg, 0.0);
      const auto& wd = ops.dims[pos];
      const int du = wd[0], wl = wd[1], dd = wd[2], wr = wd[3];
      const int Dlb = ld[0], Dlk_ = ld[2], Drk_ = rd[0], Drb = rd[2];
      MPSGPU_CHECK(ld[1] == wl && rd[1] == wr && ops.Wlr_h[pos].p, MPSGPU_BAD_SHAPE, "heff: MPO bond mismatch");
      cnt.matvecs++;
      cnt.flops += 2.0 * mv_flops(dd, wl, wr, Dlb, Drb);
      if (split_phase && split_products) {
        SplitProduct p;
        p.nh = 2;
        p.sp[0] = &smv;
        p.sp[1] = &smvh;
        p.Wm[0] = ops.Wlr[pos].p;
        p.Wm[1] = ops.Wlr_h[pos].p;
        p.Dlb = Dlb; p.Dlk = Dlk_; p.wl = wl; p.dd = dd; p.Drk = Drk_; p.du = du; p.wr = wr; p.Drb = Drb;
        p.x = xin;
        p.y = yout;
        p.alpha = make_double2(0.5, 0.0);
        p.offset = o;
        p.ws = &ws;
        rb.sr.p.push_back(p);
        cnt.split_matvecs++;
        return;
      }
      const long long n2 = (long long)Dlb * du * Drk_ * wr;
      dbuf_reserve(lc, ws.t2, n2);
      dbuf_reserve(lc, ws.t3, n2);
      rb.g1.d[rb.g1.n++] = heff_first_desc(Le, Dlb, Dlk_, wl, xin, dd, Drk_, ops.Wlr[pos].p, du, wr, ws.t2.p);
      rb.g1.d[rb.g1.n++] = heff_first_desc(Lh.p, Dlb, Dlk_, wl, xin, dd, Drk_, ops.Wlr_h[pos].p, du, wr, ws.t3.p);
      Gemm3Desc h = heff_last_desc(ws.t2.p, Dlb * du, Rt, Drk_ * wr, Drb, yout, xin, o);
      h.K2 = Drk_ * wr;
      h.A2 = ws.t3.p;
      h.lda2 = (long long)Dlb * du;
      h.B2 = Rth.p;
      h.ldb2 = (long long)Drk_ * wr;
      h.alpha = make_double2(0.5, 0.0);
      rb.g3.d[rb.g3.n++] = h;
    };
  }

  void finish(double theta) {
    cnt.site_solves++;
    if (split_phase && (*c.hsplit_err || *mc->hsplit_err))
      throw Error(MPSGPU_TIMEOUT, "findNextExcitedState: a bounded wait in the tensor-core kernel ran out");
    val = theta - offset;
    if (!first64 && (val - energy > 1e-8) && (val - energy > std::fabs(energy + offset) * 1e-10)) {
      const double margin = split_phase ? kSplitIncreaseTol : 1e-6;
      if (val - energy > std::fabs(energy + offset) * margin)
        throw Error(MPSGPU_ENERGY_INCREASE, "findNextExcitedState: energy increasing");
    }
    mps_gauge_site(c, init, pos, right ? 'R' : 'L', true, &cnt);
    for (int l = pos + 1; l < L; l++) E.outofdate_l(l);
    for (int l = pos - 1; l >= 0; l--) E.outofdate_r(l);
    const bool at_end = (right && pos == L - 1) || (!right && pos == 0);
    if (at_end && !opt.checkpoint.empty()) {
      // save at the end of every half-sweep, or every checkpoint_seconds
      // (Contractor.cpp:2868-2883)
      const auto now = std::chrono::steady_clock::now();
      if (opt.checkpoint_seconds <= 0.0 ||
          std::chrono::duration<double>(now - last_saved).count() >= opt.checkpoint_seconds) {
        mps_export_file(c, init, opt.checkpoint);
        last_saved = now;
      }
    }
    if (at_end) {
      const double change = std::fabs(energy - val);
      const bool was_split = split_phase;
      done = change < opt.convtol * std::fabs(energy + offset);
      if (!done && (change < 1e-12 || round > MAX_ROUND_EXCTD)) done = true;
      if (split_phase) {
        cnt.split_rounds++;
        if (change < std::max(opt.convtol, kSplitSwitchTol) * std::fabs(energy + offset) || round > MAX_ROUND_EXCTD) {
          split_phase = false;
          first64 = true;
        }
        done = false;
      } else if (first64) {
        first64 = false;
        done = false;
      }
      energy = val;
      if (opt.verbose) printf("mpsgpu: excited round %d energy %.15g%s\n", round, val, was_split ? " (split)" : "");
      if (!done) {
        if (right) {
          mps_gauge_site(c, init, pos, 'L', true, &cnt);
          pos--;
        } else {
          mps_gauge_site(c, init, pos, 'R', true, &cnt);
          pos++;
        }
      }
      right = !right;
      round++;
      if (!done && round >= opt.max_rounds)
        throw Error(MPSGPU_NOT_CONVERGED, "findNextExcitedState: round limit reached");
    } else {
      pos += right ? 1 : -1;
    }
  }

  void release() {
    E.release(c);
    for (auto& n : NC) n.release(c);
    for (DBuf* b : {&Lh, &Rth, &U}) dbuf_free(c, *b);
    split_matvec_release(c, smv);
    split_matvec_release(c, smvh);
    cnt.rounds += round;
  }
};

// The penalties of findNextExcitedState (Contractor.cpp:2676-2727): 20 times
// the spread of the levels' energies, or L/2 for a single level.
std::vector<double> excited_penalties(Context& c, const MpoDev& ops, const std::vector<const MpsDev*>& levels,
                                      double offset) {
  const int nk = (int)levels.size();
  double minE = 0, maxE = 0;
  for (int k = 0; k < nk; k++) {
    double e = contract(c, *levels[k], &ops, *levels[k]).x + offset;
    if (k == 0 || e < minE) minE = e;
    if (k == 0 || e > maxE) maxE = e;
  }
  double newOffset = std::max(20 * (maxE - minE), std::fabs(offset));
  if (nk == 1 || newOffset < 1e-6) newOffset = levels[0]->L * 0.5;
  return std::vector<double>(nk, newOffset);
}

void check_levels(const MpoDev& ops, const std::vector<const MpsDev*>& levels, const MpsDev& init) {
  MPSGPU_CHECK(!levels.empty(), MPSGPU_INVALID, "findNextExcitedState: no levels");
  for (auto* lv : levels) MPSGPU_CHECK(lv->L == ops.L, MPSGPU_BAD_SHAPE, "findNextExcitedState: level length");
  MPSGPU_CHECK(init.L == ops.L, MPSGPU_BAD_SHAPE, "findNextExcitedState: init length");
}

// excorthtol > 0: the levels the state still overlaps by more than
// excorthtol get their penalty doubled (true: run again)
bool raise_penalties(Context& c, const std::vector<const MpsDev*>& levels, const MpsDev& init, double excorthtol,
                     std::vector<double>& pens) {
  bool again = false;
  for (size_t k = 0; k < levels.size(); k++) {
    cplx ov = contract(c, init, nullptr, *levels[k]);
    if (std::sqrt(cabs2(ov)) > excorthtol) {
      pens[k] *= 2;
      again = true;
    }
  }
  return again;
}

}  // namespace

double find_next_excited_state(Context& c, const MpoDev& ops, int D, const std::vector<const MpsDev*>& levels,
                               MpsDev& init, double offset, const SolveOptions& opt, Counters& cnt) {
  check_levels(ops, levels, init);
  std::vector<double> pens = excited_penalties(c, ops, levels, offset);
  for (;;) {
    ExcSweep s(c, ops, D, pens, levels, init, offset, opt, cnt, c.lzone);
    std::vector<ExcSweep*> sw{&s};
    std::vector<int> status;
    std::vector<std::string> err;
    run_sweeps(c, sw, status, err);
    if (status[0] != MPSGPU_OK) throw Error((mpsgpu_status)status[0], err[0]);
    if (opt.excorthtol <= 0 || !raise_penalties(c, levels, init, opt.excorthtol, pens)) return s.energy;
  }
}

void find_next_excited_state_batch(Context& c, const std::vector<const MpoDev*>& ops, int D,
                                   const std::vector<std::vector<const MpsDev*>>& levels, std::vector<MpsDev*>& inits,
                                   double offset, const SolveOptions& opt, std::vector<double>& energies,
                                   std::vector<Counters>& cnts, std::vector<int>& status,
                                   std::vector<std::string>& err) {
  const int n = (int)inits.size();
  MPSGPU_CHECK(n >= 1 && (int)ops.size() == n && (int)levels.size() == n, MPSGPU_INVALID,
               "findNextExcitedState batch: sizes");
  cnts.assign(n, Counters());
  energies.assign(n, 0.0);
  status.assign(n, MPSGPU_OK);
  err.assign(n, std::string());
  std::vector<std::vector<double>> pens(n);
  std::vector<int> todo;
  for (int i = 0; i < n; i++) {
    try {
      check_levels(*ops[i], levels[i], *inits[i]);
      pens[i] = excited_penalties(c, *ops[i], levels[i], offset);
      todo.push_back(i);
    } catch (const Error& e) {
      status[i] = e.status;
      err[i] = e.what();
    }
  }
  std::vector<LzWork> ws(n);
  try {
    while (!todo.empty()) {
      std::vector<std::unique_ptr<ExcSweep>> own;
      std::vector<ExcSweep*> sw;
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
      for (int i : todo) {
        Context& sc = n > 1 ? context_sub(c, i) : c;
        own.emplace_back(new ExcSweep(sc, *ops[i], D, pens[i], levels[i], *inits[i], offset, opt, cnts[i], ws[i]));
        own.back()->mc = &c;
        sw.push_back(own.back().get());
      }
      std::vector<int> st;
      std::vector<std::string> er;
      run_sweeps(c, sw, st, er);
      std::vector<int> again;
      for (size_t q = 0; q < todo.size(); q++) {
        const int i = todo[q];
        status[i] = st[q];
        err[i] = er[q];
        energies[i] = sw[q]->energy;
        MPSGPU_CUDA(cudaStreamSynchronize(sw[q]->c.stream));  // the states are read on c next
        if (st[q] == MPSGPU_OK && opt.excorthtol > 0 && raise_penalties(c, levels[i], *inits[i], opt.excorthtol, pens[i]))
          again.push_back(i);
      }
      todo = again;
    }
  } catch (...) {
    for (auto& w : ws) w.release(c);
    throw;
  }
  for (auto& w : ws) w.release(c);
}

// ---------------------------------------------------------------------------
// optimize (Contractor.cpp:77-278): variational |init> ~ ops |orig> at fixed
// bond dimension, the time-evolution step of the reference.
// ---------------------------------------------------------------------------

// Contractor::checkDistanceConvergence (Contractor.cpp:940-999)
// noisy: the distance carries the error of split-precision products, so an
// increase means the sweep has reached that noise floor (it ends the sweep
// instead of failing it)
static bool check_distance(double& distance, cplx c1, cplx c2, double normA, double normB, double convtol,
                           bool noisy = false) {
  const double newd = normA * (normA * c1.x - 2 * c2.x) + normB * normB;
  MPSGPU_CHECK(std::isfinite(newd), MPSGPU_NAN, "optimize: NaN distance");
  bool done = false;
  if ((newd - distance) > convtol * std::fabs(distance)) {
    if (noisy) {
      distance = newd;
      return true;
    }
    if (std::fabs(newd) > convtol && std::fabs(newd - distance) > 1e-12)
      throw Error(MPSGPU_ENERGY_INCREASE, "optimize: distance increasing");
    done = true;
  }
  if (std::fabs((distance - newd) / distance) < convtol) done = true;
  else done = false;
  if ((std::fabs(distance) + std::fabs(newd)) * convtol < 1e-14)
    if (std::fabs(distance - newd) < convtol) done = true;
  distance = newd;
  return done;
}

void optimize(Context& c, const MpoDev& ops, const MpsDev& orig, MpsDev& init, int D, const SolveOptions& opt,
              double* errN, double* errT, Counters& cnt) {
  const int L = orig.L;
  MPSGPU_CHECK(ops.L == L && init.L == L, MPSGPU_BAD_SHAPE, "optimize: lengths");
  prepare_init(c, init, D);
  EnvCache E;
  E.init(c, L);
  double distance = std::sqrt(cabs2(contract(c, orig, nullptr, orig))) + std::sqrt(cabs2(contract(c, init, nullptr, init)));
  bool right = true, done = false;
  int pos = 0, round = 1;
  cplx c1 = make_double2(0, 0), c2 = make_double2(0, 0);
  DBuf M;
  double* dn = c.dscal + 600;
  // precision 1: the local vector as a split-precision product on the
  // tensor cores; environments, gauge moves, norms and overlaps stay FP64
  // (environments are built recursively along the chain, and the FP32
  // accumulation of the split products compounds there)
  const bool split = opt.precision == 1;
  // the distance carries the split products' error (about 1e-7 relative), so
  // its convergence test and increase guard use kSplitOptimizeTol at least
  const double ctol = split ? std::max(opt.convtol, kSplitOptimizeTol) : opt.convtol;
  SplitMatvec sm;
  try {
    while (!done) {
      calc_left(c, E, pos, &ops, orig, init, &cnt);
      calc_right(c, E, pos, &ops, orig, init, &cnt);
      // M = L W R applied to the orig site (Operator::contractMket, Operator.cpp:427-478)
      const auto od = orig.dims[pos];
      const auto ld = E.ldims[pos];
      const auto rd = E.rdims[pos];
      const int du = ops.dims[pos][0];
      const long long nM = (long long)ld[0] * du * rd[2];
      dbuf_reserve(c, M, nM);
      MPSGPU_CHECK(ld[2] == od[1] && rd[0] == od[2], MPSGPU_BAD_SHAPE, "optimize: dims");
      if (split) {
        const auto& wd = ops.dims[pos];
        split_matvec_prepare(c, sm, E.Le[pos].p, ld, ops, pos, E.Re[pos].p, rd);
        SplitRound r;
        SplitProduct p;
        p.sp[0] = &sm;
        p.Wm[0] = ops.Wlr[pos].p;
        p.Dlb = ld[0]; p.Dlk = ld[2]; p.wl = wd[1]; p.dd = wd[2]; p.Drk = rd[0]; p.du = wd[0]; p.wr = wd[3];
        p.Drb = rd[2];
        p.x = orig.A[pos].p;
        p.y = M.p;
        p.ws = &c.lzone;
        r.p.push_back(p);
        split_round_run(c, r);
        cnt.matvecs++;
        cnt.split_matvecs++;
        cnt.flops += mv_flops(wd[2], wd[1], wd[3], ld[0], rd[2]);
      } else {
        heff_apply(c, E.Le[pos].p, ld, ops, pos, false, E.Re[pos].p, rd, orig.A[pos].p, M.p, make_double2(0, 0),
                   &cnt);
      }
      // solveSiteGauge (Contractor.cpp:921-936): newA = M / |M|
      dznrm2(c.st(), (int)nM, M.p, dn, c.scratch);
      if (opt.verbose > 1) {
        double h = 0;
        MPSGPU_CUDA(cudaMemcpyAsync(&h, dn, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
        printf("mpsgpu: optimize round %d pos %d M (%d,%d,%d) |M| %.17g\n", round, pos, du, ld[0], rd[2], h);
      }
      init.dims[pos] = {du, ld[0], rd[2]};
      dbuf_reserve(c, init.A[pos], nM);
      zscal_inv(c.st(), (int)nM, M.p, dn, init.A[pos].p);
      mps_gauge_site(c, init, pos, right ? 'R' : 'L', false, &cnt);
      // contr1 = <A|A>, contr2 = <A|M> with the gauged tensor (Contractor.cpp:183-186)
      const auto nd = init.dims[pos];
      const long long nA = nel(nd);
      if (nA == nM) {
        cgemv_c(c.st(), (int)nA, 1, init.A[pos].p, nA, init.A[pos].p, c.dcplx + 700, c.scratch);
        cgemv_c(c.st(), (int)nA, 1, init.A[pos].p, nA, M.p, c.dcplx + 701, c.scratch);
      } else {
        // the gauge move changed the shape (bond clipped to min(m, n)): only the
        // chain ends enter the convergence check, where shapes never change
        zfill(c.st(), 2, make_double2(0, 0), c.dcplx + 700);
      }
      for (int l = pos + 1; l < L; l++) E.outofdate_l(l);
      for (int l = pos - 1; l >= 0; l--) E.outofdate_r(l);
      const bool at_end = (right && pos == L - 1) || (!right && pos == 0);
      if (at_end) {
        MPSGPU_CUDA(cudaMemcpyAsync(c.hcplx, c.dcplx + 700, 2 * sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
        MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
        c1 = c.hcplx[0];
        c2 = c.hcplx[1];
        if (opt.verbose) printf("mpsgpu: optimize round %d pos %d c1 %.17g c2 %.17g%+.17gi\n", round, pos, c1.x, c2.x, c2.y);
        done = check_distance(distance, c1, c2, init.normfact, orig.normfact, ctol, split);
        if (!done) {
          if (right) { mps_gauge_site(c, init, pos, 'L', false, &cnt); if (pos > 0) pos--; }
          else { mps_gauge_site(c, init, pos, 'R', false, &cnt); if (pos < L - 1) pos++; }
        }
        right = !right;
        round++;
        if (!done && round >= opt.max_rounds) throw Error(MPSGPU_NOT_CONVERGED, "optimize: round limit reached");
      } else {
        pos += right ? 1 : -1;
      }
    }
  } catch (...) {
    E.release(c);
    dbuf_free(c, M);
    split_matvec_release(c, sm);
    throw;
  }
  E.release(c);
  dbuf_free(c, M);
  split_matvec_release(c, sm);
  init.normfact = c2.x / c1.x;
  init.normfact *= orig.normfact;
  cnt.rounds += round;
  // errN = <orig|ops^dag ops|orig> + <init|init> - 2 Re <init|ops|orig>,
  // errT = the first term (Contractor.cpp:263-276)
  if (errN) {
    const double norm0 = contract2(c, ops, orig, orig).x;
    const double norm1 = contract(c, init, nullptr, init).x;
    const cplx cross = contract(c, orig, &ops, init);
    *errN = norm0 + norm1 - 2.0 * cross.x;
    if (errT) *errT = norm0;
  }
}

// ---------------------------------------------------------------------------
// optimizeSum (Contractor.cpp:2332-2477): |init> ~ sum_k beta_k |ket_k> at
// bond D, by the same sweep as optimize with w = 1 environments between
// every ket and init (calculateL0 / calculateR0, :2272-2297) and the local
// vector M = sum_k normfact_k beta_k L0_k ket_k R0_k (contractMketId,
// :860-878).  The site becomes M / normfact(init) (solveSiteGauge and the
// rescaling after it, :921-936, :2418-2420); the last site of a half-sweep
// keeps the norm in normfact (gaugeCond(pos, dir, true)).  Convergence as in
// optimize, with |M| as the norm of the target.  The initial distance is
// distanceVectors (:2302-2316), including its |beta|^2 term written there as
// re*re + im + im, so that the first convergence test sees the same value.
// ---------------------------------------------------------------------------

void optimize_sum(Context& c, const std::vector<const MpsDev*>& kets, const std::vector<cplx>& beta, MpsDev& init,
                  int D, const SolveOptions& opt, Counters& cnt) {
  const int nt = (int)kets.size();
  MPSGPU_CHECK(nt >= 1 && (int)beta.size() == nt, MPSGPU_INVALID, "optimizeSum: kets and coefficients differ");
  const int L = kets[0]->L;
  for (auto* k : kets) MPSGPU_CHECK(k->L == L, MPSGPU_BAD_SHAPE, "optimizeSum: kets of different lengths");
  MPSGPU_CHECK(init.L == L, MPSGPU_BAD_SHAPE, "optimizeSum: init length");
  prepare_init(c, init, D);
  std::vector<EnvCache> E(nt);
  for (auto& e : E) e.init(c, L);
  // distanceVectors
  double distance;
  {
    cplx sum = make_double2(0.0, 0.0);
    double sumNorms = 0.0;
    for (int k = 0; k < nt; k++) {
      sum = cadd(sum, cmul(beta[k], contract(c, *kets[k], nullptr, init)));
      const double modBeta = beta[k].x * beta[k].x + beta[k].y + beta[k].y;
      sumNorms += modBeta * contract(c, *kets[k], nullptr, *kets[k]).x;
    }
    distance = contract(c, init, nullptr, init).x - 2.0 * sum.x + sumNorms;
  }
  bool right = true, done = false;
  int pos = 0, round = 1;
  DBuf M, T;
  auto cleanup = [&]() {
    for (auto& e : E) e.release(c);
    dbuf_free(c, M);
    dbuf_free(c, T);
  };
  try {
    while (!done) {
      opt.check_cancel();
      long long nM = 0;
      std::array<int, 3> md = {0, 0, 0};
      for (int k = 0; k < nt; k++) {
        calc_left(c, E[k], pos, nullptr, *kets[k], init, &cnt);
        calc_right(c, E[k], pos, nullptr, *kets[k], init, &cnt);
        const auto kd = kets[k]->dims[pos];
        const auto ld = E[k].ldims[pos];  // (Dinit_l, 1, Dket_l)
        const auto rd = E[k].rdims[pos];  // (Dket_r, 1, Dinit_r)
        MPSGPU_CHECK(ld[2] == kd[1] && rd[0] == kd[2], MPSGPU_BAD_SHAPE, "optimizeSum: dims");
        const std::array<int, 3> mk = {kd[0], ld[0], rd[2]};
        if (k == 0) {
          md = mk;
          nM = nel(md);
          dbuf_reserve(c, M, nM);
        } else {
          MPSGPU_CHECK(mk == md, MPSGPU_BAD_SHAPE, "optimizeSum: kets disagree on the site shape");
        }
        // T[(a', s), r] = L0 (Dli x Dlk) . X_k (Dlk x d Drk)
        dbuf_reserve(c, T, (long long)ld[0] * kd[0] * kd[2]);
        GemmArgs g;
        g.M = ld[0]; g.N = kd[0] * kd[2]; g.K = kd[1];
        g.A = E[k].Le[pos].p; g.lda = ld[0];
        g.B = kets[k]->A[pos].p; g.ldb = kd[1];
        g.C = T.p; g.ldc = ld[0];
        zgemm(c.st(), g, c.scratch);
        // M (+)= normfact_k beta_k T (Dli d x Drk) . Rt0 (Drk x Dri)
        GemmArgs h;
        h.M = ld[0] * kd[0]; h.N = rd[2]; h.K = kd[2];
        h.A = T.p; h.lda = (long long)ld[0] * kd[0];
        h.B = E[k].Re[pos].p; h.ldb = kd[2];
        h.C = M.p; h.ldc = (long long)ld[0] * kd[0];
        h.alpha = cscale(beta[k], kets[k]->normfact);
        if (k > 0) {
          h.Cin = M.p; h.ldcin = h.ldc; h.beta = make_double2(1.0, 0.0);
        }
        zgemm(c.st(), h, c.scratch);
      }
      // |M| and the new site M / normfact(init)
      double* dn = c.dscal + 600;
      dznrm2(c.st(), (int)nM, M.p, dn, c.scratch);
      MPSGPU_CUDA(cudaMemcpyAsync(c.hscal, dn, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
      const double normM = c.hscal[0];
      if (pos == 0 && round == 1 && normM == 0.0)
        throw Error(MPSGPU_INVALID,
                    "optimizeSum: the initial state has no overlap with the target (the reference perturbs it "
                    "randomly here)");
      init.dims[pos] = md;
      dbuf_reserve(c, init.A[pos], nM);
      zaxpby(c.st(), (int)nM, make_double2(1.0 / init.normfact, 0.0), M.p, make_double2(0.0, 0.0),
             init.A[pos].p);
      const bool at_end = (right && pos == L - 1) || (!right && pos == 0);
      mps_gauge_site(c, init, pos, right ? 'R' : 'L', at_end, &cnt);
      for (int k = 0; k < nt; k++) {
        for (int l = pos + 1; l < L; l++) E[k].outofdate_l(l);
        for (int l = pos - 1; l >= 0; l--) E[k].outofdate_r(l);
      }
      if (at_end) {
        // contr1 = <A|A>, contr2 = <A|M> with the gauged site
        const auto nd = init.dims[pos];
        MPSGPU_CHECK(nel(nd) == nM, MPSGPU_BAD_SHAPE, "optimizeSum: edge site changed shape");
        cgemv_c(c.st(), (int)nM, 1, init.A[pos].p, nM, init.A[pos].p, c.dcplx + 700, c.scratch);
        cgemv_c(c.st(), (int)nM, 1, init.A[pos].p, nM, M.p, c.dcplx + 701, c.scratch);
        MPSGPU_CUDA(cudaMemcpyAsync(c.hcplx, c.dcplx + 700, 2 * sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
        MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
        done = check_distance(distance, c.hcplx[0], c.hcplx[1], init.normfact, normM, opt.convtol);
        if (opt.verbose) printf("mpsgpu: optimizeSum round %d distance %.17g\n", round, distance);
        if (!done) {
          if (right) { mps_gauge_site(c, init, pos, 'L', false, &cnt); pos--; }
          else { mps_gauge_site(c, init, pos, 'R', false, &cnt); pos++; }
          right = !right;
          round++;
          if (round >= opt.max_rounds) throw Error(MPSGPU_NOT_CONVERGED, "optimizeSum: round limit reached");
        }
      } else {
        pos += right ? 1 : -1;
      }
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
  init.bond = init.max_bond();
  cnt.rounds += round;
}

// ---------------------------------------------------------------------------
// Local observables: <op_k> / <psi|psi> for every site (flatIsing.cpp:258-282)
// with one left and one right pass of w=1 environments.
// ---------------------------------------------------------------------------

void expectation_local(Context& c, const MpsDev& s, const double* op, double* out) {
  const int L = s.L;
  const int d = s.dims[0][0];
  for (int k = 0; k < L; k++) MPSGPU_CHECK(s.dims[k][0] == d, MPSGPU_BAD_SHAPE, "expectation: mixed d");
  MpoDev one;
  int dims4[4] = {d, 1, d, 1};
  const double* wp[1] = {op};
  mpo_upload(c, one, 1, dims4, wp, false);
  EnvCache E;
  E.init(c, L);
  std::vector<cplx> vals(L);
  DBuf T;
  try {
    for (int p = 1; p < L; p++) {
      env_left_update(c, E.Le[p - 1].p, E.ldims[p - 1], s, nullptr, p - 1, s, E.Le[p], E.ldims[p], nullptr);
      E.okL[p] = 1;
    }
    for (int p = L - 2; p >= 0; p--) {
      env_right_update(c, E.Re[p + 1].p, E.rdims[p + 1], s, nullptr, p + 1, s, E.Re[p], E.rdims[p], nullptr);
      E.okR[p] = 1;
    }
    // norm = L[L-1] contracted with the last site
    std::array<int, 3> td;
    MpsDev view;  // site views sharing the buffers of s
    view.L = L;
    view.dims = s.dims;
    view.A = s.A;
    for (int k = 0; k < L; k++) {
      // operator on site k: MPO index k of a one-site MPO -> use a temporary MpoDev view
      MpoDev opk;
      opk.L = L;
      opk.dims.assign(L, {d, 1, d, 1});
      opk.W.assign(L, one.W[0]);
      opk.Wlr.assign(L, one.Wlr[0]);
      opk.Wrl.assign(L, one.Wrl[0]);
      env_left_update(c, E.Le[k].p, E.ldims[k], view, &opk, k, view, T, td, nullptr);
      // <op_k> = sum T[rb, 0, rk] Rt[rk, 0, rb]
      const int Db = td[0], Dk = td[2];
      dbuf_reserve(c, c.t4, (long long)Db * Dk);
      transpose_pqr_to_rqp(c.st(), E.rdims[k][0], 1, E.rdims[k][2], E.Re[k].p, c.t4.p, true);
      // sum_i T_i * R^T_i = conj( sum conj(T_i) ... ) : use cgemv_c with conj(Rt^T) as the "V" column
      cgemv_c(c.st(), Db * Dk, 1, c.t4.p, (long long)Db * Dk, T.p, c.dcplx + 800 + k % 100, c.scratch);
      MPSGPU_CUDA(cudaMemcpyAsync(&vals[k], c.dcplx + 800 + k % 100, sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
      MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    }
    // norm: contract the last left environment with the last site
    DBuf nb;
    std::array<int, 3> nd;
    env_left_update(c, E.Le[L - 1].p, E.ldims[L - 1], s, nullptr, L - 1, s, nb, nd, nullptr);
    cplx nrm;
    MPSGPU_CUDA(cudaMemcpyAsync(&nrm, nb.p, sizeof(cplx), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    dbuf_free(c, nb);
    for (int k = 0; k < L; k++) out[k] = vals[k].x / nrm.x;
  } catch (...) {
    E.release(c);
    dbuf_free(c, T);
    mpo_free(c, one);
    throw;
  }
  E.release(c);
  dbuf_free(c, T);
  mpo_free(c, one);
}

// Contractor::getSchmidtValues (Contractor.cpp:2243-2270): eigenvalues of the
// reduced density matrix of sites pos..L-1 (pos = 0 means L/2), ascending.
// Here: left-canonical copy (gaugeCond R), right-canonicalise sites L-1..pos+1
// with LQ moves, then the bond matrix L of the LQ of site pos carries the
// Schmidt coefficients of bond (pos-1, pos); lambda = sigma^2.
void schmidt_values(Context& c, const MpsDev& s, int pos, std::vector<double>& vals) {
  const int L = s.L;
  MPSGPU_CHECK(pos >= 0 && pos <= L, MPSGPU_BAD_SHAPE, "schmidt values: position out of range");
  if (pos == L) {
    vals.assign(1, 1.0);
    return;
  }
  if (pos == 0) pos = L / 2;
  MpsDev aux;
  try {
    mps_copy(c, s, aux);
    mps_gauge_all(c, aux, 'R', true);
    for (int p = L - 1; p > pos; p--) mps_gauge_site(c, aux, p, 'L', true, nullptr);
    const int Dl = aux.dims[pos][1];
    cplx r00;
    const int K = site_factor(c, aux, pos, 'L', &r00);
    // c.matR holds R' (K x Dl) with L = R'^H: same singular values
    std::vector<double> sv = singular_values(c.st(), K, Dl, c.matR.p, K, c.scratch);
    vals.resize(sv.size());
    for (size_t i = 0; i < sv.size(); i++) vals[i] = sv[sv.size() - 1 - i] * sv[sv.size() - 1 - i];
  } catch (...) {
    mps_free(c, aux);
    throw;
  }
  mps_free(c, aux);
}

// Contractor::getEntropy (Contractor.cpp:2045-2076): -sum lambda log2 lambda
// over |lambda| > 1e-12.
double entropy(Context& c, const MpsDev& s, int pos) {
  if (pos == s.L) return 0.0;
  std::vector<double> lam;
  schmidt_values(c, s, pos, lam);
  double S = 0.0;
  for (double t : lam)
    if (std::fabs(t) > 1e-12) S += -t * std::log2(t);
  return S;
}

}  // namespace mpsgpu
