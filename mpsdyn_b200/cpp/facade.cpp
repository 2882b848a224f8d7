// C++ facade with the reference's class names and call signatures
// (mwArray, MPS, MPO, Operator, Contractor, IsingHamiltonian,
// SchwingerHamiltonian) over the C ABI of libmpsgpu.  Programs written
// against the reference's headers (e.g. programs/ising/testIsing.cpp)
// compile against mpsdyn_b200/cpp/include and run their sweeps on the GPU.
//
// Host side only: tensors cross to the device once (MPO upload, MPS
// creation or setA) and stay there; getA downloads a snapshot.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Contractor.h"
#include "HeisenbergHamiltonian.h"
#include "IsingHamiltonian.h"
#include "MPO.h"
#include "MPS.h"
#include "SchwingerHamiltonian.h"
#include "mpsgpu.h"
#include "mwArray.h"

// ---------------------------------------------------------------------------
// complex_t
// ---------------------------------------------------------------------------

complex_t operator+(complex_t a, complex_t b) { return complex_t{a.re + b.re, a.im + b.im}; }
complex_t& operator+=(complex_t& a, complex_t b) {
  a.re += b.re;
  a.im += b.im;
  return a;
}
complex_t operator-(complex_t a) { return complex_t{-a.re, -a.im}; }
complex_t operator-(complex_t a, complex_t b) { return complex_t{a.re - b.re, a.im - b.im}; }
complex_t operator*(complex_t a, complex_t b) {
  return complex_t{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
complex_t& operator*=(complex_t& a, complex_t b) { return a = a * b; }
complex_t operator*(double x, complex_t a) { return complex_t{x * a.re, x * a.im}; }
complex_t operator*(complex_t a, double x) { return complex_t{x * a.re, x * a.im}; }
complex_t operator/(complex_t a, complex_t b) {
  // Smith's division (CACM 5(8), 1962): no overflow of |b|^2
  if (std::fabs(b.re) >= std::fabs(b.im)) {
    const double r = b.im / b.re, den = b.re + b.im * r;
    return complex_t{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  }
  const double r = b.re / b.im, den = b.im + b.re * r;
  return complex_t{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
complex_t operator/(complex_t a, double x) { return complex_t{a.re / x, a.im / x}; }
complex_t conjugate(complex_t a) { return complex_t{a.re, -a.im}; }
bool operator==(complex_t a, complex_t b) { return a.re == b.re && a.im == b.im; }
bool operator!=(complex_t a, complex_t b) { return !(a == b); }
std::ostream& operator<<(std::ostream& os, complex_t c) { return os << "(" << c.re << "," << c.im << ")"; }
double abs(complex_t c) { return std::hypot(c.re, c.im); }
double phase(complex_t c) { return std::atan2(c.im, c.re); }
double real(complex_t c) { return c.re; }
double imag(complex_t c) { return c.im; }
complex_t sqrt(complex_t c) {
  const double r = std::sqrt(abs(c)), t = 0.5 * phase(c);
  return complex_t{r * std::cos(t), r * std::sin(t)};
}
complex_t exp(complex_t c) {
  const double e = std::exp(c.re);
  return complex_t{e * std::cos(c.im), e * std::sin(c.im)};
}

// ---------------------------------------------------------------------------
// mwArray
// ---------------------------------------------------------------------------

namespace {

long long prod(const shrt::Indices& d) {
  long long n = 1;
  for (int x : d) n *= x;
  return n;
}

void fail(const std::string& msg) { throw MpsgpuException(MPSGPU_BAD_SHAPE, "mwArray: " + msg); }

}  // namespace

mwArray::mwArray(const shrt::Indices& dims) : dims_(dims), data_((size_t)prod(dims), ZERO_c) {}

mwArray::mwArray(const shrt::Indices& dims, const complex_t* values)
    : dims_(dims), data_(values, values + prod(dims)) {}

mwArray::mwArray(const shrt::Indices& dims, const double* values) : dims_(dims), data_((size_t)prod(dims)) {
  for (size_t i = 0; i < data_.size(); i++) data_[i] = complex_t{values[2 * i], values[2 * i + 1]};
}

mwArray::mwArray(complex_t scalar) : dims_(shrt::Indices(1)), data_(1, scalar) {}

long long mwArray::offset(const shrt::Indices& idx) const {
  if (idx.size() != dims_.size()) fail("index rank");
  long long off = 0, stride = 1;
  for (size_t k = 0; k < dims_.size(); k++) {
    if (idx[k] < 0 || idx[k] >= dims_[k]) fail("index out of range");
    off += idx[k] * stride;
    stride *= dims_[k];
  }
  return off;
}

void mwArray::reshape(const shrt::Indices& dims) {
  shrt::Indices nd = dims;
  long long known = 1;
  int free_pos = -1;
  for (size_t k = 0; k < nd.size(); k++) {
    if (nd[k] == -1) {
      if (free_pos >= 0) fail("reshape: more than one -1");
      free_pos = (int)k;
    } else {
      known *= nd[k];
    }
  }
  if (free_pos >= 0) nd[free_pos] = known > 0 ? (int)((long long)data_.size() / known) : 0;
  if (prod(nd) != (long long)data_.size()) fail("reshape: element count differs");
  dims_ = nd;
}

void mwArray::resize(const shrt::Indices& dims) {
  std::vector<complex_t> nd((size_t)prod(dims), ZERO_c);
  const size_t r = std::min(dims.size(), dims_.size());
  std::vector<int> idx(dims.size(), 0);
  for (size_t t = 0; t < nd.size(); t++) {
    // idx = multi-index of t in the new box
    long long rem = (long long)t;
    bool inside = true;
    long long off = 0, stride = 1;
    for (size_t k = 0; k < dims.size(); k++) {
      idx[k] = (int)(rem % dims[k]);
      rem /= dims[k];
      if (k < r) {
        if (idx[k] >= dims_[k]) inside = false;
        off += idx[k] * stride;
        stride *= dims_[k];
      } else if (idx[k] != 0) {
        inside = false;
      }
    }
    if (inside && !data_.empty()) nd[t] = data_[(size_t)off];
  }
  dims_ = dims;
  data_.swap(nd);
}

void mwArray::permute(const shrt::Indices& order, bool conj) {
  const int r = getRank();
  if ((int)order.size() != r) fail("permute: order rank");
  shrt::Indices nd{std::vector<int>((size_t)r, 0)};
  std::vector<long long> ostride(r);
  long long s = 1;
  for (int k = 0; k < r; k++) {
    ostride[k] = s;
    s *= dims_[k];
  }
  for (int k = 0; k < r; k++) nd[k] = dims_[order[k] - 1];
  std::vector<complex_t> out(data_.size());
  std::vector<int> idx(r, 0);
  for (size_t t = 0; t < out.size(); t++) {
    long long rem = (long long)t, off = 0;
    for (int k = 0; k < r; k++) {
      idx[k] = (int)(rem % nd[k]);
      rem /= nd[k];
      off += idx[k] * ostride[order[k] - 1];
    }
    complex_t v = data_[(size_t)off];
    if (conj) v.im = -v.im;
    out[t] = v;
  }
  dims_ = nd;
  data_.swap(out);
}

void mwArray::conjugate() {
  for (auto& v : data_) v.im = -v.im;
}

void mwArray::transpose(bool conj) {
  if (getRank() != 2) fail("transpose: rank 2 only");
  permute(shrt::Indices(2, 1), conj);
}

void mwArray::fillWithZero() {
  for (auto& v : data_) v = ZERO_c;
}

mwArray mwArray::operator*(const mwArray& rhs) const {
  if (isScalar()) return data_[0] * rhs;
  if (rhs.isScalar()) return rhs.data_[0] * *this;
  if (getRank() != 2 || rhs.getRank() != 2 || dims_[1] != rhs.dims_[0]) fail("product: shapes");
  const int m = dims_[0], k = dims_[1], n = rhs.dims_[1];
  mwArray out(shrt::Indices(m, n));
  for (int j = 0; j < n; j++)
    for (int l = 0; l < k; l++) {
      const complex_t b = rhs.data_[l + (size_t)k * j];
      for (int i = 0; i < m; i++) out.data_[i + (size_t)m * j] += data_[i + (size_t)m * l] * b;
    }
  return out;
}

void mwArray::multiplyRight(const mwArray& rhs) { *this = *this * rhs; }
void mwArray::multiplyLeft(const mwArray& lhs) { *this = lhs * *this; }

mwArray mwArray::operator+(const mwArray& rhs) const {
  if (rhs.data_.size() != data_.size()) fail("sum: shapes");
  mwArray out(*this);
  for (size_t i = 0; i < data_.size(); i++) out.data_[i] += rhs.data_[i];
  return out;
}

mwArray mwArray::operator-(const mwArray& rhs) const {
  if (rhs.data_.size() != data_.size()) fail("difference: shapes");
  mwArray out(*this);
  for (size_t i = 0; i < data_.size(); i++) out.data_[i] = out.data_[i] - rhs.data_[i];
  return out;
}

mwArray& mwArray::operator*=(complex_t c) {
  for (auto& v : data_) v = v * c;
  return *this;
}

void mwArray::save(std::ostream& os) const {
  const int rank = getRank();
  os.write(reinterpret_cast<const char*>(&rank), sizeof(int));
  for (int d : dims_) os.write(reinterpret_cast<const char*>(&d), sizeof(int));
  os.write(reinterpret_cast<const char*>(data_.data()), (std::streamsize)(data_.size() * sizeof(complex_t)));
}

void mwArray::load(std::istream& is) {
  int rank = 0;
  is.read(reinterpret_cast<char*>(&rank), sizeof(int));
  if (!is || rank < 0 || rank > 16) fail("load: bad rank");
  std::vector<int> d(rank);
  for (int& x : d) is.read(reinterpret_cast<char*>(&x), sizeof(int));
  dims_ = shrt::Indices(d);
  data_.assign((size_t)prod(dims_), ZERO_c);
  is.read(reinterpret_cast<char*>(data_.data()), (std::streamsize)(data_.size() * sizeof(complex_t)));
  if (!is) fail("load: truncated file");
}

std::ostream& operator<<(std::ostream& os, const mwArray& a) {
  os << "mwArray dims (";
  for (size_t k = 0; k < a.dims_.size(); k++) os << (k ? "," : "") << a.dims_[k];
  os << ")";
  if (a.data_.size() <= 16) {
    os << " [";
    for (size_t i = 0; i < a.data_.size(); i++) os << (i ? " " : "") << a.data_[i];
    os << "]";
  }
  return os;
}

mwArray operator*(complex_t c, const mwArray& a) {
  mwArray out(a);
  out *= c;
  return out;
}

mwArray reshape(const mwArray& a, const shrt::Indices& dims) {
  mwArray out(a);
  out.reshape(dims);
  return out;
}

mwArray permute(const mwArray& a, const shrt::Indices& order) {
  mwArray out(a);
  out.permute(order);
  return out;
}

mwArray conjugate(const mwArray& a) {
  mwArray out(a);
  out.conjugate();
  return out;
}

mwArray identityMatrix(int d) {
  mwArray out(shrt::Indices(d, d));
  for (int i = 0; i < d; i++) out.setElement(ONE_c, shrt::Indices(i, i));
  return out;
}

// ---------------------------------------------------------------------------
// Contractor (the context owner)
// ---------------------------------------------------------------------------

namespace {

mpsgpu_context* ctx() { return Contractor::theContractor().context(); }

mpsgpu_options options_from(double convtol, double eigtol, double excorthtol, int precision = 0) {
  mpsgpu_options o;
  mpsgpu_default_options(&o);
  o.precision = precision;
  o.convtol = convtol;
  o.eigtol = eigtol;
  o.excorthtol = excorthtol;
  return o;
}

}  // namespace

Contractor::Contractor() {}

Contractor& Contractor::theContractor() {
  static Contractor c;
  return c;
}

mpsgpu_context* Contractor::context() {
  if (!ctx_) {
    const char* dev = std::getenv("MPSGPU_DEVICE");
    check(mpsgpu_create(dev ? std::atoi(dev) : 0, &ctx_), "Contractor: create context");
  }
  return ctx_;
}

void Contractor::check(int status, const char* what) {
  if (status == MPSGPU_OK) return;
  std::string msg = std::string(what) + ": " + mpsgpu_status_string((mpsgpu_status)status);
  Contractor& c = theContractor();
  if (c.ctx_) {
    const char* e = mpsgpu_last_error(c.ctx_);
    if (e && *e) msg += std::string(" (") + e + ")";
  }
#ifdef MPSDYN_STRICT_EXIT
  std::cout << "Error: " << msg << std::endl;
  std::exit(212);
#else
  throw MpsgpuException(status, msg);
#endif
}

// nrLocalEig: the reference asks the local eigensolver for knr pairs and
// keeps the lowest (U.resize to the first column, Contractor.cpp:1410-1416);
// the library computes that pair directly, so the result does not depend on
// knr.  useLM (target the largest-magnitude local eigenvalue) has no
// counterpart in the library: the call warns once and targets the lowest.
static void warn_use_lm(bool useLM, const char* where) {
  static bool warned = false;
  if (useLM && !warned) {
    std::cerr << "WARNING: " << where << ": useLM is not supported by the GPU library; "
              << "the lowest local eigenvalue (SR) is targeted" << std::endl;
    warned = true;
  }
}

void Contractor::findGroundState(const MPO& ops, int D, double* lambda, MPS& init, double offset, int,
                                 const std::string& tmpfile, int freqSv, bool useLM) {
  warn_use_lm(useLM, "findGroundState");
  mpsgpu_options o = options_from(convtol, eigtol, excorthtol, precision);
  if (!tmpfile.empty()) {
    o.checkpoint_file = tmpfile.c_str();
    o.checkpoint_every = freqSv > 0 ? freqSv : 200;
  }
  check(mpsgpu_find_ground_state(context(), ops.device(), D, offset, &o, init.device(), lambda, nullptr),
        "findGroundState");
  init.changed();
}

void Contractor::findNextExcitedState(const MPO& ops, int D, const std::vector<MPS*>& levels, double* lambdak,
                                      MPS& init, double offset, int, const std::string& tmpfile, int maxTime,
                                      bool useLM) {
  warn_use_lm(useLM, "findNextExcitedState");
  std::vector<const mpsgpu_mps*> lv;
  for (const MPS* m : levels) lv.push_back(m->device());
  mpsgpu_options o = options_from(convtol, eigtol, excorthtol, precision);
  if (!tmpfile.empty()) {
    o.checkpoint_file = tmpfile.c_str();
    o.checkpoint_seconds = maxTime;
  }
  check(mpsgpu_find_next_excited_state(context(), ops.device(), D, lv.data(), (int)lv.size(), offset, &o,
                                       init.device(), lambdak, nullptr),
        "findNextExcitedState");
  init.changed();
}

void Contractor::optimizeSum(std::vector<const MPS*> kets, std::vector<complex_t> beta, MPS& init, int D) {
  if (kets.empty() || kets.size() != beta.size()) check(MPSGPU_INVALID, "optimizeSum: kets and beta differ");
  std::vector<const mpsgpu_mps*> ks;
  std::vector<double> b;
  for (size_t k = 0; k < kets.size(); k++) {
    ks.push_back(kets[k]->device());
    b.push_back(beta[k].re);
    b.push_back(beta[k].im);
  }
  const mpsgpu_options o = options_from(convtol, eigtol, excorthtol);
  check(mpsgpu_optimize_sum(context(), (int)ks.size(), ks.data(), b.data(), init.device(), D, &o, nullptr),
        "optimizeSum");
  init.changed();
}

void Contractor::optimizeMPS(const MPS& ket, MPS& init, int D, double* err) {
  const mpsgpu_options o = options_from(convtol, eigtol, excorthtol);
  check(mpsgpu_optimize_mps(context(), ket.device(), init.device(), D, &o, err, nullptr), "optimizeMPS");
  init.changed();
}

void Contractor::optimize(const MPO& ops, const MPS& ket, MPS& init, int D, double* errN, double* errT) {
  if (init.isEmpty()) init = ket;
  const mpsgpu_options o = options_from(convtol, eigtol, excorthtol);
  check(mpsgpu_optimize(context(), ops.device(), ket.device(), init.device(), D, &o, errN, errN ? errT : nullptr,
                        nullptr),
        "optimize");
  init.changed();
}

complex_t Contractor::contract(const MPS& ket, const MPS& bra, char) {
  complex_t r{0., 0.};
  check(mpsgpu_contract(context(), ket.device(), nullptr, bra.device(), &r.re, &r.im), "contract");
  return r;
}

complex_t Contractor::contract(const MPS& ket, const MPO& ops, const MPS& bra) {
  complex_t r{0., 0.};
  check(mpsgpu_contract(context(), ket.device(), ops.device(), bra.device(), &r.re, &r.im), "contract");
  return r;
}

complex_t Contractor::contract2(const MPO& ops, const MPS& ket) {
  complex_t r{0., 0.};
  check(mpsgpu_contract2(context(), ops.device(), ket.device(), nullptr, &r.re, &r.im), "contract2");
  return r;
}

complex_t Contractor::contract2(const MPS& bra, const MPO& ops, const MPS& ket) {
  complex_t r{0., 0.};
  check(mpsgpu_contract2(context(), ops.device(), ket.device(), bra.device(), &r.re, &r.im), "contract2");
  return r;
}

double Contractor::getEntropy(const MPS& state, int len) {
  double S = 0.0;
  check(mpsgpu_entropy(context(), state.device(), len, &S), "getEntropy");
  return S;
}

void Contractor::getSchmidtValues(const MPS& state, std::vector<complex_t>& lambdas, int len) {
  int L = 0;
  check(mpsgpu_mps_info(context(), state.device(), &L, nullptr, nullptr), "getSchmidtValues");
  std::vector<int> dims(3 * L);
  check(mpsgpu_mps_info(context(), state.device(), &L, dims.data(), nullptr), "getSchmidtValues");
  int cap = 1;
  for (int k = 0; k < L; k++) cap = std::max(cap, std::max(dims[3 * k + 1], dims[3 * k + 2]));
  std::vector<double> v(cap);
  int n = 0;
  check(mpsgpu_schmidt_values(context(), state.device(), len, v.data(), cap, &n), "getSchmidtValues");
  lambdas.clear();
  for (int i = 0; i < n; i++) lambdas.push_back(complex_t{v[i], 0.});
}

// ---------------------------------------------------------------------------
// MPO
// ---------------------------------------------------------------------------

MPO::MPO(const MPO& other) { *this = other; }

MPO& MPO::operator=(const MPO& other) {
  if (this == &other) return *this;
  clear();
  initLength(other.length_);
  for (int k = 0; k < length_; k++)
    if (other.ops_[k]) setOp(k, new Operator(other.ops_[k]->getFullData()), true);
  return *this;
}

MPO::~MPO() { clear(); }

void MPO::drop_device() const {
  if (dev_) {
    mpsgpu_mpo_free(ctx(), dev_);
    dev_ = nullptr;
  }
}

void MPO::initLength(int len) {
  clear();
  length_ = len;
  ops_.assign(len, nullptr);
  own_.assign(len, false);
}

void MPO::clear() {
  drop_device();
  for (size_t k = 0; k < ops_.size(); k++)
    if (own_[k]) delete ops_[k];
  ops_.clear();
  own_.clear();
  length_ = 0;
}

const Operator& MPO::getOp(int pos) const {
  if (pos < 0 || pos >= length_ || !ops_[pos]) Contractor::check(MPSGPU_INVALID, "MPO::getOp: empty position");
  return *ops_[pos];
}

void MPO::setOp(int pos, const Operator* op, bool myop) {
  if (pos < 0 || pos >= length_) Contractor::check(MPSGPU_INVALID, "MPO::setOp: position");
  if (own_[pos] && ops_[pos] != op) delete ops_[pos];
  ops_[pos] = op;
  own_[pos] = myop;
  drop_device();
}

const std::vector<int> MPO::getDimensions() const {
  std::vector<int> d(length_);
  for (int k = 0; k < length_; k++) d[k] = getOp(k).getDimension(0);
  return d;
}

mpsgpu_mpo* MPO::device() const {
  if (dev_) return dev_;
  std::vector<int> dims;
  std::vector<const double*> ptrs;
  for (int k = 0; k < length_; k++) {
    const mwArray& W = getOp(k).getFullData();
    if (W.getRank() != 4) Contractor::check(MPSGPU_BAD_SHAPE, "MPO: operators must be rank 4");
    for (int j = 0; j < 4; j++) dims.push_back(W.getDimension(j));
    ptrs.push_back(reinterpret_cast<const double*>(W.components()));
  }
  Contractor::check(mpsgpu_mpo_upload(ctx(), length_, dims.data(), ptrs.data(), &dev_), "MPO upload");
  return dev_;
}

void MPO::setFromDevice(mpsgpu_mpo* h) {
  int L = 0;
  Contractor::check(mpsgpu_mpo_info(ctx(), h, &L, nullptr), "MPO info");
  std::vector<int> dims(4 * L);
  Contractor::check(mpsgpu_mpo_info(ctx(), h, &L, dims.data()), "MPO info");
  std::vector<mwArray> host;
  std::vector<double*> ptrs;
  for (int k = 0; k < L; k++) {
    host.emplace_back(shrt::Indices(dims[4 * k], dims[4 * k + 1], dims[4 * k + 2], dims[4 * k + 3]));
  }
  for (auto& a : host) ptrs.push_back(reinterpret_cast<double*>(a.components()));
  Contractor::check(mpsgpu_mpo_download(ctx(), h, ptrs.data()), "MPO download");
  initLength(L);
  for (int k = 0; k < L; k++) setOp(k, new Operator(host[k]), true);
  dev_ = h;  // after setOp, which drops any previous device copy
}

void MPO::saveMPO(const char* filename) const {
  Contractor::check(mpsgpu_mpo_save(ctx(), device(), filename), "MPO::saveMPO");
}

void MPO::loadMPO(const char* filename) {
  mpsgpu_mpo* h = nullptr;
  Contractor::check(mpsgpu_mpo_load(ctx(), filename, &h), "MPO::loadMPO");
  setFromDevice(h);
}

// ---------------------------------------------------------------------------
// MPS
// ---------------------------------------------------------------------------

namespace {
uint64_t g_random_seed = 0;
}

void MPS::setRandomSeed(uint64_t seed) { g_random_seed = seed; }

MPS::MPS(int length, int bond, int d) {
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_product(ctx(), length, d, bond, &h), "MPS(L, D, d)");
  adopt(h);
}

MPS::MPS(const MPS& aMPS) { *this = aMPS; }

MPS::MPS(const MPS& aMPS, int bond) {
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_approximate(ctx(), aMPS.h_, bond, &h, nullptr), "MPS(mps, D)");
  adopt(h);
}

MPS::MPS(const MPO& ops, const MPS& aMPS, int bond, char dir, char gauge) { approximate(ops, aMPS, bond, dir, gauge); }

MPS& MPS::operator=(const MPS& aMPS) {
  if (this == &aMPS) return *this;
  if (!aMPS.h_) {
    release();
    return *this;
  }
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_copy(ctx(), aMPS.h_, &h), "MPS copy");
  adopt(h);
  return *this;
}

MPS::~MPS() { release(); }

void MPS::release() {
  if (h_) mpsgpu_mps_free(ctx(), h_);
  h_ = nullptr;
  length_ = 0;
  cache_.clear();
  cache_ok_ = false;
}

void MPS::adopt(mpsgpu_mps* h) {
  release();
  h_ = h;
  int L = 0;
  Contractor::check(mpsgpu_mps_info(ctx(), h_, &L, nullptr, nullptr), "MPS info");
  length_ = L;
}

int MPS::getBond() const {
  int b = 0;
  if (h_) Contractor::check(mpsgpu_mps_bond(ctx(), h_, &b, nullptr), "MPS bond");
  return b;
}

bool MPS::isGaugeL() const {
  int g = 0;
  if (h_) Contractor::check(mpsgpu_mps_bond(ctx(), h_, nullptr, &g), "MPS gauge");
  return g == gLeft || g == gBoth;
}

bool MPS::isGaugeR() const {
  int g = 0;
  if (h_) Contractor::check(mpsgpu_mps_bond(ctx(), h_, nullptr, &g), "MPS gauge");
  return g == gRight || g == gBoth;
}

double MPS::getNormFact() const {
  double nf = 0.0;
  if (h_) Contractor::check(mpsgpu_mps_info(ctx(), h_, nullptr, nullptr, &nf), "MPS normfact");
  return nf;
}

void MPS::setNormFact(double value) {
  Contractor::check(mpsgpu_mps_set_normfact(ctx(), h_, value), "MPS setNormFact");
}

void MPS::sync_cache() const {
  if (cache_ok_) return;
  int L = 0;
  Contractor::check(mpsgpu_mps_info(ctx(), h_, &L, nullptr, nullptr), "MPS info");
  std::vector<int> dims(3 * L);
  Contractor::check(mpsgpu_mps_info(ctx(), h_, &L, dims.data(), nullptr), "MPS info");
  std::vector<mwArray> host;
  for (int k = 0; k < L; k++) host.emplace_back(shrt::Indices(dims[3 * k], dims[3 * k + 1], dims[3 * k + 2]));
  std::vector<double*> ptrs;
  for (auto& a : host) ptrs.push_back(reinterpret_cast<double*>(a.components()));
  Contractor::check(mpsgpu_mps_download(ctx(), h_, ptrs.data()), "MPS download");
  cache_.clear();
  for (auto& a : host) cache_.emplace_back(a);
  cache_ok_ = true;
}

const Site_t& MPS::getA(int k) const {
  if (k < 0 || k >= length_) Contractor::check(MPSGPU_INVALID, "MPS::getA: position");
  sync_cache();
  return cache_[k];
}

void MPS::setA(int pos, const mwArray& data) {
  if (pos < 0 || pos >= length_ || data.getRank() != 3) Contractor::check(MPSGPU_INVALID, "MPS::setA");
  sync_cache();
  std::vector<mwArray> host;
  for (auto& s : cache_) host.push_back(s.getA());
  host[pos] = data;
  std::vector<int> dims;
  std::vector<const double*> ptrs;
  for (auto& a : host) {
    for (int j = 0; j < 3; j++) dims.push_back(a.getDimension(j));
    ptrs.push_back(reinterpret_cast<const double*>(a.components()));
  }
  const double nf = getNormFact();
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_upload(ctx(), length_, dims.data(), ptrs.data(), nf, &h), "MPS::setA upload");
  adopt(h);
}

void MPS::setRandomState() {
  const int L = length_;
  const int d = getA(0).getd();
  const int D = getBond();
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_random_state(ctx(), L, d, D, g_random_seed, &h), "MPS::setRandomState");
  adopt(h);
}

void MPS::gaugeCond(char dir, bool normalize, int cutD) {
  Contractor::check(mpsgpu_mps_gauge_cond(ctx(), h_, dir, normalize ? 1 : 0, cutD, nullptr), "MPS::gaugeCond");
  changed();
}

void MPS::increaseBondDimension(int D) {
  Contractor::check(mpsgpu_mps_increase_bond(ctx(), h_, D), "MPS::increaseBondDimension");
  changed();
}

void MPS::applyExactly(const MPO& ops, bool dagger, char gaugedir) {
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_apply_mpo(ctx(), ops.device(), h_, 0, dagger ? 1 : 0, gaugedir, &h, nullptr),
                    "MPS::applyExactly");
  adopt(h);
}

void MPS::approximate(const MPO& ops, const MPS& aMPS, int D, char dir, char gaugeDir) {
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_apply_mpo(ctx(), ops.device(), aMPS.h_, D, dir == 'U' ? 1 : 0, gaugeDir, &h, nullptr),
                    "MPS::approximate");
  adopt(h);
}

void MPS::exportMPS(const char* filename) const {
  std::ofstream os(filename, std::ios::binary);
  if (!os) Contractor::check(MPSGPU_INVALID, "MPS::exportMPS: cannot open file");
  sync_cache();
  const int L = length_, bond = getBond();
  int gauge = 0;
  Contractor::check(mpsgpu_mps_bond(ctx(), h_, nullptr, &gauge), "MPS gauge");
  const double nf = getNormFact();
  os.write(reinterpret_cast<const char*>(&L), sizeof(int));
  os.write(reinterpret_cast<const char*>(&bond), sizeof(int));
  os.write(reinterpret_cast<const char*>(&nf), sizeof(double));
  os.write(reinterpret_cast<const char*>(&gauge), sizeof(int));
  for (int k = 0; k < L; k++) {
    const int pos = k + 1;
    os.write(reinterpret_cast<const char*>(&pos), sizeof(int));
    cache_[k].getA().save(os);
  }
}

void MPS::importMPS(const char* filename) {
  std::ifstream is(filename, std::ios::binary);
  if (!is) Contractor::check(MPSGPU_INVALID, "MPS::importMPS: cannot open file");
  int L = 0, bond = 0, gauge = 0;
  double nf = 1.0;
  is.read(reinterpret_cast<char*>(&L), sizeof(int));
  is.read(reinterpret_cast<char*>(&bond), sizeof(int));
  is.read(reinterpret_cast<char*>(&nf), sizeof(double));
  is.read(reinterpret_cast<char*>(&gauge), sizeof(int));
  if (!is || L <= 0) Contractor::check(MPSGPU_INVALID, "MPS::importMPS: bad header");
  std::vector<mwArray> host(L);
  for (int k = 0; k < L; k++) {
    int pos = 0;
    is.read(reinterpret_cast<char*>(&pos), sizeof(int));
    host[k].load(is);
  }
  std::vector<int> dims;
  std::vector<const double*> ptrs;
  for (auto& a : host) {
    if (a.getRank() != 3) Contractor::check(MPSGPU_BAD_SHAPE, "MPS::importMPS: site rank");
    for (int j = 0; j < 3; j++) dims.push_back(a.getDimension(j));
    ptrs.push_back(reinterpret_cast<const double*>(a.components()));
  }
  mpsgpu_mps* h = nullptr;
  Contractor::check(mpsgpu_mps_upload(ctx(), L, dims.data(), ptrs.data(), nf, &h), "MPS::importMPS upload");
  adopt(h);
}

std::ostream& operator<<(std::ostream& os, const MPS& mps) {
  os << "MPS{length=" << mps.getLength() << ", bond=" << mps.getBond() << "}" << std::endl;
  int L = 0;
  if (mps.h_) {
    Contractor::check(mpsgpu_mps_info(ctx(), mps.h_, &L, nullptr, nullptr), "MPS info");
    std::vector<int> dims(3 * L);
    Contractor::check(mpsgpu_mps_info(ctx(), mps.h_, &L, dims.data(), nullptr), "MPS info");
    for (int k = 0; k < L; k++)
      os << "Site(" << k << ") (" << dims[3 * k] << "," << dims[3 * k + 1] << "," << dims[3 * k + 2] << ")"
         << std::endl;
  }
  return os;
}

// ---------------------------------------------------------------------------
// Hamiltonians
// ---------------------------------------------------------------------------

IsingHamiltonian::IsingHamiltonian(int N_, int d_, double J0, double g0, double h0, double K)
    : N(N_), d(d_), J(J0), g(g0), h(h0) {
  if (d != 2 || K != 0.0) Contractor::check(MPSGPU_INVALID, "IsingHamiltonian: d = 2 and K = 0 only");
  mpsgpu_mpo* m = nullptr;
  Contractor::check(mpsgpu_mpo_ising(ctx(), N, J, g, h, &m), "IsingHamiltonian");
  hamil.setFromDevice(m);
}

const MPO& IsingHamiltonian::getHMPO(double) { return hamil; }

void IsingHamiltonian::getUMPO(MPO& mpo, double delta, double, bool imag, int orderT, int nrOp) {
  if (orderT != 2 || nrOp != 0) Contractor::check(MPSGPU_INVALID, "IsingHamiltonian::getUMPO: second order only");
  mpsgpu_mpo* m = nullptr;
  Contractor::check(mpsgpu_mpo_ising_evolution(ctx(), N, J, g, h, delta, imag ? 1 : 0, &m),
                    "IsingHamiltonian::getUMPO");
  mpo.setFromDevice(m);
}

SchwingerHamiltonian::SchwingerHamiltonian(int N, double mu, double x, double l0, double alpha, double offset, double nu,
                                           double y) {
  if (offset != 0.0 || nu != 0.0 || y != 1.0)
    Contractor::check(MPSGPU_INVALID, "SchwingerHamiltonian: offset = nu = 0 and y = 1 only");
  mpsgpu_mpo* m = nullptr;
  Contractor::check(mpsgpu_mpo_schwinger(ctx(), N, mu, x, l0, alpha, &m), "SchwingerHamiltonian");
  hamil.setFromDevice(m);
}

HeisenbergHamiltonian::HeisenbergHamiltonian(int L, double Jx, double Jy, double Jz, double h, int d, double offset, int,
                                             double penalty) {
  build(L, Jx, Jy, Jz, 0.0, 0.0, h, d, offset, penalty);
}

HeisenbergHamiltonian::HeisenbergHamiltonian(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz,
                                             int d, double offset, int, double penalty) {
  build(L, Jx, Jy, Jz, hx, hy, hz, d, offset, penalty);
}

void HeisenbergHamiltonian::build(int L, double Jx, double Jy, double Jz, double hx, double hy, double hz, int d,
                                  double offset, double penalty) {
  if (d != 2 || penalty != 0.0)
    Contractor::check(MPSGPU_INVALID, "HeisenbergHamiltonian: d = 2 and no Sz penalty only");
  mpsgpu_mpo* m = nullptr;
  Contractor::check(mpsgpu_mpo_heisenberg(ctx(), L, Jx, Jy, Jz, hx, hy, hz, offset, &m), "HeisenbergHamiltonian");
  hamil.setFromDevice(m);
}
