// Binary MPS and MPO files in the reference's formats, for checkpoints and
// for exchanging states and operators with programs built on the reference:
//
//   mwArray   int rank, int dims[rank], double data[2 n] (column-major,
//             re/im interleaved)                  src/wrapper/mwArray.cpp:382-442
//   MPS       int length, int bond, double normfact, int gauge, then per site
//             int pos (1-based) and the site's mwArray (d, Dl, Dr)
//                                                 src/core/cpp/MPS.cpp:442-509,
//                                                 src/core/cpp/Site.cpp:561-578
//   MPO       int length, then per site the operator's mwArray (du, Dl, dd, Dr)
//                                                 src/core/cpp/MPO.cpp:214-316
//
// Host code only: states are downloaded to (or uploaded from) host buffers
// in the reference layout; byte order is the machine's, as the reference
// writes it.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "engine.h"
#include "mpsgpu.h"

namespace mpsgpu {

namespace {

void write_array(std::ostream& os, const std::vector<int>& dims, const double* data) {
  const int rank = (int)dims.size();
  long long n = 1;
  for (int d : dims) n *= d;
  os.write(reinterpret_cast<const char*>(&rank), sizeof(int));
  os.write(reinterpret_cast<const char*>(dims.data()), sizeof(int) * rank);
  os.write(reinterpret_cast<const char*>(data), sizeof(double) * 2 * n);
}

void read_array(std::istream& is, std::vector<int>& dims, std::vector<double>& data) {
  int rank = 0;
  is.read(reinterpret_cast<char*>(&rank), sizeof(int));
  MPSGPU_CHECK(is && rank >= 0 && rank <= 16, MPSGPU_INVALID, "file: bad array rank");
  dims.assign(rank, 0);
  is.read(reinterpret_cast<char*>(dims.data()), sizeof(int) * rank);
  long long n = 1;
  for (int d : dims) {
    MPSGPU_CHECK(d >= 0, MPSGPU_INVALID, "file: negative dimension");
    n *= d;
  }
  MPSGPU_CHECK(is && n < (1LL << 34), MPSGPU_INVALID, "file: truncated array header");
  data.resize(2 * n);
  is.read(reinterpret_cast<char*>(data.data()), sizeof(double) * 2 * n);
  MPSGPU_CHECK((bool)is, MPSGPU_INVALID, "file: truncated array data");
}

}  // namespace

void mps_export_file(Context& c, const MpsDev& s, const std::string& fn) {
  std::vector<std::vector<double>> host(s.L);
  std::vector<double*> ptrs(s.L);
  for (int k = 0; k < s.L; k++) {
    const auto& d = s.dims[k];
    host[k].resize(2LL * d[0] * d[1] * d[2]);
    ptrs[k] = host[k].data();
  }
  mps_download(c, s, ptrs.data());
  std::ofstream os(fn, std::ios::binary | std::ios::trunc);
  MPSGPU_CHECK((bool)os, MPSGPU_INVALID, "MPS export: cannot open " + fn);
  const int L = s.L, bond = s.bond > 0 ? s.bond : s.max_bond(), gauge = s.gauge;
  const double nf = s.normfact;
  os.write(reinterpret_cast<const char*>(&L), sizeof(int));
  os.write(reinterpret_cast<const char*>(&bond), sizeof(int));
  os.write(reinterpret_cast<const char*>(&nf), sizeof(double));
  os.write(reinterpret_cast<const char*>(&gauge), sizeof(int));
  for (int k = 0; k < L; k++) {
    const int pos = k + 1;
    os.write(reinterpret_cast<const char*>(&pos), sizeof(int));
    write_array(os, {s.dims[k][0], s.dims[k][1], s.dims[k][2]}, host[k].data());
  }
  MPSGPU_CHECK((bool)os, MPSGPU_INVALID, "MPS export: write failed for " + fn);
}

void mps_import_file(Context& c, const std::string& fn, MpsDev& s) {
  std::ifstream is(fn, std::ios::binary);
  MPSGPU_CHECK((bool)is, MPSGPU_INVALID, "MPS import: cannot open " + fn);
  int L = 0, bond = 0, gauge = 0;
  double nf = 1.0;
  is.read(reinterpret_cast<char*>(&L), sizeof(int));
  is.read(reinterpret_cast<char*>(&bond), sizeof(int));
  is.read(reinterpret_cast<char*>(&nf), sizeof(double));
  is.read(reinterpret_cast<char*>(&gauge), sizeof(int));
  MPSGPU_CHECK(is && L > 0 && L < (1 << 24), MPSGPU_INVALID, "MPS import: bad header in " + fn);
  std::vector<std::vector<double>> host(L);
  std::vector<int> dims(3 * L);
  std::vector<const double*> ptrs(L);
  for (int k = 0; k < L; k++) {
    int pos = 0;
    is.read(reinterpret_cast<char*>(&pos), sizeof(int));
    std::vector<int> d;
    read_array(is, d, host[k]);
    MPSGPU_CHECK(d.size() == 3, MPSGPU_BAD_SHAPE, "MPS import: a site is not a rank-3 array");
    for (int j = 0; j < 3; j++) dims[3 * k + j] = d[j];
    ptrs[k] = host[k].data();
  }
  mps_upload(c, s, L, dims.data(), ptrs.data(), nf);
  s.bond = bond;
  s.gauge = gauge;
}

void mpo_save_file(Context& c, const MpoDev& m, const std::string& fn) {
  std::ofstream os(fn, std::ios::binary | std::ios::trunc);
  MPSGPU_CHECK((bool)os, MPSGPU_INVALID, "MPO save: cannot open " + fn);
  const int L = m.L;
  os.write(reinterpret_cast<const char*>(&L), sizeof(int));
  std::vector<double> h;
  for (int k = 0; k < L; k++) {
    const auto& d = m.dims[k];
    h.resize(2LL * d[0] * d[1] * d[2] * d[3]);
    MPSGPU_CUDA(cudaMemcpyAsync(h.data(), m.W[k].p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    MPSGPU_CUDA(cudaStreamSynchronize(c.stream));
    write_array(os, {d[0], d[1], d[2], d[3]}, h.data());
  }
  MPSGPU_CHECK((bool)os, MPSGPU_INVALID, "MPO save: write failed for " + fn);
}

void mpo_load_file(Context& c, const std::string& fn, MpoDev& m) {
  std::ifstream is(fn, std::ios::binary);
  MPSGPU_CHECK((bool)is, MPSGPU_INVALID, "MPO load: cannot open " + fn);
  int L = 0;
  is.read(reinterpret_cast<char*>(&L), sizeof(int));
  MPSGPU_CHECK(is && L > 0 && L < (1 << 24), MPSGPU_INVALID, "MPO load: bad length in " + fn);
  std::vector<std::vector<double>> host(L);
  std::vector<int> dims(4 * L);
  std::vector<const double*> ptrs(L);
  for (int k = 0; k < L; k++) {
    std::vector<int> d;
    read_array(is, d, host[k]);
    MPSGPU_CHECK(d.size() == 4, MPSGPU_BAD_SHAPE, "MPO load: an operator is not a rank-4 array");
    for (int j = 0; j < 4; j++) dims[4 * k + j] = d[j];
    ptrs[k] = host[k].data();
  }
  mpo_upload(c, m, L, dims.data(), ptrs.data());
}

}  // namespace mpsgpu
