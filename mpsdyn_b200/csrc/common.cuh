// Shared device/host helpers of the mpsgpu library: complex FP64 arithmetic on
// double2 (re, im interleaved, the reference's complex_t layout), error
// plumbing and the per-context state every kernel launcher receives.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <stdexcept>
#include <vector>

#include "mpsgpu.h"

namespace mpsgpu {

typedef double2 cplx;

__host__ __device__ inline cplx cmake(double re, double im) { return make_double2(re, im); }
__host__ __device__ inline cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
// a * conj(b)
__host__ __device__ inline cplx cmulc(cplx a, cplx b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
__host__ __device__ inline cplx ccmul(cplx a, cplx b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Error carrying a status code; every C-ABI function catches it.
struct Error : public std::runtime_error {
  mpsgpu_status status;
  Error(mpsgpu_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

#define MPSGPU_CUDA(call)                                                        \
  do {                                                                           \
    cudaError_t _e = (call);                                                     \
    if (_e != cudaSuccess) {                                                     \
      throw ::mpsgpu::Error(_e == cudaErrorMemoryAllocation ? MPSGPU_OOM         \
                                                            : MPSGPU_CUDA_ERROR, \
                            std::string(#call) + ": " + cudaGetErrorString(_e)); \
    }                                                                            \
  } while (0)

#define MPSGPU_CHECK(cond, status, msg)                    \
  do {                                                     \
    if (!(cond)) throw ::mpsgpu::Error((status), (msg));   \
  } while (0)

// Device-time accounting of the hot kernels by class: while on, CUDA events
// are recorded on the launching stream around one launch in `every` of each
// class, with the launch's algorithmic work (flops, or bytes for the
// bandwidth-bound Lanczos step); resolved once at the end (no
// synchronisation inside the sweep).  Alone on the device, a sampled
// launch's event time is its own duration.
struct GemmProfiler {
  // 0: complex FP64 GEMMs on the DMMA pipe (zgemm, the fused contractions);
  // 1: split-precision GEMM on tcgen05 (work = BF16 tensor flops);
  // 2: the fused Lanczos step (work = bytes); 3: Householder QR (flops);
  // 4: the split products' operand passes (limb planes, MPO legs, sums of
  // K chunks; work = bytes)
  enum { GEMM64 = 0, SPLIT = 1, LZSTEP = 2, QR = 3, SPLITOPS = 4, NCLS = 5 };
  bool on = false;
  int every = 32;
  long long seen[NCLS] = {};
  std::vector<cudaEvent_t> pool;
  std::vector<int> tags;  // class of each recorded pair
  size_t used = 0;
  double work[NCLS] = {};
  long long calls[NCLS] = {};
  double ms[NCLS] = {};  // filled by resolve()
  bool sample(int cls) { return on && (seen[cls]++ % every) == 0; }
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      pool.push_back(e);
    }
    return pool[used++];
  }
  void reset() {
    used = 0;
    tags.clear();
    for (int c = 0; c < NCLS; c++) seen[c] = calls[c] = 0, work[c] = ms[c] = 0.0;
  }
  // Sums (end - start) per class over the recorded pairs; synchronises on
  // the last event.
  void resolve() {
    for (int c = 0; c < NCLS; c++) ms[c] = 0.0;
    if (used >= 2) cudaEventSynchronize(pool[used - 1]);
    for (size_t i = 0; i + 1 < used; i += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, pool[i], pool[i + 1]) == cudaSuccess) ms[tags[i / 2]] += t;
    }
  }
  ~GemmProfiler() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// Launch bookkeeping: every kernel launcher calls after_launch().
struct Stream {
  cudaStream_t s = nullptr;
  long long* launches = nullptr;
  GemmProfiler* prof = nullptr;
};

inline void after_launch(const Stream& st) {
  if (st.launches) ++(*st.launches);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error(MPSGPU_CUDA_ERROR, std::string("kernel launch: ") + cudaGetErrorString(e));
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Brackets one launch of class `cls` with profiler events when it is sampled.
struct ProfScope {
  GemmProfiler* p = nullptr;
  cudaStream_t s = nullptr;
  int cls = 0;
  double work = 0.0;
  ProfScope(const Stream& st, int cls_, double work_) : s(st.s), cls(cls_), work(work_) {
    if (st.prof && st.prof->sample(cls)) {
      cudaEvent_t e0 = st.prof->next();
      if (e0 && cudaEventRecord(e0, s) == cudaSuccess) p = st.prof;
    }
  }
  ~ProfScope() {
    if (!p) return;
    cudaEvent_t e1 = p->next();
    if (e1 && cudaEventRecord(e1, s) == cudaSuccess) {
      p->tags.push_back(cls);
      p->work[cls] += work;
      p->calls[cls]++;
    } else if (p->used > 0) {
      p->used -= e1 ? 2 : 1;  // drop the unmatched start event
    }
  }
};

// One-time set-up per device (kernel attributes live in each device's
// context): true until mark_device_done has recorded the current device.
// The set-up is idempotent, so threads that race on the first use all do it
// before any of them records it, and a thread that sees the mark knows the
// set-up is complete.
inline bool device_needs_setup(const std::atomic<unsigned long long>& done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
  return (done.load() & (1ull << dev)) == 0;
}
inline void mark_device_done(std::atomic<unsigned long long>& done) {
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) done.fetch_or(1ull << dev);
}

}  // namespace mpsgpu
