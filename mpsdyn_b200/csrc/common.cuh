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

// Device-time accounting of the tensor-pipe GEMM launches: CUDA events are
// recorded on the launching stream around every GEMM while active and
// resolved once at the end (no synchronisation inside the sweep).
struct GemmProfiler {
  bool on = false;
  int every = 32;       // sample one GEMM launch in `every` (keeps event traffic low)
  long long seen = 0;   // GEMM launches since begin
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  double flops = 0.0;   // algorithmic flops of the sampled launches
  long long calls = 0;  // sampled launches
  bool sample() { return on && (seen++ % every) == 0; }
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      pool.push_back(e);
    }
    return pool[used++];
  }
  void reset() { used = 0; flops = 0.0; calls = 0; seen = 0; }
  // Sum of (end - start) over the recorded pairs; synchronises on the last event.
  double resolve_ms() {
    double ms = 0.0;
    if (used >= 2) cudaEventSynchronize(pool[used - 1]);
    for (size_t i = 0; i + 1 < used; i += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, pool[i], pool[i + 1]) == cudaSuccess) ms += t;
    }
    return ms;
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
