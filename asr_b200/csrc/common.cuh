// Shared definitions of the asr_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/asr_b200.h"

namespace asrb {

// last error message, per host thread (asr_last_error)
void set_error(const char* fmt, ...);
const char* get_error();

#define ASR_CUDA(call)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      ::asrb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));   \
      return ASR_ECUDA;                                                                        \
    }                                                                                          \
  } while (0)

#define ASR_TRY(call)               \
  do {                              \
    int s_ = (call);                \
    if (s_ != ASR_OK) return s_;    \
  } while (0)

// Makes a device current for the rest of a scope and makes the caller's device current again at its end, so that an
// entry point leaves the calling thread's current device as it found it.
struct DeviceGuard {
  int prev = -1;
  int set(int dev) {
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) cur = -1;
    if (cur != dev) {
      cudaError_t e = cudaSetDevice(dev);
      if (e != cudaSuccess) {
        set_error("cudaSetDevice(%d): %s", dev, cudaGetErrorString(e));
        return ASR_ECUDA;
      }
      prev = cur;
    }
    return ASR_OK;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
// NVTX range over a scope (an ABI call, a chain batch): names the span on the timeline of a profiler (nsys, ncu
// --nvtx); without one attached the calls do nothing
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
// consecutive named phases inside one scope: next() ends the open phase and starts the next; the last ends with the scope
struct NvtxPhase {
  bool open = false;
  void next(const char* name) {
    if (open) nvtxRangePop();
    nvtxRangePushA(name);
    open = true;
  }
  ~NvtxPhase() {
    if (open) nvtxRangePop();
  }
};

// every entry point that works on a device: an NVTX range named after the entry point, and its device made current
#define ASR_ON_DEVICE(dev)                  \
  ::asrb::NvtxRange nvtx_call_(__func__);   \
  ::asrb::DeviceGuard dguard_;              \
  ASR_TRY(dguard_.set(dev))

// device error codes written into a flag word (the first error wins)
enum DevErr : int {
  DERR_NONE = 0,
  DERR_EDGE = 1,          // the closure reached the edge of the site cluster (neighbour -1)
  DERR_TABLE_FULL = 2,    // hash table probe ran over its capacity
  DERR_STAB = 3,          // stabiliser size * orbit size != group order
  DERR_KEY = 4,           // configuration longer than the key width
  DERR_START = 5,         // start site not invariant
  DERR_WAIT = 6,          // a bounded wait on a bulk copy ran out
};

__device__ __forceinline__ void dev_fail(int* err, int code) { atomicCAS(err, 0, code); }

// ------------------------------------------------------------------------------------------------ complex helpers
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// modulus |a|
__host__ __device__ __forceinline__ double cmag(double2 a) { return hypot(a.x, a.y); }
// Smith's algorithm for complex division (R. L. Smith, CACM 5 (1962) 435)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  } else {
    double r = b.x / b.y, den = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
  }
}
// principal square root: Re >= 0, branch cut on the negative real axis (sign of Im taken from the argument)
__host__ __device__ __forceinline__ double2 csqrt_p(double2 z) {
  double m = hypot(z.x, z.y);
  if (m == 0.0) return make_double2(0.0, z.y);
  double t = sqrt(0.5 * (m + fabs(z.x)));
  if (z.x >= 0.0) return make_double2(t, z.y / (2.0 * t));
  return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}

}  // namespace asrb
