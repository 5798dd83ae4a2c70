// Allocation-free variant of the final-state max|v| reduction.
//
// Some callers cannot allocate GPU memory at the point where they need this
// diagnostic: a Fortran driver whose device data is owned and pre-sized by
// OpenACC data regions (allocation audits require zero allocations during
// time stepping), code running while a memory pool is frozen, or a host that
// must not grow its GPU footprint after start-up.  wql3d_max_abs_noalloc lets
// them reduce a device array they already own into an output they already
// own, using only the fixed scratch below.
//
// Scratch: one static device array of per-block partial maxima and flags,
// 65536 slots of 16 bytes (1 MiB), one slot per block of 8192 elements, hence
// the WQL3D_NOALLOC_MAX_ELEMENTS limit.  It is part of the library image, so
// every GPU that loads libwql3d.so holds it until the process exits.  All calls share it: two calls
// whose kernels overlap on the GPU (different streams, no ordering between
// them) race on the scratch and may return wrong results.  Calls ordered on
// one stream are safe.  Nothing in the scratch needs to start at zero: every
// slot that the second kernel reads is written by the first kernel of the
// same call, so stale contents of an earlier, larger call are never read.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "wql3d.h"

namespace wql3d {
void set_last_error(const std::string &msg);  // wql3d_api.cu: text returned by wql3d_last_error()
}

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 32;
constexpr long long kChunk = (long long)kThreads * kPerThread;   // elements per block
constexpr int kMaxBlocks = 65536;                                  // scratch slots

struct NoallocSlot {
  double maxabs;
  int nonfinite;
  int pad;
};

static_assert((long long)kMaxBlocks * kChunk == WQL3D_NOALLOC_MAX_ELEMENTS, "scratch size and limit disagree");

static __device__ __align__(256) NoallocSlot g_noalloc_scratch[kMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
NoallocSlot *g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void k_noalloc_partial(const double *__restrict__ a, long long n, NoallocSlot *slots) {
  __shared__ double sm[kThreads];
  __shared__ int sf[kThreads];
  const long long base = (long long)blockIdx.x * kChunk;
  double m = 0.0;
  int bad = 0;
  for (int k = 0; k < kPerThread; ++k) {
    long long i = base + (long long)k * kThreads + threadIdx.x;
    if (i < n) {
      double v = fabs(a[i]);
      if (!(v <= 1.7976931348623157e308)) bad = 1;
      else if (v > m) m = v;
    }
  }
  sm[threadIdx.x] = m;
  sf[threadIdx.x] = bad;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + s]);
      sf[threadIdx.x] |= sf[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    slots[blockIdx.x].maxabs = sm[0];
    slots[blockIdx.x].nonfinite = sf[0];
  }
}

__global__ void k_noalloc_final(const NoallocSlot *slots, int nblocks, double *result, int32_t *nonfinite) {
  __shared__ double sm[1024];
  __shared__ int sf[1024];
  double m = 0.0;
  int bad = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    m = fmax(m, slots[i].maxabs);
    bad |= slots[i].nonfinite;
  }
  sm[threadIdx.x] = m;
  sf[threadIdx.x] = bad;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + s]);
      sf[threadIdx.x] |= sf[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *result = sm[0];
    if (nonfinite) *nonfinite = sf[0];
  }
}

// Device address of the scratch for the current device, looked up once per
// device (with that device current) and cached.  The same first call also
// asks for both kernels' attributes: with lazy module loading (the CUDA 12
// default) that is what puts the kernels' code on the device, so after the
// first call on a device no later call makes the driver reserve memory.  The
// cached address belongs to the device's primary context: after a
// cudaDeviceReset the cached address is stale and the entry point must not be
// called again in that process.
int scratch_for_current_device(NoallocSlot **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    wql3d::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return WQL3D_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    wql3d::set_last_error("device ordinal out of range for the scratch table");
    return WQL3D_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      wql3d::set_last_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      return WQL3D_ECUDA;
    }
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, k_noalloc_partial);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_noalloc_final);
    if (e != cudaSuccess) {
      wql3d::set_last_error(std::string("cudaFuncGetAttributes(noalloc kernels): ") + cudaGetErrorString(e));
      return WQL3D_ECUDA;
    }
    g_scratch_ptr[dev] = (NoallocSlot *)p;
  }
  *out = g_scratch_ptr[dev];
  return WQL3D_OK;
}

}  // namespace

extern "C" {

int wql3d_max_abs_noalloc(const double *array, int64_t n, double *result, int32_t *nonfinite, void *stream) {
  if (n < 0 || (n > 0 && !array) || !result) {
    wql3d::set_last_error("wql3d_max_abs_noalloc: null array/result or negative length");
    return WQL3D_EINVAL;
  }
  if (n > WQL3D_NOALLOC_MAX_ELEMENTS) {
    wql3d::set_last_error("wql3d_max_abs_noalloc: n = " + std::to_string((long long)n) +
                    " exceeds the fixed scratch limit of " + std::to_string((long long)WQL3D_NOALLOC_MAX_ELEMENTS) +
                    " elements; use wql3d_final_state or reduce in pieces");
    return WQL3D_EINVAL;
  }
  NoallocSlot *slots = nullptr;
  int rc = scratch_for_current_device(&slots);
  if (rc != WQL3D_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int nblocks = (int)((n + kChunk - 1) / kChunk);
  if (nblocks > 0) k_noalloc_partial<<<nblocks, kThreads, 0, s>>>(array, (long long)n, slots);
  k_noalloc_final<<<1, 1024, 0, s>>>(slots, nblocks, result, nonfinite);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    wql3d::set_last_error(std::string("wql3d_max_abs_noalloc launch: ") + cudaGetErrorString(e));
    return WQL3D_ECUDA;
  }
  return WQL3D_OK;
}

}  // extern "C"
