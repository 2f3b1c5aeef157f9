// All-pairs DTW without any device allocation.
//
// Some callers cannot allocate device memory where they call us: a serving or
// real-time loop that forbids allocation after start-up (cudaMalloc can
// synchronize the device and stall unrelated streams, and can fail under
// memory pressure mid-run), or a host application that owns the device's whole
// memory budget and gives its plugins no allocator.  For them the work counter
// and the per-warp swath-edge buffers live in one fixed array in the library's
// own device memory instead of a caller workspace.
//
// The array is a device global of this file's module, so it is mapped when the
// module loads: with CUDA's lazy module loading (the default) at the first call
// of this entry point on a device, otherwise when the library's modules load
// into the context.  It then stays until the context ends.  Its size caps the
// longest series and the number of warps that run at once (fewer warps for
// longer series).  Every call uses the same array: the work counter is cleared
// at the start of each call, nothing else needs clearing, and calls that
// overlap on the GPU (two streams, or two host threads) race on it and must be
// serialized by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "odba_internal.h"
#include "opendba_b200.h"
#include "pairwise_kernel.cuh"

namespace odba {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;

// The device address of g_noalloc_scratch per device, with the context it was
// looked up in.  Host threads may call at once, so the cache is read and
// written under a mutex.
struct ScratchCache {
  std::mutex mu;
  CUcontext ctx[kMaxDevices] = {};
  void *ptr[kMaxDevices] = {};
};

ScratchCache &scratch_cache() {
  static ScratchCache cache;
  return cache;
}

// The calling thread's current context, through the runtime's driver entry
// point (the library does not link the driver library itself); null if the
// driver does not offer cuCtxGetCurrent.
CUcontext current_context() {
  using GetCurrent = CUresult (*)(CUcontext *);
  static const GetCurrent get_current = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return GetCurrent(nullptr);
    return reinterpret_cast<GetCurrent>(f);
  }();
  CUcontext c = nullptr;
  if (get_current) get_current(&c);
  return c;
}

// Device address of g_noalloc_scratch for the current device.  The name of the
// array in host code is a host-side stand-in, not a device address, so the
// address comes from cudaGetSymbolAddress, with the device current.  It is
// looked up again on every call whose stream is not capturing (a device reset
// or a new context may load the module at another address); a capturing call
// reuses the address found earlier in the same context, and fails if there is
// none.
int noalloc_scratch_ptr(cudaStream_t stream, void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ODBA_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return fail(ODBA_ERR_UNSUPPORTED_DEVICE, "device index out of range");
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &capture);
  if (e != cudaSuccess) return fail(ODBA_ERR_CUDA, "cudaStreamIsCapturing failed");
  const CUcontext ctx = current_context();
  ScratchCache &cache = scratch_cache();
  std::lock_guard<std::mutex> lock(cache.mu);
  if (capture == cudaStreamCaptureStatusNone) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(ODBA_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    cache.ctx[dev] = ctx;
    cache.ptr[dev] = p;
  } else if (!cache.ptr[dev] || cache.ctx[dev] != ctx) {
    return fail(ODBA_ERR_INVALID_ARGUMENT,
                "no scratch address for this device and context: make one call outside stream "
                "capture first");
  }
  *out = cache.ptr[dev];
  return ODBA_OK;
}

template <typename T>
int pairwise_noalloc(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                     uint64_t max_len, int os, int oe, T *dists, cudaStream_t stream) {
  if (n < 0 || (n >= 2 && (!series || !offsets || !lens || !dists)))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or negative series count");
  if (max_len == 0) return fail(ODBA_ERR_INVALID_ARGUMENT, "max_len must be at least 1");
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  const size_t per_block = size_t(kWarpsPerBlock) * 2 * stride * sizeof(T);
  const size_t capacity = kNoAllocScratchBytes - 256;
  if (max_len > (1ull << 31) || per_block > capacity)
    return fail(ODBA_ERR_INVALID_ARGUMENT,
                "max_len exceeds the no-allocation limit: the 64 MiB scratch array holds the "
                "swath edges of one block of warps for series of up to 2,097,088 samples");
  if (int rc = require_sm100()) return rc;
  if (n < 2) return ODBA_OK;
  void *scratch = nullptr;
  if (int rc = noalloc_scratch_ptr(stream, &scratch)) return rc;
  int grid = grid_size<T>();
  const size_t fit = capacity / per_block;
  if (size_t(grid) > fit) grid = int(fit);
  PairwiseArgs<T> a;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
  a.pbeg = 0;
  a.npairs = (unsigned long long)n * (n - 1) / 2;
  a.dists = dists;
  a.counter = static_cast<unsigned long long *>(scratch);
  a.edges = reinterpret_cast<T *>(static_cast<char *>(scratch) + 256);
  a.edge_stride = stride;
  a.open_start = os ? 1 : 0;
  a.open_end = oe ? 1 : 0;
  // the counter is the only state that must start at zero
  cudaError_t e = cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(ODBA_ERR_CUDA, "clearing the work counter failed");
  if (a.open_end && !a.open_start)
    pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ, true><<<grid, kWarpsPerBlock * 32, 0, stream>>>(a);
  else
    pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ, false><<<grid, kWarpsPerBlock * 32, 0, stream>>>(a);
  return check_launch("pairwise DTW kernel (no-allocation variant)");
}

}  // namespace
}  // namespace odba

extern "C" int odba_dtw_pairwise_noalloc_f32(const float *series, const uint64_t *offsets,
                                             const uint64_t *lens, int n, uint64_t max_len,
                                             int use_open_start, int use_open_end, float *dists,
                                             void *stream) {
  return odba::pairwise_noalloc<float>(series, offsets, lens, n, max_len, use_open_start,
                                       use_open_end, dists, static_cast<cudaStream_t>(stream));
}
