// All-vs-all DTW distances for the medoid pass: the work of
// approximateMedoidIndices' launch loop (dba.hpp:67-161) and the pair-distance
// epilogue of DTWDistance (dtw.hpp:116-125, 242-257), as one persistent launch.
//
// Every warp of the grid pulls pairs from a device work counter, largest pair
// index first (with length-sorted input that is roughly largest cost first),
// and sweeps the pair swath by swath with the register wavefront of
// dtw_device.cuh.  The swath right-edge column goes through a per-warp
// ping-pong buffer in global memory (L2-resident in practice).
//
// Output: the reference's upper-triangle layout, pair (s, j), s < j, at
// index s*n - s*(s+1)/2 + (j - s - 1) (clustering.cuh:4-6), with
//   dist = (T) sqrtf(C[m-1][n-1])           global / open modes
//   dist = (T)(sqrtf(C[m-1][n-1]) / m)      exactly one open end
// computed in float like the reference (sqrtf even for double, dtw.hpp:121,251,254).
#include <cuda_runtime.h>

#include <cstdint>

#include "dtw_device.cuh"
#include "odba_internal.h"

namespace odba {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kMinBlocksPerSM = 3;  // 12 warps per SM measured fastest (16 is slower, 20 spills)

template <typename T>
struct PairwiseArgs {
  const T *series;
  const uint64_t *offsets;
  const uint64_t *lens;
  int n;
  unsigned long long npairs;
  T *dists;
  unsigned long long *counter;
  T *edges;
  unsigned long long edge_stride;  // elements per edge buffer
  int open_start, open_end;
};

__device__ __forceinline__ long long row_start(long long s, long long n) {
  return s * n - s * (s + 1) / 2;
}

// Upper-triangle pair index -> (s, j).
__device__ __forceinline__ void pair_of(long long p, long long n, int &s_out, int &j_out) {
  const double b = 2.0 * double(n) - 1.0;
  long long s = (long long)((b - sqrt(b * b - 8.0 * double(p))) * 0.5);
  if (s < 0) s = 0;
  if (s > n - 2) s = n - 2;
  while (s + 1 <= n - 2 && row_start(s + 1, n) <= p) ++s;
  while (s > 0 && row_start(s, n) > p) --s;
  s_out = int(s);
  j_out = int(s + 1 + (p - row_start(s, n)));
}

template <typename T>
__device__ __forceinline__ T pair_distance(T corner, int m, int n, int os, int oe) {
  float v;
  if (m == 1 && oe && !os && n > kRefSwath) {
    // single-row matrix: the reference's open-end shortcut reads back the
    // sentinel it has just stored (dtw.hpp:113, 121)
    v = __fdiv_rn(__fsqrt_rn(float(Num<T>::big())), float(m));
  } else if ((oe && !os) || (!oe && os)) {
    v = __fdiv_rn(__fsqrt_rn(float(corner)), float(m));
  } else {
    v = __fsqrt_rn(float(corner));
  }
  return T(v);
}

template <typename T, int R>
__device__ __forceinline__ void run_swath(const SwathJob<T> &job, bool last, T &corner) {
  T col[R];
  sweep_swath<T, R>(job, col);
  if (last) corner = pick_column<T, R>(col, job.c0, job.n - 1);
}

// Full swaths use RF registers per lane (swath width 32*RF); the last, partial
// swath uses the smallest multiple of RQ registers that covers it.
template <typename T, int RF, int RQ>
__device__ void sweep_pair(SwathJob<T> job, T *e0, T *e1, T &corner) {
  constexpr int W = 32 * RF;
  int k = 0;
  for (int c0 = 0; c0 < job.n; c0 += W, ++k) {
    const int width = job.n - c0 < W ? job.n - c0 : W;
    const bool last = c0 + W >= job.n;
    job.c0 = c0;
    // ping-pong: swath k writes buffer k%2 and reads buffer (k+1)%2
    job.edge_in = c0 ? ((k & 1) ? e0 : e1) : nullptr;
    job.edge_out = last ? nullptr : ((k & 1) ? e1 : e0);
    job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
    job.corner_init = c0 == 0 ? (job.r0 ? Num<T>::big() : T(0)) : (job.r0 ? T(0) : Num<T>::big());
    const int rneed = (width + 31) / 32;
    const int rq = (rneed + RQ - 1) / RQ * RQ;
    if (rq >= RF) {
      run_swath<T, RF>(job, last, corner);
    } else {
      switch (rq / RQ) {
#define ODBA_CASE(K)                                          \
  case K:                                                     \
    if constexpr (K * RQ < RF) run_swath<T, K * RQ>(job, last, corner); \
    break;
        ODBA_CASE(1)
        ODBA_CASE(2)
        ODBA_CASE(3)
        ODBA_CASE(4)
        ODBA_CASE(5)
        ODBA_CASE(6)
        ODBA_CASE(7)
#undef ODBA_CASE
        default:
          break;
      }
    }
    // the next swath's lane 0 reads what this swath's lane 31 wrote
    __syncwarp();
  }
}

template <typename T, int RF, int RQ>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocksPerSM)
    pairwise_kernel(PairwiseArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const long long slot = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  T *e0 = a.edges + slot * 2 * a.edge_stride;
  T *e1 = e0 + a.edge_stride;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= a.npairs) break;
    const long long p = (long long)(a.npairs - 1 - q);
    int s, j;
    pair_of(p, a.n, s, j);
    SwathJob<T> job;
    job.x = a.series + a.offsets[s];
    job.m = int(a.lens[s]);
    job.y = a.series + a.offsets[j];
    job.n = int(a.lens[j]);
    job.r0 = a.open_start ? 1 : 0;
    job.open_end = a.open_end != 0;
    T corner = T(0);
    sweep_pair<T, RF, RQ>(job, e0, e1, corner);
    if (lane == 0) a.dists[p] = pair_distance<T>(corner, job.m, job.n, a.open_start, a.open_end);
  }
}

template <typename T>
struct Tune;
template <>
struct Tune<float> {
  static constexpr int RF = 32, RQ = 4;
};
template <>
struct Tune<double> {
  static constexpr int RF = 16, RQ = 4;
};

template <typename T>
int grid_size() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && cached[dev]) return cached[dev];
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ>, kWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int g = sms * per_sm;
  if (dev < 64) cached[dev] = g;
  return g;
}

}  // namespace

template <typename T>
size_t pairwise_workspace_bytes(uint64_t max_len) {
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  const size_t slots = size_t(grid_size<T>()) * kWarpsPerBlock;
  return 256 + slots * 2 * stride * sizeof(T);
}

template <typename T>
int pairwise_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                    uint64_t max_len, int os, int oe, T *dists, void *workspace, size_t ws_bytes,
                    cudaStream_t stream) {
  if (n < 2) return ODBA_OK;
  const size_t need = pairwise_workspace_bytes<T>(max_len);
  if (ws_bytes < need) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small");
  PairwiseArgs<T> a;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
  a.npairs = (unsigned long long)n * (n - 1) / 2;
  a.dists = dists;
  a.counter = static_cast<unsigned long long *>(workspace);
  a.edges = reinterpret_cast<T *>(static_cast<char *>(workspace) + 256);
  a.edge_stride = (max_len + 32 + 31) / 32 * 32;
  a.open_start = os;
  a.open_end = oe;
  cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream);
  pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ>
      <<<grid_size<T>(), kWarpsPerBlock * 32, 0, stream>>>(a);
  return check_launch("pairwise DTW kernel");
}

template size_t pairwise_workspace_bytes<float>(uint64_t);
template size_t pairwise_workspace_bytes<double>(uint64_t);
template int pairwise_launch<float>(const float *, const uint64_t *, const uint64_t *, int,
                                    uint64_t, int, int, float *, void *, size_t, cudaStream_t);
template int pairwise_launch<double>(const double *, const uint64_t *, const uint64_t *, int,
                                     uint64_t, int, int, double *, void *, size_t, cudaStream_t);

}  // namespace odba

// ---------------------------------------------------------------------------
// All-pairs DTW without any device allocation.
//
// Some callers cannot allocate device memory where they call us: a serving or
// real-time loop that forbids allocation after start-up (cudaMalloc can
// synchronize the device and stall unrelated streams, and can fail under
// memory pressure mid-run), or a host application that owns the device's whole
// memory budget and gives its plugins no allocator.  For them the work counter
// and the per-warp swath-edge buffers live in one fixed array in the library's
// own device memory instead of a caller workspace.  The array exists once per
// device for as long as the library is loaded; its size caps the longest
// series and the number of warps that run at once (fewer warps for longer
// series).  Every call uses the same array: the work counter is cleared at the
// start of each call, nothing else needs clearing, and calls that overlap on
// the GPU (two streams, or two host threads) race on it and must be serialized
// by the caller.
namespace odba {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
void *g_noalloc_ptr[kMaxDevices] = {nullptr};

// Looks up (once per device, with that device current) the device address of
// g_noalloc_scratch; host code must not use the symbol itself as an address.
int noalloc_scratch_ptr(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ODBA_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return fail(ODBA_ERR_UNSUPPORTED_DEVICE, "device index out of range");
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return fail(ODBA_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
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
  if (int rc = noalloc_scratch_ptr(&scratch)) return rc;
  int grid = grid_size<T>();
  const size_t fit = capacity / per_block;
  if (size_t(grid) > fit) grid = int(fit);
  PairwiseArgs<T> a;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
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
  pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ><<<grid, kWarpsPerBlock * 32, 0, stream>>>(a);
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

// ---------------------------------------------------------------------------
// Pairs from a task list: many independent jobs (each its own set of series,
// its own alignment mode) in one persistent launch.  The caller orders the
// tasks (largest m*n first keeps the tail short); each warp takes the next
// task from the device counter.
namespace odba {
namespace {

template <typename T, int RF, int RQ>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocksPerSM)
    pairlist_kernel(const T *series, const uint64_t *offsets, const uint64_t *lens,
                    const odba_pair_task *tasks, unsigned long long ntasks, T *dists,
                    unsigned long long *counter, T *edges, unsigned long long edge_stride) {
  const int lane = threadIdx.x & 31;
  const long long slot = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  T *e0 = edges + slot * 2 * edge_stride;
  T *e1 = e0 + edge_stride;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= ntasks) break;
    const odba_pair_task task = tasks[q];
    const int os = int((task.out >> 62) & 1ull), oe = int((task.out >> 63) & 1ull);
    const unsigned long long out = task.out & ((1ull << 62) - 1);
    SwathJob<T> job;
    job.x = series + offsets[task.first];
    job.m = int(lens[task.first]);
    job.y = series + offsets[task.second];
    job.n = int(lens[task.second]);
    job.r0 = os;
    job.open_end = oe != 0;
    T corner = T(0);
    sweep_pair<T, RF, RQ>(job, e0, e1, corner);
    if (lane == 0) dists[out] = pair_distance<T>(corner, job.m, job.n, os, oe);
  }
}

}  // namespace

template <typename T>
int pairlist_launch(const T *series, const uint64_t *offsets, const uint64_t *lens,
                    const odba_pair_task *tasks, unsigned long long ntasks, uint64_t max_len,
                    T *dists, void *workspace, size_t ws_bytes, cudaStream_t stream) {
  if (ntasks == 0) return ODBA_OK;
  const size_t need = pairwise_workspace_bytes<T>(max_len);
  if (ws_bytes < need) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small");
  auto *counter = static_cast<unsigned long long *>(workspace);
  T *edges = reinterpret_cast<T *>(static_cast<char *>(workspace) + 256);
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream);
  unsigned long long blocks = (ntasks + kWarpsPerBlock - 1) / kWarpsPerBlock;
  int grid = grid_size<T>();
  if (blocks < (unsigned long long)grid) grid = int(blocks);
  pairlist_kernel<T, Tune<T>::RF, Tune<T>::RQ><<<grid, kWarpsPerBlock * 32, 0, stream>>>(
      series, offsets, lens, tasks, ntasks, dists, counter, edges, stride);
  return check_launch("pair-list DTW kernel");
}

template int pairlist_launch<float>(const float *, const uint64_t *, const uint64_t *,
                                    const odba_pair_task *, unsigned long long, uint64_t, float *,
                                    void *, size_t, cudaStream_t);
template int pairlist_launch<double>(const double *, const uint64_t *, const uint64_t *,
                                     const odba_pair_task *, unsigned long long, uint64_t,
                                     double *, void *, size_t, cudaStream_t);

}  // namespace odba
