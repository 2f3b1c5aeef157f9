// The one-warp-per-pair all-pairs DTW kernel (approximateMedoidIndices'
// launch loop, dba.hpp:67-161, with DTWDistance's pair-distance epilogue,
// dtw.hpp:116-125, 242-257) and its launch-shape helpers.
//
// Private to the library's .cu files: everything is in an anonymous
// namespace, so every translation unit that includes this header compiles its
// own copy of the kernel into its own module.  dtw_pairwise.cu launches it
// with a caller workspace, dtw_pairwise_noalloc.cu with the scratch array it
// owns (a module of its own, so that only callers of that entry point load
// the array).
#ifndef ODBA_PAIRWISE_KERNEL_CUH
#define ODBA_PAIRWISE_KERNEL_CUH

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>

#include "dtw_device.cuh"

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
  unsigned long long pbeg;    // first pair of the range (upper-triangle index)
  unsigned long long npairs;  // pairs in the range
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
  if ((oe && !os) || (!oe && os)) {
    v = __fdiv_rn(__fsqrt_rn(float(corner)), float(m));
  } else {
    v = __fsqrt_rn(float(corner));
  }
  return T(v);
}

template <typename T, int R, bool TRACK>
__device__ __forceinline__ EdgeStat<T> run_swath(const SwathJob<T> &job, bool last, T &corner) {
  T col[R];
  const EdgeStat<T> st = sweep_swath<T, R, NoGate, false, TRACK>(job, col);
  if (last) corner = pick_column<T, R>(col, job.c0, job.n - 1);
  return st;
}

// The reference's open-end shortcut (dtw.hpp:74-129, open end without open
// start) is checked on the left edge of every 1024-column reference swath that
// starts past the last row: if that edge's value on the last row equals its
// shortcut minimum (ShortcutRows), the swath and all later ones stop and the
// distance is taken from that value -- from the sentinel it has just stored
// when the matrix has one row (dtw.hpp:113, 121).  swath_checks_shortcut: the
// swath [c0, c0 + W) whose right edge is such a left edge.
template <typename T>
__device__ __forceinline__ bool swath_checks_shortcut(int c0, int W, int m, int n, bool oe, int r0) {
  const int cnext = c0 + W;
  return oe && r0 == 0 && cnext < n && (cnext % kRefSwath) == 0 && cnext > m;
}

template <typename T>
__device__ __forceinline__ bool shortcut_fires(const EdgeStat<T> &st, int m, T &corner) {
  if (st.etop != st.emin) return false;
  corner = m == 1 ? Num<T>::big() : st.etop;
  return true;
}

// Full swaths use RF registers per lane (swath width 32*RF); the last, partial
// swath uses the smallest multiple of RQ registers that covers it.  TRACK:
// the pair may take the open-end shortcut (off at compile time for launches
// without an open end, so that their sweep carries no extra work).
template <typename T, int RF, int RQ, bool TRACK>
__device__ void sweep_pair(SwathJob<T> job, T *e0, T *e1, T &corner) {
  constexpr int W = 32 * RF;
  int k = 0;
  for (int c0 = 0; c0 < job.n; c0 += W, ++k) {
    const int width = job.n - c0 < W ? job.n - c0 : W;
    const bool last = c0 + W >= job.n;
    job.c0 = c0;
    job.track = TRACK && swath_checks_shortcut<T>(c0, W, job.m, job.n, job.open_end, job.r0);
    // ping-pong: swath k writes buffer k%2 and reads buffer (k+1)%2
    job.edge_in = c0 ? ((k & 1) ? e0 : e1) : nullptr;
    job.edge_out = last ? nullptr : ((k & 1) ? e1 : e0);
    job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
    job.corner_init = c0 == 0 ? (job.r0 ? Num<T>::big() : T(0)) : (job.r0 ? T(0) : Num<T>::big());
    const int rneed = (width + 31) / 32;
    const int rq = (rneed + RQ - 1) / RQ * RQ;
    EdgeStat<T> st{Num<T>::big(), Num<T>::big()};
    if (rq >= RF) {
      st = run_swath<T, RF, TRACK>(job, last, corner);
    } else {
      switch (rq / RQ) {
#define ODBA_CASE(K)                                          \
  case K:                                                     \
    if constexpr (K * RQ < RF) st = run_swath<T, K * RQ, TRACK>(job, last, corner); \
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
    if (TRACK && job.track) {
      st.emin = __shfl_sync(kFull, st.emin, 31);
      st.etop = __shfl_sync(kFull, st.etop, 31);
      if (shortcut_fires<T>(st, job.m, corner)) return;
    }
  }
}

template <typename T, int RF, int RQ, bool TRACK>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocksPerSM)
    pairwise_kernel(PairwiseArgs<T> a) {
  __shared__ __align__(16) T stage_mem[kWarpsPerBlock * kStageElems];
  const int lane = threadIdx.x & 31;
  const long long slot = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  T *e0 = a.edges + slot * 2 * a.edge_stride;
  T *e1 = e0 + a.edge_stride;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= a.npairs) break;
    const long long p = (long long)(a.pbeg + a.npairs - 1 - q);
    int s, j;
    pair_of(p, a.n, s, j);
    SwathJob<T> job;
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    job.x = a.series + a.offsets[s];
    job.m = int(a.lens[s]);
    job.y = a.series + a.offsets[j];
    job.n = int(a.lens[j]);
    job.r0 = a.open_start ? 1 : 0;
    job.open_end = a.open_end != 0;
    if ((unsigned long long)job.m + 32 > a.edge_stride) {
      // a first series longer than the max_len the edge buffers were sized
      // for: its edges would run into the next warp's buffers
      if (lane == 0) a.dists[p] = Num<T>::quiet_nan();
      continue;
    }
    T corner = T(0);
    sweep_pair<T, RF, RQ, TRACK>(job, e0, e1, corner);
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

// Resident blocks of pairwise_kernel on the current device, cached per device
// index (host threads may call at once: the cache entries are atomics, and a
// race only computes the same value twice).
template <typename T>
int grid_size() {
  static std::atomic<int> cached[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64) {
    const int c = cached[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, pairwise_kernel<T, Tune<T>::RF, Tune<T>::RQ, false>, kWarpsPerBlock * 32, 0);
  if (per_sm < 1) per_sm = 1;
  if (sms < 1) sms = 1;
  const int g = sms * per_sm;
  if (dev >= 0 && dev < 64) cached[dev].store(g, std::memory_order_relaxed);
  return g;
}

}  // namespace
}  // namespace odba

#endif  // ODBA_PAIRWISE_KERNEL_CUH
