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

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <vector>

#include "dtw_device.cuh"
#include "dtw_pipe.cuh"
#include "odba_internal.h"
#include "pairwise_kernel.cuh"

namespace odba {

// Workspace of the one-warp-per-pair launches: the work counter and two edge
// buffers per resident warp.
template <typename T>
size_t whole_workspace_bytes(uint64_t max_len) {
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  const size_t slots = size_t(grid_size<T>()) * kWarpsPerBlock;
  return 256 + slots * 2 * stride * sizeof(T);
}

template <typename T, int RF>
int whole_pairwise_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                          uint64_t max_len, int os, int oe, unsigned long long pbeg,
                          unsigned long long npairs, T *dists, void *workspace, size_t ws_bytes,
                          cudaStream_t stream) {
  if (n < 2 || npairs == 0) return ODBA_OK;
  const size_t need = whole_workspace_bytes<T>(max_len);
  if (ws_bytes < need) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small");
  PairwiseArgs<T> a;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
  a.pbeg = pbeg;
  a.npairs = npairs;
  a.dists = dists;
  a.counter = static_cast<unsigned long long *>(workspace);
  a.edges = reinterpret_cast<T *>(static_cast<char *>(workspace) + 256);
  a.edge_stride = (max_len + 32 + 31) / 32 * 32;
  a.open_start = os;
  a.open_end = oe;
  cudaMemsetAsync(a.counter, 0, 16, stream);  // work counter and error word
  if (oe && !os)
    pairwise_kernel<T, RF, Tune<T>::RQ, true><<<grid_size<T>(), kWarpsPerBlock * 32, 0, stream>>>(a);
  else
    pairwise_kernel<T, RF, Tune<T>::RQ, false><<<grid_size<T>(), kWarpsPerBlock * 32, 0, stream>>>(a);
  return check_launch("pairwise DTW kernel");
}

}  // namespace odba

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
  __shared__ __align__(16) T stage_mem[kWarpsPerBlock * kStageElems];
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
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    job.x = series + offsets[task.first];
    job.m = int(lens[task.first]);
    job.y = series + offsets[task.second];
    job.n = int(lens[task.second]);
    job.r0 = os;
    job.open_end = oe != 0;
    T corner = T(0);
    sweep_pair<T, RF, RQ, true>(job, e0, e1, corner);
    if (lane == 0) dists[out] = pair_distance<T>(corner, job.m, job.n, os, oe);
  }
}

}  // namespace

template <typename T, int RF>
int whole_pairlist_launch(const T *series, const uint64_t *offsets, const uint64_t *lens,
                          const odba_pair_task *tasks, unsigned long long ntasks, uint64_t max_len,
                          T *dists, void *workspace, size_t ws_bytes, cudaStream_t stream) {
  if (ntasks == 0) return ODBA_OK;
  const size_t need = whole_workspace_bytes<T>(max_len);
  if (ws_bytes < need) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small");
  auto *counter = static_cast<unsigned long long *>(workspace);
  T *edges = reinterpret_cast<T *>(static_cast<char *>(workspace) + 256);
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  cudaMemsetAsync(counter, 0, 16, stream);  // work counter and error word
  unsigned long long blocks = (ntasks + kWarpsPerBlock - 1) / kWarpsPerBlock;
  int grid = grid_size<T>();
  if (blocks < (unsigned long long)grid) grid = int(blocks);
  pairlist_kernel<T, RF, Tune<T>::RQ><<<grid, kWarpsPerBlock * 32, 0, stream>>>(
      series, offsets, lens, tasks, ntasks, dists, counter, edges, stride);
  return check_launch("pair-list DTW kernel");
}

}  // namespace odba

// ---------------------------------------------------------------------------
// Few long pairs: swath-pipelined sweeps.
//
// With fewer pairs than warps (16 series of 1M-4M samples give 120 pairs for
// ~1776 resident warps), one warp per pair would leave most of the GPU idle.
// Here the unit of work is one swath of one pair: task k is swath k / P of
// pair k % P (P pairs), so swath s of a pair is always handed out after swath
// s - 1 of the same pair.  Each pair owns two edge buffers (swath s writes
// buffer s % 2 and reads buffer (s - 1) % 2), and every swath of every pair
// has its own progress word (rows stored so far), which the producing warp's
// lane 31 publishes with a gpu-scope release every 128 rows and at the end of
// its swath.  The consuming warp's lane 0 acquires the word before reading
// rows it has not seen published.  Why this cannot deadlock: a warp waits only
// on the previous swath of its pair, which was handed out earlier to a warp
// that is already running and waits only on earlier tasks, so the earliest
// unfinished task never waits.  Why two buffers suffice: swath s + 1
// overwrites row r of buffer (s - 1) % 2 only after swath s has published row
// r, and swath s reads its input rows before it computes (and publishes)
// them; swaths s and s + 2 do write one buffer at the same time, at different
// rows, which is why the progress words are per swath and not per buffer.
//
// Every wait is bounded: after kWaitLimitNs of polling (%globaltimer) the warp
// raises the launch's error word and continues; every other waiting warp sees
// the word and stops waiting, so a fault in the hand-off ends the launch
// quickly with the pairs it touched written as NaN.
namespace odba {
namespace {

template <typename T>
struct PipeArgs {
  const T *series;
  const uint64_t *offsets;
  const uint64_t *lens;
  int n;                         // series (all-vs-all) when list is null
  const odba_pair_task *list;    // pair list, or null for the upper triangle of n series
  unsigned long long pbeg;       // first pair of the range (upper triangle only)
  unsigned long long npairs;
  unsigned long long max_swaths;
  T *dists;
  unsigned long long *counter;
  unsigned *err;
  unsigned long long *progress;  // one word per (pair, swath): progress[pair * max_swaths + s]
  T *bstat;                      // per (pair, reference swath boundary): shortcut value or -1
  unsigned long long max_bounds;
  T *edges;                      // two buffers of edge_stride elements per pair
  unsigned long long edge_stride;
  int open_start, open_end;      // all-vs-all modes (a list carries its own)
  unsigned long long limit_ns;
};

template <typename T, int R, bool TRACK>
__device__ __forceinline__ EdgeStat<T> pipe_swath(const SwathJob<T> &job, const PipeGate &gate,
                                                  bool last, T &corner) {
  T col[R];
  const EdgeStat<T> st = sweep_swath<T, R, PipeGate, false, TRACK>(job, col, gate);
  if (last) corner = pick_column<T, R>(col, job.c0, job.n - 1);
  return st;
}

// TRACK: some pair may take the open-end shortcut (see sweep_pair)
template <typename T, int RF, int RQ, bool TRACK>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocksPerSM)
    swathpipe_kernel(PipeArgs<T> a) {
  constexpr int W = 32 * RF;
  __shared__ __align__(16) T stage_mem[kWarpsPerBlock * kStageElems];
  const int lane = threadIdx.x & 31;
  const unsigned long long ntasks = a.npairs * a.max_swaths;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= ntasks) break;
    const unsigned long long sw = q / a.npairs, qi = q - sw * a.npairs;
    int s, j, os, oe;
    unsigned long long out;
    if (a.list) {
      const odba_pair_task task = a.list[qi];
      s = int(task.first);
      j = int(task.second);
      os = int((task.out >> 62) & 1ull);
      oe = int((task.out >> 63) & 1ull);
      out = task.out & ((1ull << 62) - 1);
    } else {
      const long long p = (long long)(a.pbeg + a.npairs - 1 - qi);
      pair_of(p, a.n, s, j);
      os = a.open_start;
      oe = a.open_end;
      out = (unsigned long long)p;
    }
    SwathJob<T> job;
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    job.x = a.series + a.offsets[s];
    job.m = int(a.lens[s]);
    job.y = a.series + a.offsets[j];
    job.n = int(a.lens[j]);
    const unsigned long long nsw = (unsigned long long)(job.n + W - 1) / W;
    if (sw >= nsw) continue;
    const int c0 = int(sw) * W;
    const bool last = sw + 1 == nsw;
    T *b0 = a.edges + qi * 2 * a.edge_stride;
    T *b1 = b0 + a.edge_stride;
    job.c0 = c0;
    job.r0 = os;
    job.open_end = oe != 0;
    job.edge_in = sw ? (((sw - 1) & 1) ? b1 : b0) : nullptr;
    job.edge_out = last ? nullptr : ((sw & 1) ? b1 : b0);
    job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
    job.corner_init = c0 == 0 ? (job.r0 ? Num<T>::big() : T(0)) : (job.r0 ? T(0) : Num<T>::big());
    job.track = TRACK && swath_checks_shortcut<T>(c0, W, job.m, job.n, job.open_end, job.r0);
    PipeGate gate;
    unsigned long long *words = a.progress + qi * a.max_swaths;
    gate.prog_in = words + (sw ? sw - 1 : 0);
    gate.prog_out = words + sw;
    gate.err = a.err;
    gate.limit_ns = a.limit_ns;
    gate.avail = 0;
    T corner = T(0);
    const int width = job.n - c0 < W ? job.n - c0 : W;
    const int rneed = (width + 31) / 32;
    const int rq = (rneed + RQ - 1) / RQ * RQ;
    EdgeStat<T> st{Num<T>::big(), Num<T>::big()};
    if (rq >= RF) {
      st = pipe_swath<T, RF, TRACK>(job, gate, last, corner);
    } else {
      switch (rq / RQ) {
#define ODBA_PCASE(K)                                                       \
  case K:                                                                   \
    if constexpr (K * RQ < RF) st = pipe_swath<T, K * RQ, TRACK>(job, gate, last, corner); \
    break;
        ODBA_PCASE(1)
        ODBA_PCASE(2)
        ODBA_PCASE(3)
        ODBA_PCASE(4)
        ODBA_PCASE(5)
        ODBA_PCASE(6)
        ODBA_PCASE(7)
#undef ODBA_PCASE
        default:
          break;
      }
    }
    if (TRACK && job.track && lane == 31) {
      // this swath's right edge is the left edge of reference swath k + 1
      const unsigned long long k = (unsigned long long)(c0 + W) / kRefSwath - 1;
      T v;
      a.bstat[qi * a.max_bounds + k] = shortcut_fires<T>(st, job.m, v) ? v : T(-1);
    }
    if (last && lane == 0) {
      const bool bad = *reinterpret_cast<volatile unsigned *>(a.err) != 0;
      a.dists[out] = bad ? T(NAN) : pair_distance<T>(corner, job.m, job.n, os, oe);
    }
  }
}

// After the pipeline: a pair whose open-end shortcut fired on some checked
// edge takes its distance from the first such edge (the swaths after it ran
// anyway; the reference's stop there).  One thread per pair.
template <typename T>
__global__ void pipe_shortcut_kernel(PipeArgs<T> a) {
  const unsigned long long qi = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= a.npairs) return;
  if (*reinterpret_cast<volatile unsigned *>(a.err) != 0) return;
  int s, j, os, oe;
  unsigned long long out;
  if (a.list) {
    const odba_pair_task task = a.list[qi];
    s = int(task.first);
    j = int(task.second);
    os = int((task.out >> 62) & 1ull);
    oe = int((task.out >> 63) & 1ull);
    out = task.out & ((1ull << 62) - 1);
  } else {
    const long long p = (long long)(a.pbeg + a.npairs - 1 - qi);
    pair_of(p, a.n, s, j);
    os = a.open_start;
    oe = a.open_end;
    out = (unsigned long long)p;
  }
  if (!oe || os) return;
  const int m = int(a.lens[s]), n = int(a.lens[j]);
  for (int cnext = kRefSwath; cnext < n; cnext += kRefSwath) {
    if (cnext <= m) continue;
    const T v = a.bstat[qi * a.max_bounds + (unsigned long long)(cnext / kRefSwath - 1)];
    if (v >= T(0)) {
      a.dists[out] = pair_distance<T>(v, m, n, os, oe);
      return;
    }
  }
}

}  // namespace

// counter and error word | progress words | shortcut values | edge buffers
template <typename T>
size_t swathpipe_progress_bytes(unsigned long long npairs, uint64_t max_len) {
  constexpr int W = 32 * Tune<T>::RF;
  const unsigned long long max_swaths = (max_len + W - 1) / W;
  return (size_t(npairs) * max_swaths * 8 + 255) / 256 * 256;
}

inline unsigned long long swathpipe_max_bounds(uint64_t max_len) { return max_len / kRefSwath + 1; }

template <typename T>
size_t swathpipe_head_bytes(unsigned long long npairs, uint64_t max_len) {
  return 256 + swathpipe_progress_bytes<T>(npairs, max_len) +
         (size_t(npairs) * swathpipe_max_bounds(max_len) * sizeof(T) + 255) / 256 * 256;
}

template <typename T>
size_t swathpipe_workspace_bytes(unsigned long long npairs, uint64_t max_len) {
  const unsigned long long stride = (max_len + 32 + 31) / 32 * 32;
  return swathpipe_head_bytes<T>(npairs, max_len) + size_t(npairs) * 2 * stride * sizeof(T);
}

template <typename T>
int swathpipe_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                     const odba_pair_task *list, unsigned long long pbeg, unsigned long long npairs,
                     uint64_t max_len, int os, int oe, T *dists, void *workspace, size_t ws_bytes,
                     cudaStream_t stream, unsigned long long limit_ns) {
  if (npairs == 0) return ODBA_OK;
  if (ws_bytes < swathpipe_workspace_bytes<T>(npairs, max_len))
    return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small for the swath pipeline");
  constexpr int W = 32 * Tune<T>::RF;
  PipeArgs<T> a;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
  a.list = list;
  a.pbeg = pbeg;
  a.npairs = npairs;
  a.max_swaths = (max_len + W - 1) / W;
  a.dists = dists;
  char *base = static_cast<char *>(workspace);
  a.counter = reinterpret_cast<unsigned long long *>(base);
  a.err = reinterpret_cast<unsigned *>(base + 8);
  a.progress = reinterpret_cast<unsigned long long *>(base + 256);
  a.bstat = reinterpret_cast<T *>(base + 256 + swathpipe_progress_bytes<T>(npairs, max_len));
  a.max_bounds = swathpipe_max_bounds(max_len);
  const size_t head = swathpipe_head_bytes<T>(npairs, max_len);
  a.edges = reinterpret_cast<T *>(base + head);
  a.edge_stride = (max_len + 32 + 31) / 32 * 32;
  a.open_start = os;
  a.open_end = oe;
  a.limit_ns = limit_ns ? limit_ns : kWaitLimitNs;
  // the shortcut values need no clearing: every checked edge writes its entry
  if (cudaMemsetAsync(base, 0, 256 + swathpipe_progress_bytes<T>(npairs, max_len), stream) != cudaSuccess)
    return fail(ODBA_ERR_CUDA, "clearing the pipeline state failed");
  const bool track = list || (oe && !os);
  if (track) {
    swathpipe_kernel<T, Tune<T>::RF, Tune<T>::RQ, true><<<grid_size<T>(), kWarpsPerBlock * 32, 0, stream>>>(a);
    pipe_shortcut_kernel<T><<<unsigned((npairs + 127) / 128), 128, 0, stream>>>(a);
  } else {
    swathpipe_kernel<T, Tune<T>::RF, Tune<T>::RQ, false><<<grid_size<T>(), kWarpsPerBlock * 32, 0, stream>>>(a);
  }
  return check_launch("swath-pipelined DTW kernel");
}

template size_t swathpipe_workspace_bytes<float>(unsigned long long, uint64_t);
template size_t swathpipe_workspace_bytes<double>(unsigned long long, uint64_t);
template int swathpipe_launch<float>(const float *, const uint64_t *, const uint64_t *, int,
                                     const odba_pair_task *, unsigned long long, unsigned long long,
                                     uint64_t, int, int, float *, void *, size_t, cudaStream_t,
                                     unsigned long long);
template int swathpipe_launch<double>(const double *, const uint64_t *, const uint64_t *, int,
                                      const odba_pair_task *, unsigned long long, unsigned long long,
                                      uint64_t, int, int, double *, void *, size_t, cudaStream_t,
                                      unsigned long long);

}  // namespace odba

// ---------------------------------------------------------------------------
// Launch plans and the autotuner.
//
// Three plans compute the same distances (bit for bit): one warp per pair with
// 1024-column swaths (float; 512 for double), the same with half-width swaths,
// and the swath pipeline above (many warps per pair).  The plan is chosen per
// key (element size, floor(log2 max_len), floor(log2 pairs)): a plan pinned by
// odba_tune_set; else, in tuning mode, every eligible plan not yet measured for
// the key, in turn; else the fastest measured plan; else a rule of thumb (the
// pipeline when there are fewer pairs than resident warps and the longest
// series spans four or more swaths).  Measured throughput is pair-cells per
// second with max_len^2 per pair standing in for the cells (the lengths live
// on the device); CUDA events around each tuning launch are read back on the
// next call or by odba_tune_flush.
namespace odba {

namespace {

struct TuneCell {
  int pinned = 0;                        // a plan, or 0
  double rate[ODBA_PLAN_COUNT] = {0, 0, 0, 0};
};

struct Pending {
  int elem, lb, cb, plan;
  double cells;
  cudaEvent_t start, stop;
};

std::mutex g_tune_mu;
TuneCell g_tune[2][64][64];
bool g_tune_mode = false;
std::vector<Pending> g_pending;

int bucket_of(unsigned long long v) { return v ? 63 - __builtin_clzll(v) : 0; }

void harvest_locked(bool block) {
  std::vector<Pending> keep;
  for (auto &p : g_pending) {
    cudaError_t q = block ? cudaEventSynchronize(p.stop) : cudaEventQuery(p.stop);
    if (q == cudaErrorNotReady) {
      keep.push_back(p);
      continue;
    }
    float ms = 0;
    if (q == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess && ms > 0) {
      double &r = g_tune[p.elem][p.lb][p.cb].rate[p.plan];
      const double rate = p.cells / (ms * 1e-3);
      if (rate > r) r = rate;
    } else {
      cudaGetLastError();
    }
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  g_pending.swap(keep);
}

template <typename T>
bool plan_fits(int plan, unsigned long long npairs, uint64_t max_len, size_t ws_bytes) {
  constexpr int W = 32 * Tune<T>::RF;
  const unsigned long long slots = (unsigned long long)grid_size<T>() * kWarpsPerBlock;
  switch (plan) {
    case ODBA_PLAN_WHOLE_PAIR:
    case ODBA_PLAN_WHOLE_PAIR_HALF_SWATH:
      return ws_bytes >= whole_workspace_bytes<T>(max_len);
    case ODBA_PLAN_SWATH_PIPELINE:
      return npairs <= 2 * slots && (max_len + W - 1) / W >= 2 &&
             ws_bytes >= swathpipe_workspace_bytes<T>(npairs, max_len);
    default:
      return false;
  }
}

template <typename T>
int rule_of_thumb(unsigned long long npairs, uint64_t max_len) {
  constexpr int W = 32 * Tune<T>::RF;
  const unsigned long long slots = (unsigned long long)grid_size<T>() * kWarpsPerBlock;
  return (npairs < slots && (max_len + W - 1) / W >= 4) ? ODBA_PLAN_SWATH_PIPELINE
                                                         : ODBA_PLAN_WHOLE_PAIR;
}

// Chooses the plan; *measure tells the caller to time the launch for the table.
template <typename T>
int choose_plan(unsigned long long npairs, uint64_t max_len, size_t ws_bytes, bool *measure) {
  const int e = sizeof(T) == 8 ? 1 : 0, lb = bucket_of(max_len), cb = bucket_of(npairs);
  std::lock_guard<std::mutex> g(g_tune_mu);
  harvest_locked(false);
  TuneCell &c = g_tune[e][lb][cb];
  *measure = false;
  if (c.pinned && plan_fits<T>(c.pinned, npairs, max_len, ws_bytes)) return c.pinned;
  if (g_tune_mode) {
    for (int p = 1; p < ODBA_PLAN_COUNT; ++p) {
      if (c.rate[p] > 0 || !plan_fits<T>(p, npairs, max_len, ws_bytes)) continue;
      bool queued = false;
      for (auto &q : g_pending)
        if (q.elem == e && q.lb == lb && q.cb == cb && q.plan == p) queued = true;
      if (queued) continue;
      *measure = true;
      return p;
    }
  }
  int best = 0;
  for (int p = 1; p < ODBA_PLAN_COUNT; ++p)
    if (c.rate[p] > 0 && plan_fits<T>(p, npairs, max_len, ws_bytes) && (!best || c.rate[p] > c.rate[best]))
      best = p;
  if (best) return best;
  const int r = rule_of_thumb<T>(npairs, max_len);
  if (plan_fits<T>(r, npairs, max_len, ws_bytes)) return r;
  for (int p = 1; p < ODBA_PLAN_COUNT; ++p)
    if (plan_fits<T>(p, npairs, max_len, ws_bytes)) return p;
  return 0;
}

template <typename T>
void record_pending(unsigned long long npairs, uint64_t max_len, int plan, cudaEvent_t a,
                    cudaEvent_t b) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_pending.push_back(Pending{sizeof(T) == 8 ? 1 : 0, bucket_of(max_len), bucket_of(npairs), plan,
                              double(npairs) * double(max_len) * double(max_len), a, b});
}

template <typename T, typename F>
int run_planned(unsigned long long npairs, uint64_t max_len, size_t ws_bytes, cudaStream_t stream,
                F &&launch) {
  bool measure = false;
  const int plan = choose_plan<T>(npairs, max_len, ws_bytes, &measure);
  if (!plan) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "workspace too small");
  cudaEvent_t a = nullptr, b = nullptr;
  if (measure && (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)) {
    cudaGetLastError();
    measure = false;
  }
  if (measure) cudaEventRecord(a, stream);
  const int rc = launch(plan);
  if (measure) {
    cudaEventRecord(b, stream);
    if (rc == ODBA_OK) {
      record_pending<T>(npairs, max_len, plan, a, b);
    } else {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  }
  return rc;
}

}  // namespace

template <typename T>
size_t pairwise_workspace_bytes(uint64_t max_len) {
  // enough for every plan when there are at most as many pairs as resident warps
  const size_t slots = size_t(grid_size<T>()) * kWarpsPerBlock;
  return whole_workspace_bytes<T>(max_len) + swathpipe_head_bytes<T>(slots, max_len);
}

template <typename T>
size_t pairwise_workspace_bytes_n(unsigned long long npairs, uint64_t max_len) {
  const int r = rule_of_thumb<T>(npairs, max_len);
  return r == ODBA_PLAN_SWATH_PIPELINE ? swathpipe_workspace_bytes<T>(npairs, max_len)
                                       : whole_workspace_bytes<T>(max_len);
}

template <typename T>
int pairwise_range_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                          uint64_t max_len, int os, int oe, unsigned long long pbeg,
                          unsigned long long pend, T *dists, void *workspace, size_t ws_bytes,
                          cudaStream_t stream) {
  if (n < 2 || pend <= pbeg) return ODBA_OK;
  const unsigned long long npairs = pend - pbeg;
  return run_planned<T>(npairs, max_len, ws_bytes, stream, [&](int plan) {
    switch (plan) {
      case ODBA_PLAN_WHOLE_PAIR_HALF_SWATH:
        return whole_pairwise_launch<T, Tune<T>::RF / 2>(series, offsets, lens, n, max_len, os, oe,
                                                          pbeg, npairs, dists, workspace, ws_bytes,
                                                          stream);
      case ODBA_PLAN_SWATH_PIPELINE:
        return swathpipe_launch<T>(series, offsets, lens, n, nullptr, pbeg, npairs, max_len, os, oe,
                                   dists, workspace, ws_bytes, stream, 0);
      default:
        return whole_pairwise_launch<T, Tune<T>::RF>(series, offsets, lens, n, max_len, os, oe,
                                                      pbeg, npairs, dists, workspace, ws_bytes,
                                                      stream);
    }
  });
}

template <typename T>
int pairwise_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                    uint64_t max_len, int os, int oe, T *dists, void *workspace, size_t ws_bytes,
                    cudaStream_t stream) {
  if (n < 2) return ODBA_OK;
  return pairwise_range_launch<T>(series, offsets, lens, n, max_len, os, oe, 0,
                                  (unsigned long long)n * (n - 1) / 2, dists, workspace, ws_bytes,
                                  stream);
}

template <typename T>
int pairlist_launch(const T *series, const uint64_t *offsets, const uint64_t *lens,
                    const odba_pair_task *tasks, unsigned long long ntasks, uint64_t max_len,
                    T *dists, void *workspace, size_t ws_bytes, cudaStream_t stream) {
  if (ntasks == 0) return ODBA_OK;
  return run_planned<T>(ntasks, max_len, ws_bytes, stream, [&](int plan) {
    switch (plan) {
      case ODBA_PLAN_WHOLE_PAIR_HALF_SWATH:
        return whole_pairlist_launch<T, Tune<T>::RF / 2>(series, offsets, lens, tasks, ntasks,
                                                          max_len, dists, workspace, ws_bytes, stream);
      case ODBA_PLAN_SWATH_PIPELINE:
        return swathpipe_launch<T>(series, offsets, lens, 0, tasks, 0, ntasks, max_len, 0, 0, dists,
                                   workspace, ws_bytes, stream, 0);
      default:
        return whole_pairlist_launch<T, Tune<T>::RF>(series, offsets, lens, tasks, ntasks, max_len,
                                                      dists, workspace, ws_bytes, stream);
    }
  });
}

namespace {
// One warp waits on a progress word that nothing publishes, with the swath
// pipeline's own bounded wait.
__global__ void gate_selftest_kernel(unsigned long long *word, unsigned *err,
                                     unsigned long long limit_ns, int *seen) {
  if (threadIdx.x != 0) return;
  PipeGate gate;
  gate.prog_in = word;
  gate.prog_out = word + 1;
  gate.err = err;
  gate.limit_ns = limit_ns;
  gate.avail = 0;
  gate.wait_in(1);
  *seen = ld_acquire_gpu(word) != 0;
}
}  // namespace

int gate_selftest(unsigned long long limit_ns, cudaStream_t stream) {
  if (limit_ns == 0 || limit_ns > 10000000000ull)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "limit must be in (0, 10 s]");
  if (int rc = require_sm100()) return rc;
  char *buf = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void **>(&buf), 256, stream) != cudaSuccess)
    return fail(ODBA_ERR_OUT_OF_MEMORY, "self-test buffer");
  unsigned err = 0;
  int seen = 0;
  cudaMemsetAsync(buf, 0, 256, stream);
  gate_selftest_kernel<<<1, 32, 0, stream>>>(reinterpret_cast<unsigned long long *>(buf),
                                            reinterpret_cast<unsigned *>(buf + 64), limit_ns,
                                            reinterpret_cast<int *>(buf + 128));
  int rc = check_launch("wait self-test kernel");
  cudaMemcpyAsync(&err, buf + 64, sizeof err, cudaMemcpyDeviceToHost, stream);
  cudaMemcpyAsync(&seen, buf + 128, sizeof seen, cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(buf, stream);
  if (cudaStreamSynchronize(stream) != cudaSuccess) return fail(ODBA_ERR_CUDA, "wait self-test");
  if (rc) return rc;
  if (err) return fail(ODBA_ERR_TIMEOUT, "the wait ran out and raised the error word");
  return seen ? ODBA_OK : fail(ODBA_ERR_CUDA, "the wait returned without the word or a timeout");
}

int tune_set(int elem_size, int len_bucket, int count_bucket, int plan) {
  if ((elem_size != 4 && elem_size != 8) || len_bucket < 0 || len_bucket > 63 || count_bucket < 0 ||
      count_bucket > 63 || plan < 0 || plan >= ODBA_PLAN_COUNT)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "bad tuning key or plan");
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[elem_size == 8][len_bucket][count_bucket].pinned = plan;
  return ODBA_OK;
}

int tune_query(int elem_size, uint64_t max_len, unsigned long long npairs, size_t ws_bytes, int *plan,
               double *rates) {
  if (elem_size != 4 && elem_size != 8) return fail(ODBA_ERR_INVALID_ARGUMENT, "elem_size must be 4 or 8");
  bool measure = false;
  const int p = elem_size == 8 ? choose_plan<double>(npairs, max_len, ws_bytes, &measure)
                               : choose_plan<float>(npairs, max_len, ws_bytes, &measure);
  if (plan) *plan = p;
  if (rates) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    const TuneCell &c = g_tune[elem_size == 8][bucket_of(max_len)][bucket_of(npairs)];
    for (int i = 0; i < ODBA_PLAN_COUNT; ++i) rates[i] = c.rate[i];
  }
  return ODBA_OK;
}

void tune_mode(int on) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune_mode = on != 0;
}

int tune_flush() {
  std::lock_guard<std::mutex> g(g_tune_mu);
  harvest_locked(true);
  return ODBA_OK;
}

int tune_save(const char *path) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  harvest_locked(true);
  FILE *f = std::fopen(path, "w");
  if (!f) return fail(ODBA_ERR_IO, "cannot write the tuning table");
  std::fprintf(f, "# elem len_bucket count_bucket pinned rate_whole rate_half rate_pipeline\n");
  for (int e = 0; e < 2; ++e)
    for (int l = 0; l < 64; ++l)
      for (int c = 0; c < 64; ++c) {
        const TuneCell &t = g_tune[e][l][c];
        if (!t.pinned && !t.rate[1] && !t.rate[2] && !t.rate[3]) continue;
        std::fprintf(f, "%d %d %d %d %.6e %.6e %.6e\n", e ? 8 : 4, l, c, t.pinned, t.rate[1],
                     t.rate[2], t.rate[3]);
      }
  std::fclose(f);
  return ODBA_OK;
}

int tune_load(const char *path) {
  FILE *f = std::fopen(path, "r");
  if (!f) return fail(ODBA_ERR_IO, "cannot read the tuning table");
  std::lock_guard<std::mutex> g(g_tune_mu);
  char line[512];
  int rc = ODBA_OK;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    int e, l, c, pin;
    double r1, r2, r3;
    if (std::sscanf(line, "%d %d %d %d %lf %lf %lf", &e, &l, &c, &pin, &r1, &r2, &r3) != 7 ||
        (e != 4 && e != 8) || l < 0 || l > 63 || c < 0 || c > 63 || pin < 0 || pin >= ODBA_PLAN_COUNT) {
      rc = fail(ODBA_ERR_IO, "malformed tuning table line");
      break;
    }
    TuneCell &t = g_tune[e == 8][l][c];
    t.pinned = pin;
    t.rate[1] = r1;
    t.rate[2] = r2;
    t.rate[3] = r3;
  }
  std::fclose(f);
  return rc;
}

template size_t pairwise_workspace_bytes<float>(uint64_t);
template size_t pairwise_workspace_bytes<double>(uint64_t);
template size_t pairwise_workspace_bytes_n<float>(unsigned long long, uint64_t);
template size_t pairwise_workspace_bytes_n<double>(unsigned long long, uint64_t);
template int pairwise_launch<float>(const float *, const uint64_t *, const uint64_t *, int,
                                    uint64_t, int, int, float *, void *, size_t, cudaStream_t);
template int pairwise_range_launch<float>(const float *, const uint64_t *, const uint64_t *, int,
                                          uint64_t, int, int, unsigned long long, unsigned long long,
                                          float *, void *, size_t, cudaStream_t);
template int pairwise_range_launch<double>(const double *, const uint64_t *, const uint64_t *, int,
                                           uint64_t, int, int, unsigned long long, unsigned long long,
                                           double *, void *, size_t, cudaStream_t);
template int pairwise_launch<double>(const double *, const uint64_t *, const uint64_t *, int,
                                     uint64_t, int, int, double *, void *, size_t, cudaStream_t);
template int pairlist_launch<float>(const float *, const uint64_t *, const uint64_t *,
                                    const odba_pair_task *, unsigned long long, uint64_t, float *,
                                    void *, size_t, cudaStream_t);
template int pairlist_launch<double>(const double *, const uint64_t *, const uint64_t *,
                                     const odba_pair_task *, unsigned long long, uint64_t,
                                     double *, void *, size_t, cudaStream_t);

}  // namespace odba
