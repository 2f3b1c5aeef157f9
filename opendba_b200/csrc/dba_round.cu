// One DBA round on the device: DBAUpdate (dba.hpp:432-848) with the centroid
// update of updateCentroid (dba.hpp:374-423), for all members in one pass.
//
//  1. plan:      per member the orientation (the centroid goes on the Y axis
//                when open_end and it is the shorter one, dba.hpp:497-501),
//                the size and offset of its 2-bit path, and its path-file slot.
//  2. path DTW:  persistent launch, one warp per member, swath by swath with the
//                register wavefront of dtw_path.cuh; records every move and the
//                right-edge minima the open-end shortcut needs.
//  3. backtrack: one thread per member walks its path from the end cell back to
//                (0, 0) (updateCentroid's loop) and stores, per centroid index,
//                the contiguous range of member samples that index receives --
//                a path crosses every centroid index in one contiguous run.
//                Optionally it also emits the path as (i, j, move) triples in
//                the order of the reference's path file (io_utils.hpp:287-323).
//  4. reduce:    one thread per centroid index adds the member samples in the
//                reference's exact order -- members in order, each member's
//                samples from its last path row down to its first -- then
//                divides by the pile-up count in T (dba.hpp:820-822) and takes
//                max |old - new| in double (dba.hpp:830-836).
// The float sums are therefore bit-identical to the reference's serialized
// single-thread atomicAdd sequence, without atomics.
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cstdint>
#include <vector>

#include "dtw_path.cuh"
#include "dtw_pipe.cuh"
#include "odba_internal.h"

namespace odba {

namespace {

constexpr int kRoundWarps = 4;
constexpr int kReduceWarps = 4;  // centroid indices per block of the ordered reducer
constexpr int kReduceThreads = kReduceWarps * 32;
constexpr int kPlanThreads = 1024;  // members per step of the plan's prefix sums
constexpr int kRankMembers = 16384;  // longest-first task order computed up to this many members
// move codes of the reference's path matrix (dtw.hpp:10-16); kMoveDiag,
// kMoveRight and kMoveUp come with the path sweep (dtw_path.cuh)
constexpr int kMaxMoveNil = 255, kMoveOpenRight = 4, kMoveNilOpenRight = 5;

template <typename T>
struct PathTune;
// RF: registers (columns) per lane of a full swath; the last, partial swath
// of a member takes a multiple of RQ.  In the full-path round a last swath
// within PAD registers of RF is swept at RF (the extra columns past the
// series' end are swept and never walked), so that one loop body, not two of
// nearly the same size, runs in most warps.
template <>
struct PathTune<float> {
  static constexpr int RF = 32, RQ = 4, PAD = 4;
};
template <>
struct PathTune<double> {
  static constexpr int RF = 16, RQ = 4, PAD = 0;
};

// Registers per lane of a full-path swath `width` columns wide (at most
// 32 * RF).
template <typename T>
__host__ __device__ inline int path_regs(int width) {
  constexpr int RF = PathTune<T>::RF, RQ = PathTune<T>::RQ;
  const int rq = ((width + 31) / 32 + RQ - 1) / RQ * RQ;
  return rq >= RF - PathTune<T>::PAD ? RF : rq;
}

// Geometry of one member's cost matrix, identical on host and device.
struct MemberGeom {
  int flip, m, n, r0, swaths, steps;
  unsigned long long words;
};

template <typename T>
__host__ __device__ inline MemberGeom member_geom(uint64_t len, uint64_t Lc, int os, int oe,
                                                  int centroid_rows = 0) {
  MemberGeom g;
  g.flip = ((oe && Lc < len) || centroid_rows) ? 1 : 0;
  g.m = int(g.flip ? Lc : len);
  g.n = int(g.flip ? len : Lc);
  g.r0 = os ? 1 : 0;
  const int W = 32 * PathTune<T>::RF;
  g.swaths = (g.n + W - 1) / W;
  g.steps = (g.m - g.r0 + 1) / 2 + 31;
  g.words = (unsigned long long)g.swaths * g.steps * 64ull;
  return g;
}

// Rows of a swath-pipeline task.  With nbands > 1 each member's rows r0 ..
// m-1 are cut into bands of an even height of at least kMinBandRows (so a
// band's steps are the whole swath's steps from (rb - r0) / 2 on); count is
// the member's number of bands, band b covers rows rb .. re-1.
constexpr int kMinBandRows = 1024;
struct Band {
  int rb, re, count;
};
__host__ __device__ inline Band member_band(const MemberGeom &g, int nbands, int b) {
  const int rows = g.m - g.r0;
  Band o;
  int h = rows;
  if (nbands > 1 && rows > 0) {
    h = (rows + nbands - 1) / nbands;
    h = (h + 1) & ~1;
    if (h < kMinBandRows) h = kMinBandRows;
  }
  o.count = (rows > 0 && h > 0) ? (rows + h - 1) / h : 1;
  o.rb = g.r0 + b * h;
  o.re = b >= o.count - 1 ? g.m : o.rb + h;
  return o;
}

// Jobs share one launch: job J owns centroid centroids[coff[J] .. + clen[J]),
// flags (bit 0 open start, bit 1 open end, bit 2 active, bit 3 centroid on
// the rows whatever the lengths -- the prefix-chop orientation) and the members
// job_mbeg[J] .. job_mend[J]-1 of the member list (member k is series
// mem_series[k] of the series table).  Members of a job are contiguous and in
// the job's order, which is the order their samples are added.
template <typename T>
struct RoundArgs {
  const T *centroids;
  const unsigned long long *coff;
  const int *clen;
  const int *jflags;
  const int *mbeg, *mend;
  int njobs;
  const T *series;
  const uint64_t *offsets;
  const uint64_t *lens;
  const int *mseries, *mjob, *order;
  int nmem;
  unsigned long long *counter;
  unsigned long long *path_off;  // word offset of member k's path
  unsigned long long *trip_off;  // triple offset of member k's path listing
  unsigned long long *rng_off;   // offset of member k's per-centroid-index ranges
  // backtrack without a path listing: per member, per row, the column
  // interval of the row's contributing cells (runs_off[k] = member k's first)
  unsigned long long *runs_off = nullptr;
  int2 *runs = nullptr;
  int *shortcut;                 // first column of the open-end shortcut, or 0
  int2 *ranges;
  T *edges;
  unsigned long long edge_stride;
  unsigned long long *words;
  // swath pipeline (many warps per member): one progress word and the right
  // edge's minimum and top-row value per (member, swath)
  unsigned long long *prog;
  T *emtop;  // per (band, member, swath)
  unsigned *err;
  int max_swaths;
  // row bands of the swath pipeline (member_band): per (member, swath) the
  // last row and edge corner of the band done so far, and that band's count
  int nbands = 1;
  T *rowbuf = nullptr;
  unsigned long long *bdone = nullptr;
  // the backtrack's row walk inside the path DTW: a member's last task to
  // finish walks its path (per member, the count of its tasks done)
  int walk_in_sweep = 0;
  unsigned long long *mdone = nullptr;
  T *means;
  uint32_t *counts;
  double *deltas;
  int32_t *triples;
  int64_t *triple_counts;
  // stripe mode with an open end: one more sample index per (member, centroid
  // index), added after its range (-1: none)
  const int *extra = nullptr;
};

template <typename T>
__device__ __forceinline__ MemberGeom geom_of(const RoundArgs<T> &a, int k, int &job) {
  job = a.mjob[k];
  const int f = a.jflags[job];
  return member_geom<T>(a.lens[a.mseries[k]], uint64_t(a.clen[job]), f & 1, (f >> 1) & 1,
                        (f >> 3) & 1);
}

// Members of inactive jobs take no path words and no ranges (a caller can run
// a large set of jobs in waves with a workspace sized for one wave); the path
// listing keeps a slot for every member so its layout does not depend on the
// flags.
template <typename T>
__global__ void __launch_bounds__(kPlanThreads) plan_kernel(RoundArgs<T> a) {
  // exclusive prefix sums over the members, kPlanThreads at a time: path
  // words, path-listing triples (every member), ranges and rows (active
  // members only)
  __shared__ unsigned long long s_warp[4][kPlanThreads / 32];
  __shared__ unsigned long long s_carry[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x < 4) s_carry[threadIdx.x] = 0;
  __syncthreads();
  for (int base = 0; base < a.nmem; base += kPlanThreads) {
    const int k = base + threadIdx.x;
    unsigned long long v[4] = {0ull, 0ull, 0ull, 0ull}, x[4];
    if (k < a.nmem) {
      int job;
      const MemberGeom g = geom_of<T>(a, k, job);
      v[1] = (unsigned long long)(g.m + g.n + 1);
      if (a.jflags[job] & 4) {
        v[0] = g.words;
        v[2] = (unsigned long long)a.clen[job];
        v[3] = (unsigned long long)g.m;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      x[q] = v[q];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x[q], off);
        if (lane >= off) x[q] += y;
      }
      if (lane == 31) s_warp[q][wid] = x[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const unsigned long long t = lane < kPlanThreads / 32 ? s_warp[q][lane] : 0ull;
        unsigned long long y = t;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const unsigned long long z = __shfl_up_sync(kFull, y, off);
          if (lane >= off) y += z;
        }
        if (lane < kPlanThreads / 32) s_warp[q][lane] = y - t;  // exclusive over warps
      }
    }
    __syncthreads();
    unsigned long long ex[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) ex[q] = s_carry[q] + s_warp[q][wid] + x[q] - v[q];
    if (k < a.nmem) {
      a.path_off[k] = ex[0];
      a.trip_off[k] = ex[1];
      a.rng_off[k] = ex[2];
      if (a.runs_off) a.runs_off[k] = ex[3];
    }
    __syncthreads();
    // the last thread's inclusive sums are the next chunk's carries
    if (threadIdx.x == kPlanThreads - 1) {
#pragma unroll
      for (int q = 0; q < 4; ++q) s_carry[q] = ex[q] + v[q];
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < a.njobs; j += kPlanThreads)
    if (a.jflags[j] & 4) a.deltas[j] = 0.0;
}

// Longest first: member k's place in the swath pipeline's task order is the
// number of members with more rows, or as many and a lower index (inactive
// members last).  The last tasks taken, and with the row walk in the sweep
// the last walks, are then the shortest.  Rows come in tiles of the block's
// size through shared memory.
template <typename T>
__global__ void __launch_bounds__(256) rank_members_kernel(RoundArgs<T> a, int *order) {
  __shared__ int s_rows[256];
  auto rows_of = [&](int i) {
    int jb;
    const MemberGeom g = geom_of<T>(a, i, jb);
    return (a.jflags[jb] & 4) ? g.m : -1;
  };
  const int k = blockIdx.x * 256 + threadIdx.x;
  const int mine = k < a.nmem ? rows_of(k) : -1;
  int rank = 0;
  for (int base = 0; base < a.nmem; base += 256) {
    const int i = base + threadIdx.x;
    s_rows[threadIdx.x] = i < a.nmem ? rows_of(i) : -1;
    __syncthreads();
    const int lim = a.nmem - base < 256 ? a.nmem - base : 256;
    for (int u = 0; u < lim; ++u) {
      const int ri = s_rows[u];
      rank += int(ri > mine) | int(ri == mine && base + u < k);
    }
    __syncthreads();
  }
  if (k < a.nmem) order[rank] = k;
}

__global__ void fill_ranges_kernel(int2 *r, unsigned long long count) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x)
    r[i] = make_int2(1, 0);
}

template <typename T, int R>
__device__ __forceinline__ void path_swath(const SwathJob<T> &job, const PathOut &po, T &emin,
                                           T &etop) {
  T col[R];
  sweep_swath_path<T, R>(job, po, col, emin, etop);
}

template <typename T, int RF, int RQ, int WARPS>
__global__ void __launch_bounds__(kRoundWarps * 32) path_dtw_kernel(RoundArgs<T> a) {
  __shared__ __align__(16) T stage_mem[WARPS * kStageElems];
  const int lane = threadIdx.x & 31;
  const long long slot = (long long)blockIdx.x * WARPS + (threadIdx.x >> 5);
  T *e0 = a.edges + slot * 2 * a.edge_stride;
  T *e1 = e0 + a.edge_stride;
  constexpr int W = 32 * RF;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= (unsigned long long)a.nmem) break;
    // longest members first when the caller's order (or member order) is by length
    const int k = a.order ? a.order[q] : a.nmem - 1 - int(q);
    int jb;
    const MemberGeom g = geom_of<T>(a, k, jb);
    const int flags = a.jflags[jb];
    if (!(flags & 4)) continue;
    const int os = flags & 1, oe = (flags >> 1) & 1;
    const T *seq = a.series + a.offsets[a.mseries[k]];
    const T *cen = a.centroids + a.coff[jb];
    SwathJob<T> job;
    job.x = g.flip ? cen : seq;
    job.y = g.flip ? seq : cen;
    job.m = g.m;
    job.n = g.n;
    job.r0 = g.r0;
    job.open_end = oe != 0;
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    int shortcut = 0;
    const bool check_short = oe && !os;
    for (int s = 0; s < g.swaths; ++s) {
      const int c0 = s * W;
      const bool last = s == g.swaths - 1;
      job.c0 = c0;
      job.edge_in = c0 ? ((s & 1) ? e0 : e1) : nullptr;
      job.edge_out = last ? nullptr : ((s & 1) ? e1 : e0);
      job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
      job.corner_init = c0 == 0 ? (job.r0 ? Num<T>::big() : T(0)) : (job.r0 ? T(0) : Num<T>::big());
      PathOut po;
      po.words = a.words + a.path_off[k] + (unsigned long long)s * g.steps * 64ull;
      po.track_min = true;
      T emin, etop;
      const int width = g.n - c0 < W ? g.n - c0 : W;
      const int rq = path_regs<T>(width);
      if (rq >= RF) {
        path_swath<T, RF>(job, po, emin, etop);
      } else {
        switch (rq / RQ) {
#define ODBA_CASE(K)                                                          \
  case K:                                                                     \
    if constexpr (K * RQ < RF) path_swath<T, K * RQ>(job, po, emin, etop);    \
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
      // The reference checks, at every swath start past the first series'
      // length, whether the top row already holds the column minimum; from
      // the first hit on, the rest of the top row is OPEN_RIGHT.
      const int cnext = c0 + W;
      if (check_short && !shortcut && !last && cnext % kRefSwath == 0 && cnext > g.m &&
          cnext < g.n && etop == emin)
        shortcut = cnext;
      __syncwarp();
    }
    if (lane == 0) a.shortcut[k] = shortcut;
  }
}

// The open-end shortcut of swath-pipeline member k (the rule of
// path_dtw_kernel, applied to the per-swath right-edge minima afterwards; a
// swath's minimum is the least of its bands', its top-row value the top
// band's, the other bands leaving theirs at big): the first qualifying
// swath boundary, or 0.
template <typename T>
__device__ __forceinline__ int member_shortcut(const RoundArgs<T> &a, int k, const MemberGeom &g,
                                               int flags) {
  const int os = flags & 1, oe = (flags >> 1) & 1;
  constexpr int W = 32 * PathTune<T>::RF;
  if (!oe || os) return 0;
  const int nb = member_band(g, a.nbands, 0).count;
  const unsigned long long layer = (unsigned long long)a.nmem * a.max_swaths;
  for (int s = 0; s + 1 < g.swaths; ++s) {
    const int cnext = (s + 1) * W;
    if (cnext % kRefSwath != 0 || cnext <= g.m || cnext >= g.n) continue;
    T emin = Num<T>::big(), etop = Num<T>::big();
    for (int b = 0; b < nb; ++b) {
      const T *et = a.emtop + ((unsigned long long)b * layer + (unsigned long long)k * a.max_swaths + s) * 2;
      emin = Num<T>::min2(emin, et[0]);
      etop = Num<T>::min2(etop, et[1]);
    }
    if (etop == emin) return cnext;
  }
  return 0;
}

template <typename T>
__device__ __forceinline__ bool walk_member_runs(const RoundArgs<T> &a, const MemberGeom &g, int k,
                                                 int os, int oe, int2 *runs);

template <typename T, int R>
__device__ __forceinline__ void path_pipe_swath(const SwathJob<T> &job, const PathOut &po,
                                                BandGate gate, TileIn<T> tile, T &emin,
                                                T &etop) {
  T col[R];
  sweep_swath_path<T, R, BandGate>(job, po, col, emin, etop, tile, gate);
}

// Path DTW as the swath pipeline: task q is band q / (nmem * max_swaths) of
// swath (q / nmem) % max_swaths of the (q % nmem)-th member in alignment
// order, so a member's swaths run on different warps at once (few or long
// members keep the GPU busy).  The right edge of swath s goes to buffer s % 2
// of the member with one progress word per (member, swath), as in the
// all-pairs swath pipeline.  With more than one band (member_band), a band
// starts from the last row and edge corner the band below left in the
// (member, swath)'s row buffer, once that band has raised the (member,
// swath)'s band word; bands only shorten the tasks, so the last wave of
// warps is shorter, and leave every recorded move as it is.  Each band also
// stores its right edge's minimum and top-row value for the open-end
// shortcut, which shortcut_kernel resolves afterwards (it never changes a
// recorded move).  Every wait is on a task taken earlier from the counter.
template <typename T, int RF, int RQ>
__global__ void __launch_bounds__(kRoundWarps * 32, sizeof(T) == 4 ? 3 : 2) path_pipe_kernel(RoundArgs<T> a) {
  __shared__ __align__(16) T stage_mem[kRoundWarps * kStageElems];
  constexpr int W = 32 * RF;
  const int lane = threadIdx.x & 31;
  const unsigned long long layer = (unsigned long long)a.nmem * a.max_swaths;
  const unsigned long long ntasks = layer * a.nbands;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= ntasks) break;
    const int b = int(q / layer);
    const unsigned long long ql = q - (unsigned long long)b * layer;
    const int s = int(ql / a.nmem), qi = int(ql - (unsigned long long)s * a.nmem);
    const int k = a.order ? a.order[qi] : a.nmem - 1 - qi;
    int jb;
    const MemberGeom g = geom_of<T>(a, k, jb);
    const int flags = a.jflags[jb];
    if (!(flags & 4) || s >= g.swaths) continue;
    const Band bd = member_band(g, a.nbands, b);
    if (b >= bd.count) continue;
    const int oe = (flags >> 1) & 1;
    const T *seq = a.series + a.offsets[a.mseries[k]];
    const T *cen = a.centroids + a.coff[jb];
    T *b0 = a.edges + (unsigned long long)k * 2 * a.edge_stride;
    T *b1 = b0 + a.edge_stride;
    const int c0 = s * W;
    const bool last = s == g.swaths - 1;
    const int base = bd.rb - g.r0;  // even: bands keep the step layout
    const unsigned long long ks = (unsigned long long)k * a.max_swaths + s;
    T *row = a.rowbuf ? a.rowbuf + ks * (W + 32) : nullptr;
    TileIn<T> tile{nullptr, g.m - 1};
    T corner = c0 == 0 ? (g.r0 ? Num<T>::big() : T(0)) : (g.r0 ? T(0) : Num<T>::big());
    if (b > 0) {
      // the band below, complete: its last row, and its left edge's value there
      if (lane == 0) wait_word_at_least(a.bdone + ks, (unsigned long long)b, a.err, kWaitLimitNs);
      __syncwarp();
      (void)ld_acquire_gpu(a.bdone + ks);
      tile.col_init = row;
      corner = s ? row[W] : Num<T>::big();
    }
    if (b + 1 < bd.count) {
      tile.row_out = row;
      tile.corner_out = row + W;
    }
    SwathJob<T> job;
    job.x = g.flip ? cen : seq;
    job.y = g.flip ? seq : cen;
    job.m = bd.re;
    job.n = g.n;
    job.c0 = c0;
    job.r0 = bd.rb;
    job.open_end = oe != 0;
    job.edge_in = s ? (((s - 1) & 1) ? b1 : b0) + base : nullptr;
    job.edge_out = last ? nullptr : ((s & 1) ? b1 : b0) + base;
    job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
    job.corner_init = corner;
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    PathOut po;
    po.words = a.words + a.path_off[k] + (unsigned long long)s * g.steps * 64ull +
               (unsigned long long)(base / 2) * 64ull;
    po.track_min = true;
    unsigned long long *words = a.prog + (unsigned long long)k * a.max_swaths;
    BandGate gate;
    gate.g.prog_in = words + (s ? s - 1 : 0);
    gate.g.prog_out = words + s;
    gate.g.err = a.err;
    gate.g.limit_ns = kWaitLimitNs;
    gate.g.avail = 0;
    gate.base = base;
    T emin, etop;
    const int width = g.n - c0 < W ? g.n - c0 : W;
    const int rq = path_regs<T>(width);
    if (rq >= RF) {
      path_pipe_swath<T, RF>(job, po, gate, tile, emin, etop);
    } else {
      switch (rq / RQ) {
#define ODBA_PPCASE(K)                                                                          \
  case K:                                                                                       \
    if constexpr (K * RQ < RF) path_pipe_swath<T, K * RQ>(job, po, gate, tile, emin, etop);     \
    break;
        ODBA_PPCASE(1)
        ODBA_PPCASE(2)
        ODBA_PPCASE(3)
        ODBA_PPCASE(4)
        ODBA_PPCASE(5)
        ODBA_PPCASE(6)
        ODBA_PPCASE(7)
#undef ODBA_PPCASE
        default:
          break;
      }
    }
    if (lane == 0) {
      T *et = a.emtop + ((unsigned long long)b * layer + ks) * 2;
      et[0] = emin;
      et[1] = etop;
    }
    if (b + 1 < bd.count) {
      // the row buffer and corner of every lane, then the band word
      __threadfence();
      __syncwarp();
      if (lane == 0) st_release_gpu(a.bdone + ks, (unsigned long long)(b + 1));
    }
    if (a.walk_in_sweep) {
      // Member k's last task to finish resolves its shortcut and walks its
      // path (pass 1 of the backtrack) while other warps sweep: every task
      // makes its moves and edge values visible before it is counted.
      __threadfence();
      __syncwarp();
      unsigned long long n = 0;
      if (lane == 0) n = atomicAdd(a.mdone + k, 1ull) + 1;
      n = __shfl_sync(kFull, n, 0);
      if (n == (unsigned long long)g.swaths * bd.count) {
        __syncwarp();
        (void)ld_acquire_gpu(a.mdone + k);  // every lane: after all the member's tasks
        if (lane == 0) a.shortcut[k] = member_shortcut<T>(a, k, g, flags);
        __syncwarp();
        walk_member_runs<T>(a, g, k, flags & 1, oe, a.runs + a.runs_off[k]);
      }
    }
  }
}

// The open-end shortcut of the swath pipeline's members (member_shortcut),
// when the row walk does not run inside the path DTW.
template <typename T>
__global__ void shortcut_kernel(RoundArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nmem) return;
  int jb;
  const MemberGeom g = geom_of<T>(a, k, jb);
  const int flags = a.jflags[jb];
  if (!(flags & 4)) return;
  a.shortcut[k] = member_shortcut<T>(a, k, g, flags);
}

// Walks member k's path from its end cell toward (0, 0) with one warp and
// calls visit(move, r, c) for every cell; the last call has NIL or
// NIL_OPEN_RIGHT.  Returns false if the walk failed.  Every lane holds the
// move word of one of the 32 rows at and below the current cell (the word of
// the lane that owned the current column in the path sweep), so the walk
// advances by shuffles and reloads only when it leaves those 32 rows or that
// owner's columns -- about once per 32 steps instead of one dependent global
// load per step.  Every lane keeps the same walk state (visitors store from
// lane 0 only).  Moves are decoded as the reference defines them: the
// open-end shortcut overrides the top row first (with a single-row matrix that
// row is row 0, dtw.hpp:105-108 runs before the row-0 loop), then row 0
// (RIGHT or OPEN_RIGHT, NIL / NIL_OPEN_RIGHT at (0, 0)), then the recorded
// code with RIGHT on the open-end top row meaning OPEN_RIGHT.
template <typename T, typename Visit>
__device__ __forceinline__ bool walk_member_path(const RoundArgs<T> &a, const MemberGeom &g, int k,
                                                 int os, int oe, Visit &&visit) {
  const int lane = threadIdx.x & 31;
  constexpr int RF = PathTune<T>::RF, W = 32 * RF;
  const unsigned long long *w = a.words + a.path_off[k];
  const int shortcut = a.shortcut[k];
  // A path has at most m + n - 1 cells and never leaves the matrix; the checks
  // only keep a corrupt path buffer from turning into an endless or
  // out-of-bounds walk.
  const long long max_cells = (long long)g.m + g.n - 1;
  long long steps = 0;
  int r = g.m - 1, c = g.n - 1;
  for (;;) {
    const int s = c / W, c0 = s * W;
    int R = RF;
    if (s == g.swaths - 1) R = path_regs<T>(g.n - c0);
    const int top = r, owner = (c - c0) / R, cbeg = c0 + owner * R;
    unsigned long long word = 0;
    const int my_row = top - lane;
    if (my_row >= 1) {
      const int rr = my_row - g.r0;
      const unsigned long long t = (unsigned long long)owner + (rr >> 1);
      word = w[(unsigned long long)s * g.steps * 64ull + (t * 32 + owner) * 2 + (rr & 1)];
    }
    for (;;) {
      const unsigned long long wv = __shfl_sync(kFull, word, (top - r) & 31);
      int mv;
      if (shortcut && r == g.m - 1 && c >= shortcut) {
        mv = kMoveOpenRight;
      } else if (r == 0) {
        mv = c == 0 ? (os ? kMoveNilOpenRight : kMaxMoveNil) : (os ? kMoveOpenRight : kMoveRight);
      } else {
        mv = decode_move(wv, c - cbeg);
        if (mv == kMoveRight && oe && r == g.m - 1) mv = kMoveOpenRight;
      }
      if (mv == kMaxMoveNil || mv == kMoveNilOpenRight) {
        visit(mv, r, c);
        return true;
      }
      if (steps >= max_cells - 1) return false;
      visit(mv, r, c);
      ++steps;
      if (mv == kMoveDiag) {
        --r;
        --c;
      } else if (mv == kMoveUp) {
        --r;
      } else {
        --c;
      }
      if (r < 0 || c < 0) return false;
      if (top - r >= 32 || c < cbeg) break;  // reload the window
    }
  }
}

// The backtrack's ranges alone (no path listing), in two passes.  Pass 1 (one
// warp per member) walks the path a row at a time: in a row the backward walk
// moves left through RIGHT cells until the first cell whose D or U bit is set,
// one count-leading-zeros on the row's step word away, and the walk stores
// the row's interval of contributing cells' columns at runs[r] ((1, 0) if
// none).  The contributing cells are those of walk_member_path with the
// backtrack's visitor: the top row's OPEN_RIGHT cells (from the open-end
// shortcut's column on, and RIGHT on the open-end top row) contribute
// nothing, so that row contributes only its last cell; row 0 is RIGHT
// (OPEN_RIGHT with open start) down to (0, 0), which contributes unless it is
// NIL_OPEN_RIGHT.  Pass 2 (runs_to_ranges_kernel) turns the intervals into
// per-centroid-index ranges in parallel.  Returns false if the walk failed.
template <typename T>
__device__ __forceinline__ bool walk_member_runs(const RoundArgs<T> &a, const MemberGeom &g, int k,
                                                 int os, int oe, int2 *runs) {
  const int lane = threadIdx.x & 31;
  constexpr int RF = PathTune<T>::RF, W = 32 * RF;
  const unsigned long long *w = a.words + a.path_off[k];
  const int shortcut = a.shortcut[k];
  const bool lead = lane == 0;
  // every window advances the walk by a row or an owner: a bound on windows
  const long long max_windows = (long long)g.m + g.n + 64;
  long long windows = 0;
  int r = g.m - 1, c = g.n - 1;
  if (shortcut && c >= shortcut) c = shortcut - 1;  // OPEN_RIGHT from the shortcut's column on
  // the column the walk entered row r at; -1 on the open-end top row, whose
  // interval is its first cell alone
  int entry = oe ? -1 : c;
  // A window: rows top .. top - 31 of one owner lane's columns cbeg .. cbeg +
  // R - 1 (swath s, owner); lane l holds row top - l's planes, word idx of
  // the member's path (step t = owner + (row - r0) / 2 of the swath: word
  // (t * 32 + owner) * 2 + (row - r0) % 2).  The windows below (same owner,
  // 32 rows = 16 steps down: idx - 1024) and to the left (owner - 1, idx -
  // 66; or the previous swath's last owner) are loaded with it, so a window
  // left through its last row or its first column is replaced without
  // waiting on memory or dividing.
  const long long swath_words = (long long)g.steps * 64;
  int s = 0, owner = 0, cbeg = 0, R = RF, top = -1;
  long long idx = 0, down_idx = 0, left_idx = 0;
  int ls = 0, lowner = 0, lcbeg = 0, lR = RF;
  unsigned long long word = 0, down_w = 0, left_w = 0;
  int j = 0;
  for (;;) {
    if (c < 0) return false;  // walked off column 0
    if (r == 0) {
      if (lead) runs[0] = os ? make_int2(1, 0) : make_int2(0, c);
      return true;
    }
    if (++windows > max_windows) return false;
    if (top >= 0 && j >= 0 && r == top - 32) {
      top -= 32;  // the window below
      word = down_w;
      idx = down_idx;
    } else if (top >= 0 && j < 0 && r > top - 32 && cbeg > 0) {
      s = ls;  // the window to the left
      owner = lowner;
      cbeg = lcbeg;
      R = lR;
      word = left_w;
      idx = left_idx;
    } else {
      s = c / W;
      const int c0 = s * W;
      R = RF;
      if (s == g.swaths - 1) R = path_regs<T>(g.n - c0);
      owner = (c - c0) / R;
      cbeg = c0 + owner * R;
      top = r;
      const int rr = top - lane - g.r0;
      idx = s * swath_words + owner * 66 + (long long)(rr >> 1) * 64 + (rr & 1);
      word = top - lane >= 1 ? w[idx] : 0ull;
    }
    down_idx = idx - 1024;
    down_w = top - 32 - lane >= 1 ? w[down_idx] : 0ull;
    if (cbeg > 0) {
      if (owner > 0) {
        ls = s;
        lowner = owner - 1;
        lcbeg = cbeg - R;
        lR = R;
        left_idx = idx - 66;
      } else {
        ls = s - 1;
        lowner = 31;
        lcbeg = cbeg - RF;
        lR = RF;
        left_idx = idx - swath_words + 31 * 66;
      }
      left_w = top - lane >= 1 ? w[left_idx] : 0ull;
    }
    const unsigned dul = unsigned(word) | unsigned(word >> 32), dl = unsigned(word);
    // j: the walk's column within the window; a row's planes are shuffled
    // one row ahead, off the chain through j
    const int lim = top - 32 > 0 ? top - 32 : 0;
    j = c - cbeg;
    int2 *rp = runs + r;
    unsigned du_r = __shfl_sync(kFull, dul, (top - r) & 31);
    unsigned d_r = __shfl_sync(kFull, dl, (top - r) & 31);
    for (;;) {
      const int ln = (top - r + 1) & 31;
      const unsigned du_n = __shfl_sync(kFull, dul, ln);
      const unsigned d_n = __shfl_sync(kFull, dl, ln);
      const unsigned x = du_r << (31 - j);  // the row's moves at or left of j, top-aligned
      if (x == 0) {
        // RIGHT through the owner's first column: on in the owner to the left
        j = -1;
        break;
      }
      const int jp = j - __clz(x);
      const int cp = cbeg + jp;
      if (lead) *rp = make_int2(cp, cp > entry ? cp : entry);
      --rp;
      --r;
      j = jp - int((d_r >> jp) & 1u);  // one column left after DIAG
      entry = cbeg + j;
      du_r = du_n;
      d_r = d_n;
      if ((r <= lim) | (j < 0)) break;  // row 0, or a new window
    }
    c = cbeg + j;
  }
}

// Pass 2, one block per member: the contributing columns of row r are the
// interval runs[r] = [x, y].  Member on the rows (centroid index t = column):
// column t's range is [lowest, highest] row holding t.  Consecutive rows'
// intervals share at most one column -- row r's first with row r - 1's last
// (an UP move) and row r's last with row r + 1's first -- so row r stores a
// column's high end unless row r + 1 also holds it and its low end unless row
// r - 1 also holds it; every other column of the interval is row r's alone.
// Centroid on the rows (t = row): the interval is the range.
template <typename T>
__global__ void runs_to_ranges_kernel(RoundArgs<T> a) {
  const int k = blockIdx.x;
  int jb;
  const MemberGeom g = geom_of<T>(a, k, jb);
  if (!(a.jflags[jb] & 4)) return;
  const int2 *runs = a.runs + a.runs_off[k];
  int2 *rg = a.ranges + a.rng_off[k];
  for (int r = threadIdx.x; r < g.m; r += blockDim.x) {
    const int2 iv = runs[r];
    if (iv.x > iv.y) continue;
    if (g.flip) {
      rg[r] = iv;
      continue;
    }
    const int2 above = r + 1 < g.m ? runs[r + 1] : make_int2(1, 0);
    const int2 below = r > 0 ? runs[r - 1] : make_int2(1, 0);
    const bool top_shared = above.x <= iv.y && iv.y <= above.y;
    const bool low_shared = below.x <= iv.x && iv.x <= below.y;
    for (int t = iv.x; t <= iv.y; ++t) {
      if (!(t == iv.y && top_shared)) rg[t].y = r;
      if (!(t == iv.x && low_shared)) rg[t].x = r;
    }
  }
}

// The backtrack (updateCentroid's loop, dba.hpp:374-423): per member the
// contiguous range of member samples each centroid index receives, and the
// path listing if asked.  One warp per member; without a listing it runs pass
// 1 of the two-pass ranges (walk_member_runs; launch_backtrack adds pass 2).
template <typename T>
__global__ void __launch_bounds__(kRoundWarps * 32) backtrack_kernel(RoundArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
  if (k >= a.nmem) return;
  int jb;
  const MemberGeom g = geom_of<T>(a, k, jb);
  const int flags = a.jflags[jb];
  if (!(flags & 4)) return;
  const int os = flags & 1, oe = (flags >> 1) & 1;
  int2 *rg = a.ranges + a.rng_off[k];
  if (!a.triples) {
    walk_member_runs<T>(a, g, k, os, oe, a.runs + a.runs_off[k]);
    return;
  }
  int32_t *tri = a.triples + 3ull * a.trip_off[k];
  const bool lead = lane == 0;
  long long nt = 0;
  int cur_t = -1, lo = 1, hi = 0;
  auto contribute = [&](int rr, int cc) {
    const int ti = g.flip ? rr : cc;  // centroid index
    const int mi = g.flip ? cc : rr;  // member sample index
    if (ti != cur_t) {
      if (lead && cur_t >= 0 && hi >= lo) rg[cur_t] = make_int2(lo, hi);
      cur_t = ti;
      lo = mi;
      hi = mi;
    } else {
      lo = mi;  // the walk only moves toward smaller indices
    }
  };
  const bool ok = walk_member_path<T>(a, g, k, os, oe, [&](int mv, int r, int c) {
    if (mv == kMaxMoveNil || mv == kMoveNilOpenRight) {
      // the start cell (dba.hpp:412-415)
      if (mv != kMoveNilOpenRight) contribute(0, 0);
      if (lead && cur_t >= 0 && hi >= lo) rg[cur_t] = make_int2(lo, hi);
    } else if (mv != kMoveOpenRight) {
      contribute(r, c);
    }
    if (lead && tri) {
      tri[3 * nt] = r;
      tri[3 * nt + 1] = c;
      tri[3 * nt + 2] = mv;
    }
    ++nt;
  });
  if (lead && a.triple_counts) a.triple_counts[k] = ok ? nt : -1;
}

// Prefix chop (chopPrefixFromSequences' host walk, dba.hpp:1313-1336), on
// each series' open-end path against the leader (leader on the rows): skip
// the OPEN_RIGHT run along the top row from the end cell; the column reached
// is the chop position; then count, per leader row, the path cells from there
// to (0, 0) (the cell reached counts 1 on the top row).  One warp per series;
// rows are visited in one run each, so each count is stored once.
template <typename T>
__global__ void __launch_bounds__(kRoundWarps * 32) chop_walk_kernel(RoundArgs<T> a, long long *chop,
                                                                    int *hist, int P) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
  if (k >= a.nmem) return;
  int jb;
  const MemberGeom g = geom_of<T>(a, k, jb);
  const int flags = a.jflags[jb];
  if (!(flags & 4)) return;
  const bool lead = lane == 0;
  int *h = hist + (unsigned long long)k * P;
  bool skipping = true;
  long long pos = -1;
  int row = -1, count = 0;
  const bool ok = walk_member_path<T>(a, g, k, flags & 1, (flags >> 1) & 1, [&](int mv, int r, int c) {
    if (skipping) {
      if (mv == kMoveOpenRight) return;
      skipping = false;
      pos = c;
      row = r;
      count = 1;
      return;
    }
    if (r == row) {
      ++count;
    } else {
      if (lead) h[row] = count;
      row = r;
      count = 1;
    }
  });
  if (lead) {
    if (ok && row >= 0) h[row] = count;
    chop[k] = ok ? pos : -1;
  }
}

// The reference divides on the host (dba.hpp:820-822); a centroid index that
// received no sample gives 0/0, which x86 answers with its default NaN (sign
// bit set, printed "-nan").  The device's 0/0 NaN differs, so it is replaced.
template <typename T>
__device__ __forceinline__ T host_default_nan();
template <>
__device__ __forceinline__ float host_default_nan<float>() { return __int_as_float(0xffc00000); }
template <>
__device__ __forceinline__ double host_default_nan<double>() {
  return __longlong_as_double((long long)0xfff8000000000000ull);
}

template <typename T>
__device__ __forceinline__ T div_rn(T a, T b);
template <>
__device__ __forceinline__ float div_rn<float>(float a, float b) { return __fdiv_rn(a, b); }
template <>
__device__ __forceinline__ double div_rn<double>(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// grid: (ceil(max centroid length / 256), jobs)
template <typename T>
__global__ void __launch_bounds__(kReduceThreads) reduce_kernel(RoundArgs<T> a) {
  // One warp per centroid index: the index's sum is a chain of additions in
  // the reference's order (members in order, each member's samples from the
  // highest down, the stripe-mode extra sample last), so the warp's lanes
  // load the samples of consecutive members at once (lane l the l-th group
  // of kMpl members of a chunk) and lay them out in that order in the warp's
  // shared-memory buffer; lane 0 then adds the buffer.  Many warps per SM
  // keep the loads and the chains of different indices in flight together.
  constexpr int kCap = 8192 / int(sizeof(T));  // samples per warp's buffer
  constexpr int kMpl = 8;                      // members per lane per chunk
  __shared__ T s_buf[kReduceWarps][kCap];
  __shared__ double s_max[kReduceWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int jb = blockIdx.y;
  const int t = blockIdx.x * kReduceWarps + wid;
  const int Lc = a.clen[jb];
  const bool live = (a.jflags[jb] & 4) != 0;
  double dl = 0.0;
  if (live && t < Lc) {
    T sum = T(0);
    uint32_t cnt = 0;
    T *buf = s_buf[wid];
    const int kb = a.mbeg[jb], ke = a.mend[jb];
    for (int k0 = kb; k0 < ke; k0 += 32 * kMpl) {
      int2 r[kMpl];
      int e[kMpl];
      const T *sq[kMpl];
      int n_l = 0;
#pragma unroll
      for (int u = 0; u < kMpl; ++u) {
        const int m = k0 + lane * kMpl + u;
        r[u] = make_int2(1, 0);
        e[u] = -1;
        sq[u] = a.series;
        if (m < ke) {
          const unsigned long long ro = a.rng_off[m];
          r[u] = a.ranges[ro + t];
          sq[u] = a.series + a.offsets[a.mseries[m]];
          if (a.extra) e[u] = a.extra[ro + t];
        }
        if (r[u].y >= r[u].x) n_l += r[u].y - r[u].x + 1 + (e[u] >= 0 ? 1 : 0);
      }
      int incl = n_l;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, off);
        if (lane >= off) incl += y;
      }
      const int total = __shfl_sync(kFull, incl, 31);
      cnt += uint32_t(total);
      if (total <= kCap) {
        int p = incl - n_l;
#pragma unroll
        for (int u = 0; u < kMpl; ++u) {
          if (r[u].y < r[u].x) continue;
          for (int i = r[u].y; i >= r[u].x; --i) buf[p++] = __ldg(sq[u] + i);
          if (e[u] >= 0) buf[p++] = __ldg(sq[u] + e[u]);
        }
        __syncwarp();
        if (lane == 0)
          for (int q = 0; q < total; ++q) sum = add_rn(sum, buf[q]);
        __syncwarp();
      } else {
        // more samples than the buffer holds: the lanes add theirs in turn,
        // each starting from the previous lane's sum
        for (int L = 0; L < 32; ++L) {
          if (lane == L) {
#pragma unroll
            for (int u = 0; u < kMpl; ++u) {
              if (r[u].y < r[u].x) continue;
              for (int i = r[u].y; i >= r[u].x; --i) sum = add_rn(sum, sq[u][i]);
              if (e[u] >= 0) sum = add_rn(sum, sq[u][e[u]]);
            }
          }
          sum = __shfl_sync(kFull, sum, L);
        }
      }
    }
    if (lane == 0) {
      const T mean = cnt ? div_rn<T>(sum, T(cnt)) : host_default_nan<T>();
      a.means[a.coff[jb] + t] = mean;
      a.counts[a.coff[jb] + t] = cnt;
      const double d = fabs(double(a.centroids[a.coff[jb] + t] - mean));
      dl = d > 0.0 ? d : 0.0;  // NaN never raises the maximum (dba.hpp:833)
    }
  }
  if (lane == 0) s_max[wid] = dl;
  __syncthreads();
  if (threadIdx.x == 0 && live) {
    double m = s_max[0];
    for (int q = 1; q < kReduceWarps; ++q) m = s_max[q] > m ? s_max[q] : m;
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(a.deltas + jb), (unsigned long long)__double_as_longlong(m));
  }
}

// One job, members 0..n-1 in order (the single-cluster DBAUpdate call).
__global__ void single_job_kernel(int *mseries, int *mjob, int n, int *clen, int Lc, int *jflags,
                                  int flags, int *mbeg, int *mend, unsigned long long *coff) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    mseries[k] = k;
    mjob[k] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    clen[0] = Lc;
    jflags[0] = flags;
    mbeg[0] = 0;
    mend[0] = n;
    coff[0] = 0;
  }
}

template <typename T>
int round_grid() {
  static std::atomic<int> cached[64];  // per device; host threads may race (same value)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64) {
    const int c = cached[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ, kRoundWarps>, kRoundWarps * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int g = sms * per_sm;
  if (dev >= 0 && dev < 64) cached[dev].store(g, std::memory_order_relaxed);
  return g;
}

struct RoundLayout {
  size_t off_counter, off_path, off_trip, off_rng, off_runoff, off_short, off_single, off_ranges,
      off_runs, off_edges, off_words, off_prog, off_bdone, off_mdone, off_order, off_emtop,
      off_rowbuf, total;
  unsigned long long edge_stride;
  int max_swaths;
  int nbands;  // row bands of the swath pipeline
  bool pipe;   // path DTW as the swath pipeline (two edge columns per member)
};

constexpr size_t kPipeEdgeBytes = size_t(8) << 30;  // per-member edge columns up to 8 GB
constexpr int kMaxBands = 8;
constexpr size_t kMaxRowBufBytes = size_t(256) << 20;
std::atomic<int> g_round_bands{0};  // odba_round_set_bands (0: chosen per launch)

// Row bands of the swath pipeline for `tasks` (member, swath) tasks on
// `slots` resident warps: two when the tasks make more than one wave and at
// most four, one otherwise.  Tasks that fit one wave run at once, and bands
// would only lengthen each (member, swath)'s chain.  Past one wave, halving
// the tasks halves the last partial wave; more bands cost more than they
// save, because a band taken from the counter before the band below it is
// done holds its warp while it waits (400 members x 6 swaths on 1776 warps:
// path DTW 7.02 ms with one band, 6.84 with two, 7.56 with three, 8.97 with
// four; 800 members: 11.42, 10.97 and 11.71 ms).
int pipe_bands(unsigned long long tasks, size_t slots) {
  const int forced = g_round_bands.load(std::memory_order_relaxed);
  if (forced > 0) return forced < kMaxBands ? forced : kMaxBands;
  return (tasks > slots && tasks <= 4ull * slots) ? 2 : 1;
}

// Workspace layout for nmem members / njobs jobs with the given totals.
template <typename T>
RoundLayout round_layout(int nmem, int njobs, unsigned long long words,
                         unsigned long long ranges, unsigned long long maxm, int max_swaths = 0,
                         unsigned long long rows = 0, unsigned long long tasks = 0) {
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  RoundLayout L;
  L.edge_stride = (maxm + 32 + 31) / 32 * 32;
  const size_t slots = size_t(round_grid<T>()) * kRoundWarps;
  L.max_swaths = max_swaths;
  L.pipe = max_swaths > 0 && size_t(nmem) * 2 * L.edge_stride * sizeof(T) <= kPipeEdgeBytes;
  const size_t edge_cols = L.pipe ? size_t(nmem) : slots;
  size_t o = 0;
  L.off_counter = o; o += 256;
  L.off_path = o; o += up(size_t(nmem) * 8);
  L.off_trip = o; o += up(size_t(nmem) * 8);
  L.off_rng = o; o += up(size_t(nmem) * 8);
  L.off_runoff = o; o += up(size_t(nmem) * 8);
  L.off_short = o; o += up(size_t(nmem) * 4);
  // single-job descriptors: mseries, mjob (nmem ints each), clen, jflags, mbeg, mend, coff
  L.off_single = o; o += up(size_t(nmem) * 8 + 64);
  L.off_ranges = o; o += up(size_t(ranges) * sizeof(int2));
  L.off_runs = o; o += up(size_t(rows) * sizeof(int2));  // cleared with the ranges
  L.off_edges = o; o += up(edge_cols * 2 * L.edge_stride * sizeof(T));
  L.off_words = o; o += up(words * 8);
  const size_t ps = L.pipe ? size_t(nmem) * size_t(max_swaths) : 0;
  L.nbands = L.pipe ? pipe_bands(tasks, slots) : 1;
  // row buffers for at most kMaxRowBufBytes (many inactive members: no bands)
  if (L.nbands > 1 && ps * (32 * PathTune<T>::RF + 32) * sizeof(T) > kMaxRowBufBytes) L.nbands = 1;
  L.off_prog = o; o += up(ps * 8);
  L.off_bdone = o; o += up(ps * 8);  // cleared with the progress words
  L.off_mdone = o; o += L.pipe ? up(size_t(nmem) * 8) : 0;  // likewise
  L.off_order = o; o += L.pipe ? up(size_t(nmem) * 4) : 0;
  L.off_emtop = o; o += up(ps * L.nbands * 2 * sizeof(T));
  L.off_rowbuf = o; o += L.nbands > 1 ? up(ps * (32 * PathTune<T>::RF + 32) * sizeof(T)) : 0;
  L.total = o;
  (void)njobs;
  return L;
}

template <typename T>
void host_totals(const uint64_t *h_lens, const int *h_mjob, int nmem, const uint64_t *h_clen,
                 const int *h_flags, unsigned long long &words, unsigned long long &ranges,
                 unsigned long long &maxm, int *max_swaths = nullptr,
                 unsigned long long *rows = nullptr, unsigned long long *tasks = nullptr) {
  words = ranges = 0;
  maxm = 1;
  if (max_swaths) *max_swaths = 1;
  if (rows) *rows = 0;
  if (tasks) *tasks = 0;
  for (int k = 0; k < nmem; ++k) {
    const int j = h_mjob ? h_mjob[k] : 0;
    const int f = h_flags[j];
    if (!(f & 4)) continue;
    const MemberGeom g = member_geom<T>(h_lens[k], h_clen[j], f & 1, (f >> 1) & 1, (f >> 3) & 1);
    words += g.words;
    ranges += h_clen[j];
    if ((unsigned long long)g.m > maxm) maxm = g.m;
    if (max_swaths && g.swaths > *max_swaths) *max_swaths = g.swaths;
    if (rows) *rows += (unsigned long long)g.m;
    if (tasks) *tasks += (unsigned long long)g.swaths;
  }
}

// Planning, range clearing and the path DTW of a round (everything before
// the backtrack).
template <typename T>
void launch_paths(RoundArgs<T> &a, const RoundLayout &L, char *base, cudaStream_t stream,
                  bool walk_runs = false) {
  a.counter = reinterpret_cast<unsigned long long *>(base + L.off_counter);
  a.path_off = reinterpret_cast<unsigned long long *>(base + L.off_path);
  a.trip_off = reinterpret_cast<unsigned long long *>(base + L.off_trip);
  a.rng_off = reinterpret_cast<unsigned long long *>(base + L.off_rng);
  a.runs_off = reinterpret_cast<unsigned long long *>(base + L.off_runoff);
  a.shortcut = reinterpret_cast<int *>(base + L.off_short);
  a.ranges = reinterpret_cast<int2 *>(base + L.off_ranges);
  a.runs = reinterpret_cast<int2 *>(base + L.off_runs);
  a.edges = reinterpret_cast<T *>(base + L.off_edges);
  a.edge_stride = L.edge_stride;
  a.words = reinterpret_cast<unsigned long long *>(base + L.off_words);
  a.prog = reinterpret_cast<unsigned long long *>(base + L.off_prog);
  a.emtop = reinterpret_cast<T *>(base + L.off_emtop);
  a.bdone = reinterpret_cast<unsigned long long *>(base + L.off_bdone);
  a.rowbuf = L.nbands > 1 ? reinterpret_cast<T *>(base + L.off_rowbuf) : nullptr;
  a.nbands = L.nbands;
  a.mdone = reinterpret_cast<unsigned long long *>(base + L.off_mdone);
  a.walk_in_sweep = (L.pipe && walk_runs) ? 1 : 0;
  a.err = reinterpret_cast<unsigned *>(base + L.off_counter + 8);
  a.max_swaths = L.max_swaths;
  const unsigned long long nr = (L.off_edges - L.off_ranges) / sizeof(int2);
  cudaMemsetAsync(a.counter, 0, 16, stream);  // work counter and error word
  plan_kernel<T><<<1, kPlanThreads, 0, stream>>>(a);
  fill_ranges_kernel<<<int(nr / 256 + 1 < 4096 ? nr / 256 + 1 : 4096), 256, 0, stream>>>(a.ranges, nr);
  // with fewer members than resident warps, one block per member spreads
  // them over the SMs instead of leaving them to the first blocks placed
  const bool spread = a.nmem < round_grid<T>() * kRoundWarps;
  if (L.pipe) {
    cudaMemsetAsync(a.prog, 0, L.off_order - L.off_prog, stream);  // progress, band, member words
    if (!a.order && a.nmem <= kRankMembers) {
      int *ord = reinterpret_cast<int *>(base + L.off_order);
      rank_members_kernel<T><<<(a.nmem + 255) / 256, 256, 0, stream>>>(a, ord);
      a.order = ord;
    }
    path_pipe_kernel<T, PathTune<T>::RF, PathTune<T>::RQ>
        <<<round_grid<T>(), kRoundWarps * 32, 0, stream>>>(a);
    if (!a.walk_in_sweep) shortcut_kernel<T><<<(a.nmem + 127) / 128, 128, 0, stream>>>(a);
  } else if (spread)
    path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ, 1><<<a.nmem, 32, 0, stream>>>(a);
  else
    path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ, kRoundWarps>
        <<<round_grid<T>(), kRoundWarps * 32, 0, stream>>>(a);
}

// The backtrack: with a path listing one kernel walking cell by cell; without,
// the row walk (pass 1, inside the swath pipeline's path DTW when it ran
// there) and the parallel conversion of its row intervals into ranges
// (pass 2).
template <typename T>
void launch_backtrack(const RoundArgs<T> &a, cudaStream_t stream) {
  if (!a.walk_in_sweep)
    backtrack_kernel<T><<<(a.nmem + kRoundWarps - 1) / kRoundWarps, kRoundWarps * 32, 0, stream>>>(a);
  if (!a.triples) runs_to_ranges_kernel<T><<<a.nmem, 256, 0, stream>>>(a);
}

template <typename T>
int launch_round(RoundArgs<T> &a, const RoundLayout &L, char *base, int max_clen,
                 cudaStream_t stream) {
  launch_paths<T>(a, L, base, stream, !a.triples);
  launch_backtrack<T>(a, stream);
  dim3 rg((max_clen + kReduceWarps - 1) / kReduceWarps, a.njobs);
  reduce_kernel<T><<<rg, kReduceThreads, 0, stream>>>(a);
  return check_launch("DBA round kernels");
}

}  // namespace

int dba_round_bands(int n) { return g_round_bands.exchange(n); }

template <typename T>
size_t dba_round_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = Lc;
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  int ms = 1;
  unsigned long long rows = 0, tasks = 0;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm, &ms, &rows, &tasks);
  if (Lc > maxm) maxm = Lc;
  return round_layout<T>(n, 1, words, ranges, maxm, ms, rows, tasks).total;
}

namespace {

// The descriptors of a one-job round (members 0..n-1 in order, all active)
// in the workspace, and round arguments pointing at them; outputs unset.
template <typename T>
RoundArgs<T> single_job_round(const T *centroid, uint64_t Lc, const T *series,
                              const uint64_t *offsets, const uint64_t *lens, int n, int flags,
                              const RoundLayout &L, char *base, cudaStream_t stream) {
  int *single = reinterpret_cast<int *>(base + L.off_single);
  int *mseries = single, *mjob = single + n, *d_clen = single + 2 * n, *d_flags = single + 2 * n + 1,
      *d_mbeg = single + 2 * n + 2, *d_mend = single + 2 * n + 3;
  unsigned long long *d_coff =
      reinterpret_cast<unsigned long long *>(base + L.off_single + ((size_t(2 * n + 4) * 4 + 7) / 8) * 8);
  single_job_kernel<<<(n + 255) / 256, 256, 0, stream>>>(mseries, mjob, n, d_clen, int(Lc), d_flags,
                                                        flags, d_mbeg, d_mend, d_coff);
  RoundArgs<T> a;
  a.centroids = centroid;
  a.coff = d_coff;
  a.clen = d_clen;
  a.jflags = d_flags;
  a.mbeg = d_mbeg;
  a.mend = d_mend;
  a.njobs = 1;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.mseries = mseries;
  a.mjob = mjob;
  a.order = nullptr;
  a.nmem = n;
  a.means = nullptr;
  a.counts = nullptr;
  a.deltas = nullptr;
  a.triples = nullptr;
  a.triple_counts = nullptr;
  return a;
}

template <typename T>
RoundLayout single_job_layout(const uint64_t *h_lens, int n, uint64_t Lc, int flags) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = Lc;
  int ms = 1;
  unsigned long long rows = 0, tasks = 0;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm, &ms, &rows, &tasks);
  if (Lc > maxm) maxm = Lc;
  return round_layout<T>(n, 1, words, ranges, maxm, ms, rows, tasks);
}

}  // namespace

template <typename T>
int dba_round_launch(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                     const uint64_t *lens, const uint64_t *h_lens, int n, int os, int oe, T *mean,
                     uint32_t *counts, double *delta, int32_t *triples, int64_t *triple_counts,
                     void *ws, size_t ws_bytes, cudaStream_t stream) {
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  const RoundLayout L = single_job_layout<T>(h_lens, n, Lc, flags);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "DBA round workspace too small");
  char *base = static_cast<char *>(ws);
  RoundArgs<T> a = single_job_round<T>(centroid, Lc, series, offsets, lens, n, flags, L, base, stream);
  a.means = mean;
  a.counts = counts;
  a.deltas = delta;
  a.triples = triples;
  a.triple_counts = triple_counts;
  return launch_round<T>(a, L, base, int(Lc), stream);
}

// The first half of a round for a share of the members (a multi-GPU round
// deals members to ranks): path DTW and backtrack, then every member's
// per-centroid-index sample ranges copied to ranges_out (member k's at
// k * Lc; (1, 0) where a centroid index receives nothing).  Same workspace as
// dba_round_launch.
template <typename T>
int dba_round_ranges_launch(const T *centroid, uint64_t Lc, const T *series,
                            const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                            int n, int os, int oe, int2 *ranges_out, void *ws, size_t ws_bytes,
                            cudaStream_t stream) {
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  const RoundLayout L = single_job_layout<T>(h_lens, n, Lc, flags);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "DBA round workspace too small");
  char *base = static_cast<char *>(ws);
  RoundArgs<T> a = single_job_round<T>(centroid, Lc, series, offsets, lens, n, flags, L, base, stream);
  // the plan clears the job's delta: point it at a spare word of the header
  a.deltas = reinterpret_cast<double *>(base + L.off_counter + 16);
  launch_paths<T>(a, L, base, stream, true);
  launch_backtrack<T>(a, stream);
  cudaMemcpyAsync(ranges_out, a.ranges, size_t(n) * Lc * sizeof(int2), cudaMemcpyDeviceToDevice, stream);
  return check_launch("DBA round path and backtrack kernels");
}

template <typename T>
size_t dba_reduce_workspace_bytes(int n) {
  return round_layout<T>(n, 1, 0, 0, 1, 0).total;
}

// The second half: the ordered reducer over all n members' sample ranges
// (from dba_round_ranges_launch, members in the round's order), giving the
// new centroid, the pile-up counts and the delta exactly as the whole round
// does.
template <typename T>
int dba_reduce_ranges_launch(const T *centroid, uint64_t Lc, const T *series,
                             const uint64_t *offsets, const uint64_t *lens, int n, int os, int oe,
                             const int2 *ranges, T *mean, uint32_t *counts, double *delta, void *ws,
                             size_t ws_bytes, cudaStream_t stream) {
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  const RoundLayout L = round_layout<T>(n, 1, 0, 0, 1, 0);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "reducer workspace too small");
  char *base = static_cast<char *>(ws);
  RoundArgs<T> a = single_job_round<T>(centroid, Lc, series, offsets, lens, n, flags, L, base, stream);
  a.path_off = reinterpret_cast<unsigned long long *>(base + L.off_path);
  a.trip_off = reinterpret_cast<unsigned long long *>(base + L.off_trip);
  a.rng_off = reinterpret_cast<unsigned long long *>(base + L.off_rng);
  a.ranges = const_cast<int2 *>(ranges);
  a.means = mean;
  a.counts = counts;
  a.deltas = delta;
  plan_kernel<T><<<1, kPlanThreads, 0, stream>>>(a);
  reduce_kernel<T><<<dim3(unsigned((Lc + kReduceWarps - 1) / kReduceWarps), 1), kReduceThreads, 0, stream>>>(a);
  return check_launch("DBA reducer kernels");
}

template <typename T>
size_t dba_batch_workspace_bytes(const uint64_t *h_mlens, const int *h_mjob, int nmem,
                                 const uint64_t *h_clen, const int *h_flags, int njobs) {
  unsigned long long words, ranges, maxm;
  int ms = 1;
  unsigned long long rows = 0, tasks = 0;
  host_totals<T>(h_mlens, h_mjob, nmem, h_clen, h_flags, words, ranges, maxm, &ms, &rows, &tasks);
  for (int j = 0; j < njobs; ++j)
    if (h_clen[j] > maxm) maxm = h_clen[j];
  return round_layout<T>(nmem, njobs, words, ranges, maxm, ms, rows, tasks).total;
}

template <typename T>
int dba_batch_launch(const T *centroids, const unsigned long long *coff, const int *clen,
                     const int *jflags, const int *mbeg, const int *mend, int njobs, int max_clen,
                     const T *series, const uint64_t *offsets, const uint64_t *lens,
                     const int *mseries, const int *mjob, const int *order, int nmem,
                     const uint64_t *h_mlens, const int *h_mjob, const uint64_t *h_clen,
                     const int *h_flags, T *means, uint32_t *counts, double *deltas,
                     int32_t *triples, int64_t *triple_counts, void *ws, size_t ws_bytes,
                     cudaStream_t stream) {
  unsigned long long words, ranges, maxm;
  int ms = 1;
  unsigned long long rows = 0, tasks = 0;
  host_totals<T>(h_mlens, h_mjob, nmem, h_clen, h_flags, words, ranges, maxm, &ms, &rows, &tasks);
  for (int j = 0; j < njobs; ++j)
    if (h_clen[j] > maxm) maxm = h_clen[j];
  const RoundLayout L = round_layout<T>(nmem, njobs, words, ranges, maxm, ms, rows, tasks);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "DBA batch workspace too small");
  RoundArgs<T> a;
  a.centroids = centroids;
  a.coff = coff;
  a.clen = clen;
  a.jflags = jflags;
  a.mbeg = mbeg;
  a.mend = mend;
  a.njobs = njobs;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.mseries = mseries;
  a.mjob = mjob;
  a.order = order;
  a.nmem = nmem;
  a.means = means;
  a.counts = counts;
  a.deltas = deltas;
  a.triples = triples;
  a.triple_counts = triple_counts;
  return launch_round<T>(a, L, static_cast<char *>(ws), max_clen, stream);
}

// ---------------------------------------------------------------------------
// Stripe mode: one DBA round for members whose 2-bit path does not fit in
// memory (the reference's stripe mode, dba.hpp:515-763).  Per member, in the
// orientation of the full-path round (centroid on the rows when an open end
// flips the member, dba.hpp:497-501):
//   1. forward: the swath pipeline (many warps, bounded hand-off waits) over
//      the member's swaths; every swath's right edge is kept (E, one column of
//      rows per swath) and every K-th cost row is kept across all columns (Q);
//   2. backtrack, reference stripe by reference stripe (1024 columns) from the
//      right: every K-row tile of the stripe's swaths below the current
//      backtrack height H is recomputed with its moves in parallel (one warp
//      per tile: its row below comes from Q, its left edge from E), then one
//      warp continues the walk through the stripe and records the
//      per-centroid-index sample ranges (and the path listing);
//   3. the ordered reducer of the full-path round.
// The reference re-runs each stripe with the first sequence's length set to H
// (dba.hpp:700-721), so with an open end its top-row rule acts on row H-1 and
// its shortcut (dtw.hpp:74-129, open end only) is checked on the stored left
// edge's rows below H whenever the stripe starts past column H: if it fires,
// the stripe's row H-1 is all OPEN_RIGHT.  Stripes from the first one whose
// shortcut fired in the forward pass on take that branch too (the reference's
// forward pass stopped there and left those edges unwritten).  The recompute
// here does the same: rows below H-1 are the forward pass's, row H-1 follows
// the open-end rules (for double, whose swaths are 512 wide, the second half
// of a stripe continues the first half's recomputed top row).  Without an open
// end the round equals the full-path round bit for bit.
namespace {

struct StripeWalk {
  int r, c, h, cur_t, lo, hi, state;  // state: 0 walking, 1 done, 2 failed
  int s_fwd;                          // first stripe whose forward shortcut fired, or INT_MAX
  long long nt;
};

template <typename T>
struct StripeArgs {
  const T *series;
  const uint64_t *offsets;
  int member;                   // series + offsets[member]
  const T *centroid;
  int flip;                     // centroid on the rows
  int m, n, r0, oe, swaths, shift;  // tile height K = 1 << shift
  T *E;
  unsigned long long e_stride;
  T *Q;
  unsigned long long q_stride;
  unsigned long long *prog;     // one progress word per swath
  unsigned *err;
  unsigned long long *counter;
  unsigned long long *words;    // move words of one swath, full-path layout (two buffers
  unsigned long long words_stride;  // words_stride apart when a stripe has two swaths)
  StripeWalk *walk;
  int2 *ranges;                 // this member's ranges (one per centroid index)
  int *extra;                   // this member's extra samples, or null
  unsigned long long *fmin;     // per stripe: forward shortcut minimum (value bits)
  unsigned long long *cmin;     // per stripe: shortcut minimum below H (value bits)
  T *top_carry;                 // recomputed top row at the first half's right edge
  int32_t *triples;             // this member's path listing, or null
  int64_t *triple_count;        // or null
  unsigned long long limit_ns;
};

template <typename T>
__device__ __forceinline__ const T *stripe_member_ptr(const StripeArgs<T> &a) {
  return a.series + a.offsets[a.member];
}
template <typename T>
__device__ __forceinline__ const T *stripe_rows_ptr(const StripeArgs<T> &a) {
  return a.flip ? a.centroid : stripe_member_ptr(a);
}
template <typename T>
__device__ __forceinline__ const T *stripe_cols_ptr(const StripeArgs<T> &a) {
  return a.flip ? stripe_member_ptr(a) : a.centroid;
}

// Non-negative costs order like their bit patterns (float zero-extended).
__device__ __forceinline__ unsigned long long cost_bits(float v) { return __float_as_uint(v); }
__device__ __forceinline__ unsigned long long cost_bits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

// Registers per lane of swath s (the last, partial swath is narrower).
template <typename T>
__host__ __device__ inline int stripe_regs(int n, int s) {
  constexpr int RF = PathTune<T>::RF, RQ = PathTune<T>::RQ, W = 32 * RF;
  const int c0 = s * W;
  const int width = n - c0 < W ? n - c0 : W;
  const int rq = ((width + 31) / 32 + RQ - 1) / RQ * RQ;
  return rq < RF ? rq : RF;
}

template <typename T>
__device__ __forceinline__ T stripe_corner(int c0, int r0) {
  return c0 == 0 ? (r0 ? Num<T>::big() : T(0)) : (r0 ? T(0) : Num<T>::big());
}

// The stored right edge of the swath ending at column c - 1 (c a multiple of
// the swath width, 0 < c < n).
template <typename T>
__device__ __forceinline__ const T *stripe_edge_before(const StripeArgs<T> &a, int c) {
  constexpr int W = 32 * PathTune<T>::RF;
  return a.E + (unsigned long long)(c / W - 1) * a.e_stride;
}

// Whether the reference's re-run of stripe t at height H takes its shortcut
// branch (the whole of row H-1 OPEN_RIGHT).
template <typename T>
__device__ __forceinline__ bool stripe_fires(const StripeArgs<T> &a, int t, int H,
                                             const StripeWalk &w) {
  if (!a.oe || a.r0) return false;
  const long long L = (long long)t * kRefSwath;
  if (L <= H) return false;
  if (t >= w.s_fwd) return true;
  return cost_bits(stripe_edge_before(a, int(L))[H - 1]) == a.cmin[t];
}

template <typename T, int R>
__device__ __forceinline__ void stripe_fwd_swath(const SwathJob<T> &job, const PipeGate &gate,
                                                 const CkptOut<T> &ck) {
  T col[R];
  sweep_swath<T, R, PipeGate, true, false>(job, col, gate, ck);
}

// OE: open end; FLIP: centroid on the rows (compile-time switches, so that
// one of the two series pointers stays a kernel parameter and the sweep keeps
// its registers)
template <typename T, int RF, int RQ, bool OE, bool FLIP>
__global__ void __launch_bounds__(kRoundWarps * 32) stripe_forward_kernel(StripeArgs<T> a) {
  __shared__ __align__(16) T stage_mem[kRoundWarps * kStageElems];
  constexpr int W = 32 * RF;
  const int lane = threadIdx.x & 31;
  const T *x = FLIP ? a.centroid : stripe_member_ptr(a);
  const T *y = FLIP ? stripe_member_ptr(a) : a.centroid;
  for (;;) {
    unsigned long long q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1ull);
    q = __shfl_sync(kFull, q, 0);
    if (q >= (unsigned long long)a.swaths) break;
    const int sw = int(q), c0 = sw * W;
    SwathJob<T> job;
    job.x = x;
    job.y = y;
    job.m = a.m;
    job.n = a.n;
    job.c0 = c0;
    job.r0 = a.r0;
    job.edge_in = sw ? a.E + (unsigned long long)(sw - 1) * a.e_stride : nullptr;
    job.edge_out = sw + 1 < a.swaths ? a.E + (unsigned long long)sw * a.e_stride : nullptr;
    job.open_end = OE;
    job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
    job.corner_init = stripe_corner<T>(c0, a.r0);
    job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
    PipeGate gate;
    gate.prog_in = a.prog + (sw ? sw - 1 : 0);
    gate.prog_out = a.prog + sw;
    gate.err = a.err;
    gate.limit_ns = a.limit_ns;
    gate.avail = 0;
    const CkptOut<T> ck{a.Q + c0, a.q_stride, a.shift};
    const int R = stripe_regs<T>(a.n, sw);
    if (R == RF) {
      stripe_fwd_swath<T, RF>(job, gate, ck);
    } else {
      switch (R / RQ) {
#define ODBA_SCASE(K)                                                         \
  case K:                                                                     \
    if constexpr (K * RQ < RF) stripe_fwd_swath<T, K * RQ>(job, gate, ck);    \
    break;
        ODBA_SCASE(1)
        ODBA_SCASE(2)
        ODBA_SCASE(3)
        ODBA_SCASE(4)
        ODBA_SCASE(5)
        ODBA_SCASE(6)
        ODBA_SCASE(7)
#undef ODBA_SCASE
        default:
          break;
      }
    }
  }
}

// Shortcut minimum of the stored edge before stripe t over rows [0, H)
// (ShortcutRows), reduced into slot[t].  Forward pass (fwd): every stripe t
// in [tlo, thi] (stripes past the last row), H = m.  Backtrack: the one
// stripe tlo, H the walk's height, skipped where the stripe's branch is
// already decided.
template <typename T>
__global__ void stripe_min_kernel(StripeArgs<T> a, int tlo, int thi, int fwd) {
  __shared__ unsigned long long smin[256];
  const StripeWalk *wp = a.walk;
  int H = a.m;
  if (!fwd) {
    if (wp->state != 0) return;
    H = wp->h;
    if ((long long)tlo * kRefSwath <= H || tlo >= wp->s_fwd) return;
  }
  unsigned long long *slot = fwd ? a.fmin : a.cmin;
  for (int t = tlo + int(blockIdx.y); t <= thi; t += int(gridDim.y)) {
    const T *e = stripe_edge_before(a, t * kRefSwath);
    unsigned long long best = ~0ull;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < H;
         r += (long long)gridDim.x * blockDim.x) {
      if (!shortcut_row<T>(int(r))) continue;
      const unsigned long long b = cost_bits(e[r]);
      best = b < best ? b : best;
    }
    smin[threadIdx.x] = best;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s && smin[threadIdx.x + s] < smin[threadIdx.x])
        smin[threadIdx.x] = smin[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0 && smin[0] != ~0ull) atomicMin(slot + t, smin[0]);
    __syncthreads();
  }
}

// The first stripe in [tlo, thi] whose forward shortcut fires (one warp).
template <typename T>
__global__ void stripe_sfwd_kernel(StripeArgs<T> a, int tlo, int thi) {
  const int lane = threadIdx.x & 31;
  for (int t0 = tlo; t0 <= thi; t0 += 32) {
    const int t = t0 + lane;
    bool f = false;
    if (t <= thi) f = cost_bits(stripe_edge_before(a, t * kRefSwath)[a.m - 1]) == a.fmin[t];
    const unsigned ballot = __ballot_sync(kFull, f);
    if (ballot) {
      if (lane == 0) a.walk->s_fwd = t0 + __ffs(ballot) - 1;
      return;
    }
  }
}

template <typename T, int R>
__device__ __forceinline__ T stripe_tile_swath(const SwathJob<T> &job, const PathOut &po,
                                               const TileIn<T> &tile) {
  T col[R];
  T emin, etop;
  sweep_swath_path<T, R>(job, po, col, emin, etop, tile);
  return etop;
}

// One warp per K-row tile of swath s below the backtrack height, into move
// buffer buf.
template <typename T, int RF, int RQ>
__global__ void __launch_bounds__(kRoundWarps * 32) stripe_tile_kernel(StripeArgs<T> a, int s, int buf) {
  __shared__ __align__(16) T stage_mem[kRoundWarps * kStageElems];
  constexpr int W = 32 * RF;
  const int kt = blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
  const StripeWalk w = *a.walk;
  const int H = w.h;
  const int K = 1 << a.shift;
  const long long rb_l = (long long)a.r0 + (long long)kt * K;
  const int c0 = s * W;
  if (w.state != 0 || rb_l >= H || stripe_fires(a, c0 / kRefSwath, H, w)) return;
  const int rb = int(rb_l);
  const int re = rb + K < H ? rb + K : H;
  SwathJob<T> job;
  job.x = stripe_rows_ptr(a);
  job.y = stripe_cols_ptr(a);
  job.m = re;
  job.n = a.n;
  job.c0 = c0;
  job.r0 = rb;
  const T *left = s ? a.E + (unsigned long long)(s - 1) * a.e_stride : nullptr;
  job.edge_in = left ? left + (unsigned long long)kt * K : nullptr;
  job.edge_out = nullptr;
  job.open_end = a.oe != 0;
  job.free_diag0 = c0 > 0 && (c0 % kRefSwath) == 0;
  job.corner_init = kt == 0 ? stripe_corner<T>(c0, a.r0)
                            : (left ? left[(unsigned long long)kt * K - 1] : Num<T>::big());
  job.stage = stage_mem + (threadIdx.x >> 5) * kStageElems;
  TileIn<T> tile;
  tile.col_init = kt ? a.Q + (unsigned long long)(kt - 1) * a.q_stride + c0 : nullptr;
  // the re-run's top row is the backtrack height's (open end), the last row otherwise
  tile.top_row = a.oe ? H - 1 : a.m - 1;
  tile.top_left = (a.oe && (c0 % kRefSwath) != 0) ? a.top_carry : nullptr;
  PathOut po;
  po.words = a.words + (unsigned long long)buf * a.words_stride + (unsigned long long)kt * (K / 2) * 64ull;
  po.track_min = false;
  const int R = stripe_regs<T>(a.n, s);
  T etop = T(0);
  if (R == RF) {
    etop = stripe_tile_swath<T, RF>(job, po, tile);
  } else {
    switch (R / RQ) {
#define ODBA_TCASE(K)                                                         \
  case K:                                                                     \
    if constexpr (K * RQ < RF) etop = stripe_tile_swath<T, K * RQ>(job, po, tile); \
    break;
      ODBA_TCASE(1)
      ODBA_TCASE(2)
      ODBA_TCASE(3)
      ODBA_TCASE(4)
      ODBA_TCASE(5)
      ODBA_TCASE(6)
      ODBA_TCASE(7)
#undef ODBA_TCASE
      default:
        break;
    }
  }
  // the first half of a two-swath stripe hands its recomputed top row's last
  // value to the second half
  if (a.oe && re == H && (c0 % kRefSwath) == 0 && c0 + W < a.n && W < kRefSwath &&
      (threadIdx.x & 31) == 0)
    *a.top_carry = etop;
}

__global__ void stripe_walk_init_kernel(StripeWalk *w, int m, int n) {
  if (threadIdx.x || blockIdx.x) return;
  w->r = m - 1;
  w->c = n - 1;
  w->h = m;
  w->cur_t = -1;
  w->lo = 1;
  w->hi = 0;
  w->state = 0;
  w->s_fwd = INT_MAX;
  w->nt = 0;
}

// Continues the backtrack through swath s (updateCentroid's loop,
// dba.hpp:393-421, with the stripe branch's height, dba.hpp:384-386) until it
// leaves the swath to the left or reaches the start cell.  One warp: every
// lane holds the move word of one of the 32 rows at and below the current
// cell (the word of the lane that owns the current column), so the walk
// advances by shuffles and reloads the window only when it leaves those 32
// rows or that owner's columns.  Every lane keeps the same walk state; lane 0
// does the stores.  The height moves to the walk's row when it leaves a
// reference stripe (with an open end only then; a shorter re-run is the same
// without one).
template <typename T>
__global__ void stripe_walk_kernel(StripeArgs<T> a, int s, int buf) {
  const int lane = threadIdx.x & 31;
  if (blockIdx.x) return;
  StripeWalk w = *a.walk;
  if (w.state) return;
  constexpr int W = 32 * PathTune<T>::RF;
  const int c0 = s * W, R = stripe_regs<T>(a.n, s);
  const int os = a.r0;
  const long long max_cells = (long long)a.m + a.n - 1;
  const unsigned long long *words = a.words + (unsigned long long)buf * a.words_stride;
  int2 *rg = a.ranges;
  int32_t *tri = a.triples;
  const bool lead = lane == 0;
  // rr: the member's sample index, cc: the centroid index
  auto contribute = [&](int rr, int cc) {
    if (cc != w.cur_t) {
      if (lead && w.cur_t >= 0 && w.hi >= w.lo) rg[w.cur_t] = make_int2(w.lo, w.hi);
      w.cur_t = cc;
      w.lo = rr;
      w.hi = rr;
    } else if (rr == w.lo - 1) {
      w.lo = rr;
    } else if (lead && a.extra) {
      // past an OPEN_RIGHT run on a re-run's top row (centroid on the rows)
      a.extra[cc] = rr;
    }
  };
  auto contribute_cell = [&](int r, int c) {
    if (a.flip)
      contribute(c, r);
    else
      contribute(r, c);
  };
  auto emit = [&](int mv) {
    if (lead && tri) {
      tri[3 * w.nt] = w.r;
      tri[3 * w.nt + 1] = w.c;
      tri[3 * w.nt + 2] = mv;
    }
    ++w.nt;
  };
  const int H = w.h;
  if (stripe_fires(a, c0 / kRefSwath, H, w)) {
    // the re-run's shortcut: row H-1 of the stripe is OPEN_RIGHT throughout
    for (; w.c >= c0; --w.c) {
      if (w.nt >= max_cells - 1) {
        w.state = 2;
        break;
      }
      emit(kMoveOpenRight);
    }
  }
  bool swath_done = w.c < c0 || w.state != 0;
  while (!swath_done && w.state == 0) {
    // window: rows w.r - lane, columns of the owner lane of w.c
    const int top = w.r, owner = (w.c - c0) / R, cbeg = c0 + owner * R;
    unsigned long long word = 0;
    const int my_row = top - lane;
    if (my_row >= 1) {
      const int rr = my_row - a.r0;
      const unsigned long long t = (unsigned long long)owner + (rr >> 1);
      word = words[(t * 32 + owner) * 2 + (rr & 1)];
    }
    for (;;) {
      int mv;
      const unsigned long long wv = __shfl_sync(kFull, word, (top - w.r) & 31);
      if (w.r == 0) {
        mv = w.c == 0 ? (os ? kMoveNilOpenRight : kMaxMoveNil) : (os ? kMoveOpenRight : kMoveRight);
      } else {
        mv = decode_move(wv, w.c - cbeg);
        if (mv == kMoveRight && a.oe && w.r == H - 1) mv = kMoveOpenRight;
      }
      if (mv == kMaxMoveNil || mv == kMoveNilOpenRight) {
        // the start cell (dba.hpp:412-415)
        if (mv != kMoveNilOpenRight) contribute(0, 0);
        if (lead && w.cur_t >= 0 && w.hi >= w.lo) rg[w.cur_t] = make_int2(w.lo, w.hi);
        emit(mv);
        if (lead && a.triple_count) *a.triple_count = w.nt;
        w.state = 1;
        break;
      }
      if (w.nt >= max_cells - 1) {
        w.state = 2;
        break;
      }
      emit(mv);
      if (mv != kMoveOpenRight) contribute_cell(w.r, w.c);
      if (mv == kMoveDiag) {
        --w.r;
        --w.c;
      } else if (mv == kMoveUp) {
        --w.r;
      } else {
        --w.c;
      }
      if (w.r < 0 || w.c < 0) {
        w.state = 2;
        break;
      }
      if (w.c < c0) {
        swath_done = true;
        break;
      }
      if (top - w.r >= 32 || w.c < cbeg) break;  // reload the window
    }
  }
  if (w.state == 0 && w.c < c0 && (!a.oe || (c0 % kRefSwath) == 0)) w.h = w.r + 1;
  if (lead) {
    if (w.state == 2 && a.triple_count) *a.triple_count = -1;
    *a.walk = w;
  }
}

template <typename T>
int stripe_grid() {
  static std::atomic<int> cached[64];  // per device; host threads may race (same value)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64) {
    const int c = cached[dev].load(std::memory_order_relaxed);
    if (c) return c;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, stripe_forward_kernel<T, PathTune<T>::RF, PathTune<T>::RQ, false, false>,
      kRoundWarps * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int g = sms * per_sm;
  if (dev >= 0 && dev < 64) cached[dev].store(g, std::memory_order_relaxed);
  return g;
}

// One member's matrix: rows x columns in the round's orientation.
struct StripeDims {
  int flip;
  uint64_t rows, cols;
};
inline StripeDims stripe_dims(uint64_t len, uint64_t Lc, int oe) {
  StripeDims d;
  d.flip = (oe && Lc < len) ? 1 : 0;
  d.rows = d.flip ? Lc : len;
  d.cols = d.flip ? len : Lc;
  return d;
}

struct StripeLayout {
  RoundLayout round;
  size_t off_head, off_prog, off_E, off_Q, off_W, off_min, off_extra, total;
  unsigned long long e_stride, q_stride, words_stride;
  int swaths_max, stripes_max;
};

template <typename T>
StripeLayout stripe_layout(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe, int shift) {
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  constexpr int W = 32 * PathTune<T>::RF;
  uint64_t max_rows = 1, max_cols = 1;
  for (int k = 0; k < n; ++k) {
    const StripeDims d = stripe_dims(h_lens[k], Lc, oe);
    max_rows = d.rows > max_rows ? d.rows : max_rows;
    max_cols = d.cols > max_cols ? d.cols : max_cols;
  }
  StripeLayout S;
  S.round = round_layout<T>(n, 1, 0, (unsigned long long)n * Lc, 1);
  S.swaths_max = int((max_cols + W - 1) / W);
  S.stripes_max = int((max_cols + kRefSwath - 1) / kRefSwath);
  S.e_stride = (max_rows + 64 + 31) / 32 * 32;
  S.q_stride = (unsigned long long)S.swaths_max * W;
  const unsigned long long K = 1ull << shift;
  const unsigned long long nq = (max_rows - (os ? 1 : 0)) / K + 1;
  const unsigned long long steps = (max_rows + 1) / 2 + 32;
  S.words_stride = steps * 64;
  const int bufs = (oe && W < kRefSwath) ? 2 : 1;
  size_t o = S.round.total;
  S.off_head = o; o += 256;
  S.off_prog = o; o += up(size_t(S.swaths_max) * 8);
  S.off_E = o; o += up(size_t(S.swaths_max > 1 ? S.swaths_max - 1 : 1) * S.e_stride * sizeof(T));
  S.off_Q = o; o += up(size_t(nq) * S.q_stride * sizeof(T));
  S.off_W = o; o += up(size_t(bufs) * S.words_stride * 8);
  S.off_min = o; o += up(size_t(2) * (S.stripes_max + 1) * 8);
  S.off_extra = o; o += oe ? up(size_t(n) * Lc * 4) : 0;
  S.total = o;
  return S;
}

int stripe_shift(int ckpt_rows) {
  if (ckpt_rows == 0) return 12;  // 4096 rows per tile
  if (ckpt_rows < 2 || (ckpt_rows & (ckpt_rows - 1))) return -1;
  int sh = 0;
  while ((1 << sh) < ckpt_rows) ++sh;
  return sh;
}

}  // namespace

template <typename T>
size_t dba_round_stripe_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe,
                                        int ckpt_rows) {
  const int sh = stripe_shift(ckpt_rows);
  if (sh < 0 || n < 1 || Lc == 0) return 0;
  return stripe_layout<T>(h_lens, n, Lc, os, oe, sh).total;
}

template <typename T>
int dba_round_stripe_launch(const T *centroid, uint64_t Lc, const T *series,
                            const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                            int n, int os, int oe, int ckpt_rows, T *mean, uint32_t *counts,
                            double *delta, int32_t *triples, int64_t *triple_counts, void *ws,
                            size_t ws_bytes, cudaStream_t stream) {
  const int sh = stripe_shift(ckpt_rows);
  if (sh < 0) return fail(ODBA_ERR_INVALID_ARGUMENT, "checkpoint rows must be a power of two >= 2 (0: default)");
  const StripeLayout S = stripe_layout<T>(h_lens, n, Lc, os, oe, sh);
  if (ws_bytes < S.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "stripe DBA round workspace too small");
  const RoundLayout &L = S.round;
  char *base = static_cast<char *>(ws);
  int *single = reinterpret_cast<int *>(base + L.off_single);
  int *mseries = single, *mjob = single + n, *d_clen = single + 2 * n, *d_flags = single + 2 * n + 1,
      *d_mbeg = single + 2 * n + 2, *d_mend = single + 2 * n + 3;
  unsigned long long *d_coff =
      reinterpret_cast<unsigned long long *>(base + L.off_single + ((size_t(2 * n + 4) * 4 + 7) / 8) * 8);
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  single_job_kernel<<<(n + 255) / 256, 256, 0, stream>>>(mseries, mjob, n, d_clen, int(Lc), d_flags,
                                                        flags, d_mbeg, d_mend, d_coff);
  int *extra = oe ? reinterpret_cast<int *>(base + S.off_extra) : nullptr;
  RoundArgs<T> a;
  a.centroids = centroid;
  a.coff = d_coff;
  a.clen = d_clen;
  a.jflags = d_flags;
  a.mbeg = d_mbeg;
  a.mend = d_mend;
  a.njobs = 1;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.mseries = mseries;
  a.mjob = mjob;
  a.order = nullptr;
  a.nmem = n;
  a.means = mean;
  a.counts = counts;
  a.deltas = delta;
  a.triples = triples;
  a.triple_counts = triple_counts;
  a.extra = extra;
  a.counter = reinterpret_cast<unsigned long long *>(base + L.off_counter);
  a.path_off = reinterpret_cast<unsigned long long *>(base + L.off_path);
  a.trip_off = reinterpret_cast<unsigned long long *>(base + L.off_trip);
  a.rng_off = reinterpret_cast<unsigned long long *>(base + L.off_rng);
  a.shortcut = reinterpret_cast<int *>(base + L.off_short);
  a.ranges = reinterpret_cast<int2 *>(base + L.off_ranges);
  a.edges = reinterpret_cast<T *>(base + L.off_edges);
  a.edge_stride = L.edge_stride;
  a.words = reinterpret_cast<unsigned long long *>(base + L.off_words);
  const unsigned long long nr = (unsigned long long)n * Lc;
  plan_kernel<T><<<1, kPlanThreads, 0, stream>>>(a);
  fill_ranges_kernel<<<int(nr / 256 + 1 < 4096 ? nr / 256 + 1 : 4096), 256, 0, stream>>>(a.ranges, nr);
  if (extra) cudaMemsetAsync(extra, 0xff, size_t(nr) * 4, stream);
  if (int rc = check_launch("stripe DBA round set-up")) return rc;

  constexpr int RF = PathTune<T>::RF, RQ = PathTune<T>::RQ;
  constexpr int W = 32 * RF;
  constexpr int kPerStripe = kRefSwath / W;  // swaths per reference stripe
  char *head = base + S.off_head;
  StripeArgs<T> sa;
  sa.series = series;
  sa.offsets = offsets;
  sa.centroid = centroid;
  sa.r0 = os ? 1 : 0;
  sa.oe = oe ? 1 : 0;
  sa.shift = sh;
  sa.E = reinterpret_cast<T *>(base + S.off_E);
  sa.e_stride = S.e_stride;
  sa.Q = reinterpret_cast<T *>(base + S.off_Q);
  sa.q_stride = S.q_stride;
  sa.prog = reinterpret_cast<unsigned long long *>(base + S.off_prog);
  sa.counter = reinterpret_cast<unsigned long long *>(head);
  // the wait error word is byte 8 of the workspace, as in the full-path round
  sa.err = reinterpret_cast<unsigned *>(base + L.off_counter + 8);
  cudaMemsetAsync(base + L.off_counter, 0, 16, stream);
  sa.walk = reinterpret_cast<StripeWalk *>(head + 64);
  sa.top_carry = reinterpret_cast<T *>(head + 192);
  sa.words = reinterpret_cast<unsigned long long *>(base + S.off_W);
  sa.words_stride = S.words_stride;
  sa.fmin = reinterpret_cast<unsigned long long *>(base + S.off_min);
  sa.cmin = sa.fmin + (S.stripes_max + 1);
  sa.limit_ns = kWaitLimitNs;
  const bool check_short = oe && !os;
  const int K = 1 << sh;
  unsigned long long trip = 0;
  for (int k = 0; k < n; ++k) {
    const StripeDims d = stripe_dims(h_lens[k], Lc, oe);
    const int m = int(d.rows), ncols = int(d.cols);
    const int swaths = (ncols + W - 1) / W;
    const int stripes = (ncols + kRefSwath - 1) / kRefSwath;
    sa.member = k;
    sa.flip = d.flip;
    sa.m = m;
    sa.n = ncols;
    sa.swaths = swaths;
    sa.ranges = a.ranges + (unsigned long long)k * Lc;
    sa.extra = extra ? extra + (unsigned long long)k * Lc : nullptr;
    sa.triples = triples ? triples + 3ull * trip : nullptr;
    sa.triple_count = triple_counts ? triple_counts + k : nullptr;
    trip += h_lens[k] + Lc + 1;
    cudaMemsetAsync(head, 0, 64, stream);
    cudaMemsetAsync(sa.prog, 0, size_t(swaths) * 8, stream);
    if (check_short) cudaMemsetAsync(sa.fmin, 0xff, size_t(2) * (S.stripes_max + 1) * 8, stream);
    stripe_walk_init_kernel<<<1, 32, 0, stream>>>(sa.walk, m, ncols);
    const int fgrid = swaths < stripe_grid<T>() * kRoundWarps ? (swaths + kRoundWarps - 1) / kRoundWarps
                                                              : stripe_grid<T>();
    if (!oe)
      stripe_forward_kernel<T, RF, RQ, false, false><<<fgrid, kRoundWarps * 32, 0, stream>>>(sa);
    else if (!d.flip)
      stripe_forward_kernel<T, RF, RQ, true, false><<<fgrid, kRoundWarps * 32, 0, stream>>>(sa);
    else
      stripe_forward_kernel<T, RF, RQ, true, true><<<fgrid, kRoundWarps * 32, 0, stream>>>(sa);
    // stripes past the last row: where the forward pass's shortcut fired first
    const int tlo = m / kRefSwath + 1, thi = stripes - 1;
    const int gx = (m + 2047) / 2048 < 64 ? (m + 2047) / 2048 : 64;
    if (check_short && tlo <= thi) {
      const int gy = thi - tlo + 1 < 1024 ? thi - tlo + 1 : 1024;
      stripe_min_kernel<T><<<dim3(gx, gy), 256, 0, stream>>>(sa, tlo, thi, 1);
      stripe_sfwd_kernel<T><<<1, 32, 0, stream>>>(sa, tlo, thi);
    }
    const int tiles = (m - sa.r0 + K - 1) / K;
    const int tgrid = ((tiles > 1 ? tiles : 1) + kRoundWarps - 1) / kRoundWarps;
    auto tile = [&](int s, int buf) {
      stripe_tile_kernel<T, RF, RQ><<<tgrid, kRoundWarps * 32, 0, stream>>>(sa, s, buf);
    };
    auto walk = [&](int s, int buf) { stripe_walk_kernel<T><<<1, 32, 0, stream>>>(sa, s, buf); };
    for (int t = stripes - 1; t >= 0; --t) {
      if (check_short && t >= 1) stripe_min_kernel<T><<<dim3(gx, 1), 256, 0, stream>>>(sa, t, t, 0);
      const int s_lo = t * kPerStripe;
      const int s_hi = s_lo + kPerStripe - 1 < swaths - 1 ? s_lo + kPerStripe - 1 : swaths - 1;
      if (oe && s_hi > s_lo) {
        // the second half continues the first half's recomputed top row
        for (int s = s_lo; s <= s_hi; ++s) tile(s, s - s_lo);
        for (int s = s_hi; s >= s_lo; --s) walk(s, s - s_lo);
      } else {
        for (int s = s_hi; s >= s_lo; --s) {
          tile(s, 0);
          walk(s, 0);
        }
      }
    }
    if (int rc = check_launch("stripe DBA round member kernels")) return rc;
  }
  dim3 rg((unsigned(Lc) + kReduceWarps - 1) / kReduceWarps, 1);
  reduce_kernel<T><<<rg, kReduceThreads, 0, stream>>>(a);
  return check_launch("stripe DBA round reduce");
}

template size_t dba_round_stripe_workspace_bytes<float>(const uint64_t *, int, uint64_t, int, int, int);
template size_t dba_round_stripe_workspace_bytes<double>(const uint64_t *, int, uint64_t, int, int, int);
template int dba_round_stripe_launch<float>(const float *, uint64_t, const float *, const uint64_t *,
                                            const uint64_t *, const uint64_t *, int, int, int, int,
                                            float *, uint32_t *, double *, int32_t *, int64_t *,
                                            void *, size_t, cudaStream_t);
template int dba_round_stripe_launch<double>(const double *, uint64_t, const double *,
                                             const uint64_t *, const uint64_t *, const uint64_t *,
                                             int, int, int, int, double *, uint32_t *, double *,
                                             int32_t *, int64_t *, void *, size_t, cudaStream_t);

// ---------------------------------------------------------------------------
// Prefix chop (chopPrefixFromSequences, dba.hpp:1191-1395): every series is
// aligned to the leader with open-end DTW and a recorded path (leader on the
// rows, whatever the lengths), by the DBA round's path kernels; then one warp
// per series walks its path (chop_walk_kernel).
namespace {
constexpr int kChopFlags = 2 | 4 | 8;  // open end, active, centroid (the leader) on the rows
}  // namespace

template <typename T>
size_t prefix_chop_workspace_bytes(const uint64_t *h_lens, int n, uint64_t P) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = P;
  const int flags = kChopFlags;
  int ms = 1;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm, &ms);
  if (P > maxm) maxm = P;
  return round_layout<T>(n, 1, words, ranges, maxm, ms).total;
}

template <typename T>
int prefix_chop_launch(const T *prefix, uint64_t P, const T *series, const uint64_t *offsets,
                       const uint64_t *lens, const uint64_t *h_lens, int n, long long *chop,
                       int *hist, void *ws, size_t ws_bytes, cudaStream_t stream) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = P;
  const int flags = kChopFlags;
  int ms = 1;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm, &ms);
  if (P > maxm) maxm = P;
  const RoundLayout L = round_layout<T>(n, 1, words, ranges, maxm, ms);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "prefix chop workspace too small");
  char *base = static_cast<char *>(ws);
  int *single = reinterpret_cast<int *>(base + L.off_single);
  int *mseries = single, *mjob = single + n, *d_clen = single + 2 * n, *d_flags = single + 2 * n + 1,
      *d_mbeg = single + 2 * n + 2, *d_mend = single + 2 * n + 3;
  unsigned long long *d_coff =
      reinterpret_cast<unsigned long long *>(base + L.off_single + ((size_t(2 * n + 4) * 4 + 7) / 8) * 8);
  single_job_kernel<<<(n + 255) / 256, 256, 0, stream>>>(mseries, mjob, n, d_clen, int(P), d_flags,
                                                        flags, d_mbeg, d_mend, d_coff);
  RoundArgs<T> a;
  a.centroids = prefix;
  a.coff = d_coff;
  a.clen = d_clen;
  a.jflags = d_flags;
  a.mbeg = d_mbeg;
  a.mend = d_mend;
  a.njobs = 1;
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.mseries = mseries;
  a.mjob = mjob;
  a.order = nullptr;
  a.nmem = n;
  a.means = nullptr;
  a.counts = nullptr;
  // the planner clears the job's delta: a spare word of the counter block
  a.deltas = reinterpret_cast<double *>(base + L.off_counter + 16);
  a.triples = nullptr;
  a.triple_counts = nullptr;
  cudaMemsetAsync(hist, 0, size_t(n) * P * sizeof(int), stream);
  launch_paths<T>(a, L, base, stream);
  chop_walk_kernel<T><<<(n + kRoundWarps - 1) / kRoundWarps, kRoundWarps * 32, 0, stream>>>(a, chop, hist,
                                                                                          int(P));
  return check_launch("prefix chop kernels");
}

template size_t prefix_chop_workspace_bytes<float>(const uint64_t *, int, uint64_t);
template size_t prefix_chop_workspace_bytes<double>(const uint64_t *, int, uint64_t);
template int prefix_chop_launch<float>(const float *, uint64_t, const float *, const uint64_t *,
                                       const uint64_t *, const uint64_t *, int, long long *, int *,
                                       void *, size_t, cudaStream_t);
template int prefix_chop_launch<double>(const double *, uint64_t, const double *, const uint64_t *,
                                        const uint64_t *, const uint64_t *, int, long long *, int *,
                                        void *, size_t, cudaStream_t);

template size_t dba_round_workspace_bytes<float>(const uint64_t *, int, uint64_t, int, int);
template size_t dba_round_workspace_bytes<double>(const uint64_t *, int, uint64_t, int, int);
template int dba_round_launch<float>(const float *, uint64_t, const float *, const uint64_t *,
                                     const uint64_t *, const uint64_t *, int, int, int, float *,
                                     uint32_t *, double *, int32_t *, int64_t *, void *, size_t,
                                     cudaStream_t);
template int dba_round_launch<double>(const double *, uint64_t, const double *, const uint64_t *,
                                      const uint64_t *, const uint64_t *, int, int, int, double *,
                                      uint32_t *, double *, int32_t *, int64_t *, void *, size_t,
                                      cudaStream_t);
template int dba_round_ranges_launch<float>(const float *, uint64_t, const float *, const uint64_t *,
                                            const uint64_t *, const uint64_t *, int, int, int, int2 *,
                                            void *, size_t, cudaStream_t);
template int dba_round_ranges_launch<double>(const double *, uint64_t, const double *,
                                             const uint64_t *, const uint64_t *, const uint64_t *, int,
                                             int, int, int2 *, void *, size_t, cudaStream_t);
template size_t dba_reduce_workspace_bytes<float>(int);
template size_t dba_reduce_workspace_bytes<double>(int);
template int dba_reduce_ranges_launch<float>(const float *, uint64_t, const float *, const uint64_t *,
                                             const uint64_t *, int, int, int, const int2 *, float *,
                                             uint32_t *, double *, void *, size_t, cudaStream_t);
template int dba_reduce_ranges_launch<double>(const double *, uint64_t, const double *,
                                              const uint64_t *, const uint64_t *, int, int, int,
                                              const int2 *, double *, uint32_t *, double *, void *,
                                              size_t, cudaStream_t);
template size_t dba_batch_workspace_bytes<float>(const uint64_t *, const int *, int,
                                                 const uint64_t *, const int *, int);
template size_t dba_batch_workspace_bytes<double>(const uint64_t *, const int *, int,
                                                  const uint64_t *, const int *, int);
template int dba_batch_launch<float>(const float *, const unsigned long long *, const int *,
                                     const int *, const int *, const int *, int, int,
                                     const float *, const uint64_t *, const uint64_t *,
                                     const int *, const int *, const int *, int, const uint64_t *,
                                     const int *, const uint64_t *, const int *, float *,
                                     uint32_t *, double *, int32_t *, int64_t *, void *, size_t,
                                     cudaStream_t);
template int dba_batch_launch<double>(const double *, const unsigned long long *, const int *,
                                      const int *, const int *, const int *, int, int,
                                      const double *, const uint64_t *, const uint64_t *,
                                      const int *, const int *, const int *, int,
                                      const uint64_t *, const int *, const uint64_t *, const int *,
                                      double *, uint32_t *, double *, int32_t *, int64_t *, void *,
                                      size_t, cudaStream_t);

}  // namespace odba
