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

#include <cstdint>
#include <vector>

#include "dtw_path.cuh"
#include "odba_internal.h"

namespace odba {

namespace {

constexpr int kRoundWarps = 4;
constexpr int kMaxMoveNil = 255, kMoveDiag = 1, kMoveRight = 2, kMoveUp = 3, kMoveOpenRight = 4,
              kMoveNilOpenRight = 5;

template <typename T>
struct PathTune;
template <>
struct PathTune<float> {
  static constexpr int RF = 32, RQ = 4;
};
template <>
struct PathTune<double> {
  static constexpr int RF = 16, RQ = 4;
};

// Geometry of one member's cost matrix, identical on host and device.
struct MemberGeom {
  int flip, m, n, r0, swaths, steps;
  unsigned long long words;
};

template <typename T>
__host__ __device__ inline MemberGeom member_geom(uint64_t len, uint64_t Lc, int os, int oe) {
  MemberGeom g;
  g.flip = (oe && Lc < len) ? 1 : 0;
  g.m = int(g.flip ? Lc : len);
  g.n = int(g.flip ? len : Lc);
  g.r0 = os ? 1 : 0;
  const int W = 32 * PathTune<T>::RF;
  g.swaths = (g.n + W - 1) / W;
  g.steps = (g.m - g.r0 + 1) / 2 + 31;
  g.words = (unsigned long long)g.swaths * g.steps * 64ull;
  return g;
}

// Jobs share one launch: job J owns centroid centroids[coff[J] .. + clen[J]),
// flags (bit 0 open start, bit 1 open end, bit 2 active) and the members
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
  int *shortcut;                 // first column of the open-end shortcut, or 0
  int2 *ranges;
  T *edges;
  unsigned long long edge_stride;
  unsigned long long *words;
  T *means;
  uint32_t *counts;
  double *deltas;
  int32_t *triples;
  int64_t *triple_counts;
};

template <typename T>
__device__ __forceinline__ MemberGeom geom_of(const RoundArgs<T> &a, int k, int &job) {
  job = a.mjob[k];
  const int f = a.jflags[job];
  return member_geom<T>(a.lens[a.mseries[k]], uint64_t(a.clen[job]), f & 1, (f >> 1) & 1);
}

template <typename T>
__global__ void plan_kernel(RoundArgs<T> a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long w = 0, p = 0, r = 0;
  for (int k = 0; k < a.nmem; ++k) {
    int job;
    const MemberGeom g = geom_of<T>(a, k, job);
    a.path_off[k] = w;
    a.trip_off[k] = p;
    a.rng_off[k] = r;
    w += g.words;
    p += (unsigned long long)(g.m + g.n + 1);
    r += (unsigned long long)a.clen[job];
  }
  for (int j = 0; j < a.njobs; ++j)
    if (a.jflags[j] & 4) a.deltas[j] = 0.0;
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

template <typename T, int RF, int RQ>
__global__ void __launch_bounds__(kRoundWarps * 32) path_dtw_kernel(RoundArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const long long slot = (long long)blockIdx.x * kRoundWarps + (threadIdx.x >> 5);
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
      const int rq = ((width + 31) / 32 + RQ - 1) / RQ * RQ;
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

// Decodes the reference's move at (r, c) of member geometry g.
template <typename T>
__device__ __forceinline__ int move_at(const MemberGeom &g, int os, int oe,
                                       const unsigned long long *w, int shortcut, int r, int c,
                                       unsigned long long &cache_idx,
                                       unsigned long long &cache_word) {
  // the shortcut overrides the top row first: with a single-row matrix that
  // row is row 0 (dtw.hpp:105-108 runs before the row-0 loop)
  if (shortcut && r == g.m - 1 && c >= shortcut) return kMoveOpenRight;
  if (r == 0) {
    if (c == 0) return os ? kMoveNilOpenRight : kMaxMoveNil;
    return os ? kMoveOpenRight : kMoveRight;
  }
  constexpr int RF = PathTune<T>::RF, RQ = PathTune<T>::RQ, W = 32 * RF;
  const int s = c / W;
  const int c0 = s * W;
  int R = RF;
  if (s == g.swaths - 1) {
    const int width = g.n - c0;
    const int rq = ((width + 31) / 32 + RQ - 1) / RQ * RQ;
    R = rq < RF ? rq : RF;
  }
  const int cl = c - c0;
  const int lane = cl / R, j = cl - lane * R;
  const int rr = r - g.r0;
  const int t = lane + (rr >> 1);
  const unsigned long long idx =
      (unsigned long long)s * g.steps * 64ull + ((unsigned long long)t * 32 + lane) * 2 + (rr & 1);
  if (idx != cache_idx) {
    cache_word = w[idx];
    cache_idx = idx;
  }
  const int code = int((cache_word >> (2 * j)) & 3ull);
  if (code == kMoveRight && oe && r == g.m - 1) return kMoveOpenRight;
  return code;
}

template <typename T>
__global__ void backtrack_kernel(RoundArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nmem) return;
  int jb;
  const MemberGeom g = geom_of<T>(a, k, jb);
  const int flags = a.jflags[jb];
  if (!(flags & 4)) return;
  const int os = flags & 1, oe = (flags >> 1) & 1;
  const unsigned long long *w = a.words + a.path_off[k];
  const int shortcut = a.shortcut[k];
  int2 *rg = a.ranges + a.rng_off[k];
  int32_t *tri = a.triples ? a.triples + 3ull * a.trip_off[k] : nullptr;
  long long nt = 0;
  int r = g.m - 1, c = g.n - 1;
  unsigned long long cache_idx = ~0ull, cache_word = 0;
  int cur_t = -1, lo = 1, hi = 0;
  auto contribute = [&](int rr, int cc) {
    const int ti = g.flip ? rr : cc;     // centroid index
    const int mi = g.flip ? cc : rr;     // member sample index
    if (ti != cur_t) {
      if (cur_t >= 0 && hi >= lo) rg[cur_t] = make_int2(lo, hi);
      cur_t = ti;
      lo = mi;
      hi = mi;
    } else {
      lo = mi;  // the walk only moves toward smaller indices
    }
  };
  int mv = move_at<T>(g, os, oe, w, shortcut, r, c, cache_idx, cache_word);
  // A path has at most m + n - 1 cells and never leaves the matrix; the checks
  // only keep a corrupt path buffer from turning into an endless or
  // out-of-bounds walk (the member is then reported with a count of -1).
  const long long max_cells = (long long)g.m + g.n - 1;
  while (mv != kMaxMoveNil && mv != kMoveNilOpenRight) {
    if (nt >= max_cells - 1) {
      if (a.triple_counts) a.triple_counts[k] = -1;
      return;
    }
    if (tri) {
      tri[3 * nt] = r;
      tri[3 * nt + 1] = c;
      tri[3 * nt + 2] = mv;
    }
    ++nt;
    if (mv != kMoveOpenRight) contribute(r, c);
    if (mv == kMoveDiag) {
      --r;
      --c;
    } else if (mv == kMoveUp) {
      --r;
    } else {
      --c;
    }
    if (r < 0 || c < 0) {
      if (a.triple_counts) a.triple_counts[k] = -1;
      return;
    }
    mv = move_at<T>(g, os, oe, w, shortcut, r, c, cache_idx, cache_word);
  }
  // the start cell (dba.hpp:412-415)
  if (mv != kMoveNilOpenRight) contribute(0, 0);
  if (cur_t >= 0 && hi >= lo) rg[cur_t] = make_int2(lo, hi);
  if (tri) {
    tri[3 * nt] = r;
    tri[3 * nt + 1] = c;
    tri[3 * nt + 2] = mv;
  }
  ++nt;
  if (a.triple_counts) a.triple_counts[k] = nt;
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
__global__ void reduce_kernel(RoundArgs<T> a) {
  __shared__ double smax[256];
  const int jb = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int Lc = a.clen[jb];
  const bool live = (a.jflags[jb] & 4) != 0;
  double dl = 0.0;
  if (live && t < Lc) {
    T sum = T(0);
    uint32_t cnt = 0;
    for (int k = a.mbeg[jb]; k < a.mend[jb]; ++k) {
      const int2 r = a.ranges[a.rng_off[k] + t];
      if (r.y < r.x) continue;
      const T *seq = a.series + a.offsets[a.mseries[k]];
      for (int i = r.y; i >= r.x; --i) sum = add_rn(sum, seq[i]);
      cnt += uint32_t(r.y - r.x + 1);
    }
    const T mean = cnt ? div_rn<T>(sum, T(cnt)) : host_default_nan<T>();
    a.means[a.coff[jb] + t] = mean;
    a.counts[a.coff[jb] + t] = cnt;
    const double d = fabs(double(a.centroids[a.coff[jb] + t] - mean));
    dl = d > 0.0 ? d : 0.0;  // NaN never raises the maximum (dba.hpp:833)
  }
  smax[threadIdx.x] = dl;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && smax[threadIdx.x + s] > smax[threadIdx.x])
      smax[threadIdx.x] = smax[threadIdx.x + s];
    __syncthreads();
  }
  // non-negative doubles order like their bit patterns
  if (threadIdx.x == 0 && live)
    atomicMax(reinterpret_cast<unsigned long long *>(a.deltas + jb),
              (unsigned long long)__double_as_longlong(smax[0]));
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
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && cached[dev]) return cached[dev];
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ>, kRoundWarps * 32, 0);
  if (per_sm < 1) per_sm = 1;
  const int g = sms * per_sm;
  if (dev < 64) cached[dev] = g;
  return g;
}

struct RoundLayout {
  size_t off_counter, off_path, off_trip, off_rng, off_short, off_single, off_ranges, off_edges,
      off_words, total;
  unsigned long long edge_stride;
};

// Workspace layout for nmem members / njobs jobs with the given totals.
template <typename T>
RoundLayout round_layout(int nmem, int njobs, unsigned long long words,
                         unsigned long long ranges, unsigned long long maxm) {
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  RoundLayout L;
  L.edge_stride = (maxm + 32 + 31) / 32 * 32;
  const size_t slots = size_t(round_grid<T>()) * kRoundWarps;
  size_t o = 0;
  L.off_counter = o; o += 256;
  L.off_path = o; o += up(size_t(nmem) * 8);
  L.off_trip = o; o += up(size_t(nmem) * 8);
  L.off_rng = o; o += up(size_t(nmem) * 8);
  L.off_short = o; o += up(size_t(nmem) * 4);
  // single-job descriptors: mseries, mjob (nmem ints each), clen, jflags, mbeg, mend, coff
  L.off_single = o; o += up(size_t(nmem) * 8 + 64);
  L.off_ranges = o; o += up(size_t(ranges) * sizeof(int2));
  L.off_edges = o; o += up(slots * 2 * L.edge_stride * sizeof(T));
  L.off_words = o; o += up(words * 8);
  L.total = o;
  (void)njobs;
  return L;
}

template <typename T>
void host_totals(const uint64_t *h_lens, const int *h_mjob, int nmem, const uint64_t *h_clen,
                 const int *h_flags, unsigned long long &words, unsigned long long &ranges,
                 unsigned long long &maxm) {
  words = ranges = 0;
  maxm = 1;
  for (int k = 0; k < nmem; ++k) {
    const int j = h_mjob ? h_mjob[k] : 0;
    const int f = h_flags[j];
    const MemberGeom g = member_geom<T>(h_lens[k], h_clen[j], f & 1, (f >> 1) & 1);
    words += g.words;
    ranges += h_clen[j];
    if ((unsigned long long)g.m > maxm) maxm = g.m;
  }
}

template <typename T>
int launch_round(RoundArgs<T> &a, const RoundLayout &L, char *base, int max_clen,
                 cudaStream_t stream) {
  a.counter = reinterpret_cast<unsigned long long *>(base + L.off_counter);
  a.path_off = reinterpret_cast<unsigned long long *>(base + L.off_path);
  a.trip_off = reinterpret_cast<unsigned long long *>(base + L.off_trip);
  a.rng_off = reinterpret_cast<unsigned long long *>(base + L.off_rng);
  a.shortcut = reinterpret_cast<int *>(base + L.off_short);
  a.ranges = reinterpret_cast<int2 *>(base + L.off_ranges);
  a.edges = reinterpret_cast<T *>(base + L.off_edges);
  a.edge_stride = L.edge_stride;
  a.words = reinterpret_cast<unsigned long long *>(base + L.off_words);
  const unsigned long long nr = (L.off_edges - L.off_ranges) / sizeof(int2);
  cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream);
  plan_kernel<T><<<1, 32, 0, stream>>>(a);
  fill_ranges_kernel<<<int(nr / 256 + 1 < 4096 ? nr / 256 + 1 : 4096), 256, 0, stream>>>(a.ranges, nr);
  path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ>
      <<<round_grid<T>(), kRoundWarps * 32, 0, stream>>>(a);
  backtrack_kernel<T><<<(a.nmem + 127) / 128, 128, 0, stream>>>(a);
  dim3 rg((max_clen + 255) / 256, a.njobs);
  reduce_kernel<T><<<rg, 256, 0, stream>>>(a);
  return check_launch("DBA round kernels");
}

}  // namespace

template <typename T>
size_t dba_round_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = Lc;
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm);
  if (Lc > maxm) maxm = Lc;
  return round_layout<T>(n, 1, words, ranges, maxm).total;
}

template <typename T>
int dba_round_launch(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                     const uint64_t *lens, const uint64_t *h_lens, int n, int os, int oe, T *mean,
                     uint32_t *counts, double *delta, int32_t *triples, int64_t *triple_counts,
                     void *ws, size_t ws_bytes, cudaStream_t stream) {
  unsigned long long words, ranges, maxm;
  const uint64_t clen = Lc;
  const int flags = (os ? 1 : 0) | (oe ? 2 : 0) | 4;
  host_totals<T>(h_lens, nullptr, n, &clen, &flags, words, ranges, maxm);
  if (Lc > maxm) maxm = Lc;
  const RoundLayout L = round_layout<T>(n, 1, words, ranges, maxm);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "DBA round workspace too small");
  char *base = static_cast<char *>(ws);
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
  a.means = mean;
  a.counts = counts;
  a.deltas = delta;
  a.triples = triples;
  a.triple_counts = triple_counts;
  return launch_round<T>(a, L, base, int(Lc), stream);
}

template <typename T>
size_t dba_batch_workspace_bytes(const uint64_t *h_mlens, const int *h_mjob, int nmem,
                                 const uint64_t *h_clen, const int *h_flags, int njobs) {
  unsigned long long words, ranges, maxm;
  host_totals<T>(h_mlens, h_mjob, nmem, h_clen, h_flags, words, ranges, maxm);
  for (int j = 0; j < njobs; ++j)
    if (h_clen[j] > maxm) maxm = h_clen[j];
  return round_layout<T>(nmem, njobs, words, ranges, maxm).total;
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
  host_totals<T>(h_mlens, h_mjob, nmem, h_clen, h_flags, words, ranges, maxm);
  for (int j = 0; j < njobs; ++j)
    if (h_clen[j] > maxm) maxm = h_clen[j];
  const RoundLayout L = round_layout<T>(nmem, njobs, words, ranges, maxm);
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
