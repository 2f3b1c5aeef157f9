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

template <typename T>
struct RoundArgs {
  const T *centroid;
  int Lc;
  const T *series;
  const uint64_t *offsets;
  const uint64_t *lens;
  int n, os, oe;
  unsigned long long *counter;
  unsigned long long *path_off;  // word offset of member k's path
  unsigned long long *trip_off;  // triple offset of member k's path listing
  int *shortcut;                 // first column of the open-end shortcut, or 0
  int2 *ranges;                  // [n][Lc] contiguous member-sample range per centroid index
  T *edges;
  unsigned long long edge_stride;
  unsigned long long *words;
  T *mean;
  uint32_t *counts;
  double *delta;
  int32_t *triples;              // optional path listing (i, j, move) per member
  int64_t *triple_counts;
};

template <typename T>
__global__ void plan_kernel(RoundArgs<T> a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long w = 0, p = 0;
  for (int k = 0; k < a.n; ++k) {
    const MemberGeom g = member_geom<T>(a.lens[k], a.Lc, a.os, a.oe);
    a.path_off[k] = w;
    a.trip_off[k] = p;
    w += g.words;
    p += (unsigned long long)(g.m + g.n + 1);
  }
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
    if (q >= (unsigned long long)a.n) break;
    const int k = a.n - 1 - int(q);  // longest members first when sorted by length
    const uint64_t len = a.lens[k];
    const MemberGeom g = member_geom<T>(len, a.Lc, a.os, a.oe);
    const T *seq = a.series + a.offsets[k];
    SwathJob<T> job;
    job.x = g.flip ? a.centroid : seq;
    job.y = g.flip ? seq : a.centroid;
    job.m = g.m;
    job.n = g.n;
    job.r0 = g.r0;
    job.open_end = a.oe != 0;
    int shortcut = 0;
    const bool check_short = a.oe && !a.os;
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
__device__ __forceinline__ int move_at(const RoundArgs<T> &a, const MemberGeom &g,
                                       const unsigned long long *w, int shortcut, int r, int c,
                                       unsigned long long &cache_idx,
                                       unsigned long long &cache_word) {
  // the shortcut overrides the top row first: with a single-row matrix that
  // row is row 0 (dtw.hpp:105-108 runs before the row-0 loop)
  if (shortcut && r == g.m - 1 && c >= shortcut) return kMoveOpenRight;
  if (r == 0) {
    if (c == 0) return a.os ? kMoveNilOpenRight : kMaxMoveNil;
    return a.os ? kMoveOpenRight : kMoveRight;
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
  if (code == kMoveRight && a.oe && r == g.m - 1) return kMoveOpenRight;
  return code;
}

template <typename T>
__global__ void backtrack_kernel(RoundArgs<T> a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.n) return;
  const MemberGeom g = member_geom<T>(a.lens[k], a.Lc, a.os, a.oe);
  const unsigned long long *w = a.words + a.path_off[k];
  const int shortcut = a.shortcut[k];
  int2 *rg = a.ranges + (unsigned long long)k * a.Lc;
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
  int mv = move_at<T>(a, g, w, shortcut, r, c, cache_idx, cache_word);
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
    mv = move_at<T>(a, g, w, shortcut, r, c, cache_idx, cache_word);
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

template <typename T>
__global__ void reduce_kernel(RoundArgs<T> a, double *block_max) {
  __shared__ double smax[256];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double dl = 0.0;
  if (t < a.Lc) {
    T sum = T(0);
    uint32_t cnt = 0;
    for (int k = 0; k < a.n; ++k) {
      const int2 r = a.ranges[(unsigned long long)k * a.Lc + t];
      if (r.y < r.x) continue;
      const T *seq = a.series + a.offsets[k];
      for (int i = r.y; i >= r.x; --i) sum = add_rn(sum, seq[i]);
      cnt += uint32_t(r.y - r.x + 1);
    }
    const T mean = cnt ? div_rn<T>(sum, T(cnt)) : host_default_nan<T>();
    a.mean[t] = mean;
    a.counts[t] = cnt;
    const double d = fabs(double(a.centroid[t] - mean));
    dl = d > 0.0 ? d : 0.0;  // NaN never raises the maximum (dba.hpp:833)
  }
  smax[threadIdx.x] = dl;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && smax[threadIdx.x + s] > smax[threadIdx.x])
      smax[threadIdx.x] = smax[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) block_max[blockIdx.x] = smax[0];
}

__global__ void final_max_kernel(const double *block_max, int nb, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = 0.0;
  for (int i = 0; i < nb; ++i) m = block_max[i] > m ? block_max[i] : m;
  *out = m;
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
  size_t off_counter, off_path, off_trip, off_short, off_ranges, off_blockmax, off_edges, off_words,
      total;
  unsigned long long edge_stride;
};

template <typename T>
RoundLayout round_layout(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe) {
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  unsigned long long words = 0, maxm = Lc;
  for (int k = 0; k < n; ++k) {
    const MemberGeom g = member_geom<T>(h_lens[k], Lc, os, oe);
    words += g.words;
    if ((unsigned long long)g.m > maxm) maxm = g.m;
  }
  RoundLayout L;
  L.edge_stride = (maxm + 32 + 31) / 32 * 32;
  const size_t slots = size_t(round_grid<T>()) * kRoundWarps;
  const int nb = int((Lc + 255) / 256);
  size_t o = 0;
  L.off_counter = o; o += 256;
  L.off_path = o; o += up(size_t(n) * 8);
  L.off_trip = o; o += up(size_t(n) * 8);
  L.off_short = o; o += up(size_t(n) * 4);
  L.off_ranges = o; o += up(size_t(n) * Lc * sizeof(int2));
  L.off_blockmax = o; o += up(size_t(nb) * 8);
  L.off_edges = o; o += up(slots * 2 * L.edge_stride * sizeof(T));
  L.off_words = o; o += up(words * 8);
  L.total = o;
  return L;
}

}  // namespace

template <typename T>
size_t dba_round_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe) {
  return round_layout<T>(h_lens, n, Lc, os, oe).total;
}

template <typename T>
int dba_round_launch(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                     const uint64_t *lens, const uint64_t *h_lens, int n, int os, int oe, T *mean,
                     uint32_t *counts, double *delta, int32_t *triples, int64_t *triple_counts,
                     void *ws, size_t ws_bytes, cudaStream_t stream) {
  const RoundLayout L = round_layout<T>(h_lens, n, Lc, os, oe);
  if (ws_bytes < L.total) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "DBA round workspace too small");
  char *base = static_cast<char *>(ws);
  RoundArgs<T> a;
  a.centroid = centroid;
  a.Lc = int(Lc);
  a.series = series;
  a.offsets = offsets;
  a.lens = lens;
  a.n = n;
  a.os = os ? 1 : 0;
  a.oe = oe ? 1 : 0;
  a.counter = reinterpret_cast<unsigned long long *>(base + L.off_counter);
  a.path_off = reinterpret_cast<unsigned long long *>(base + L.off_path);
  a.trip_off = reinterpret_cast<unsigned long long *>(base + L.off_trip);
  a.shortcut = reinterpret_cast<int *>(base + L.off_short);
  a.ranges = reinterpret_cast<int2 *>(base + L.off_ranges);
  a.edges = reinterpret_cast<T *>(base + L.off_edges);
  a.edge_stride = L.edge_stride;
  a.words = reinterpret_cast<unsigned long long *>(base + L.off_words);
  a.mean = mean;
  a.counts = counts;
  a.delta = delta;
  a.triples = triples;
  a.triple_counts = triple_counts;
  double *bmax = reinterpret_cast<double *>(base + L.off_blockmax);
  const int nb = int((Lc + 255) / 256);
  cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), stream);
  plan_kernel<T><<<1, 32, 0, stream>>>(a);
  const unsigned long long nr = (unsigned long long)n * Lc;
  fill_ranges_kernel<<<nr > 0 ? int((nr + 255) / 256 < 4096 ? (nr + 255) / 256 : 4096) : 1, 256, 0,
                       stream>>>(a.ranges, nr);
  path_dtw_kernel<T, PathTune<T>::RF, PathTune<T>::RQ>
      <<<round_grid<T>(), kRoundWarps * 32, 0, stream>>>(a);
  backtrack_kernel<T><<<(n + 127) / 128, 128, 0, stream>>>(a);
  reduce_kernel<T><<<nb, 256, 0, stream>>>(a, bmax);
  final_max_kernel<<<1, 32, 0, stream>>>(bmax, nb, delta);
  return check_launch("DBA round kernels");
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

}  // namespace odba
