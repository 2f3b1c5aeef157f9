// Device-side DTW engine for sm_100a: one warp sweeps one vertical swath of
// the cost matrix with an anti-diagonal wavefront carried by __shfl_sync.
//
// Matrix convention (the reference's, dtw.hpp:35-42): rows r in [0, m) walk
// the FIRST series x (the Y axis), columns c in [0, n) walk the SECOND series y
// (the X axis).  Cell rule (dtw.hpp:158-239), with d = x[r] - y[c]:
//     C[r][c] = fma(d, d, min(C[r-1][c], C[r][c-1], C[r-1][c-1]))
// The reference's nvcc build fuses "cost + diff*diff" into one fma on sm_100a;
// that choice is pinned against the reference's own GPU outputs.
//
// Layout of one swath in one warp: lane l owns the R consecutive columns
// c0 + l*R + j (j < R), holding y[c] and the running column costs in
// registers.  At step t lane l works on rows ra = r0 + 2(t - l) and ra + 1
// (two interleaved dependency chains), so lane l needs from lane l-1 the costs
// of the same two rows one column to the left (produced one step earlier) --
// shuffles carry them, with the two x values.  The swath's left edge is
// read from the previous swath's spilled right-edge column, the right edge is
// spilled for the next swath.  With R = 32 a float swath is exactly the
// reference's 1024-column swath, so the reference's swath-dependent open-end
// rule (a free diagonal at columns c % 1024 == 0, dtw.hpp:172-186) lands on
// lane 0 / register 0.
#pragma once

#include <cfloat>
#include <cstdint>

namespace odba {

constexpr int kRefSwath = 1024;  // blockDim.x of every reference DTWDistance launch
constexpr unsigned kFull = 0xffffffffu;

// The reference's open-end shortcut (dtw.hpp:74-129) compares the swath's
// left-edge value on the last row with a minimum that warp 0 reduces and all
// 32 of its lanes store to one shared word (dtw.hpp:97-105); lane l's partial
// minimum covers the rows r with r % 1024 >= 32*l.  On the B200 the float
// build's check reads lane 0's store (all rows), the double build's lane 16's
// (rows with r % 1024 >= 512), as its own open-end and stripe-mode runs show.
template <typename T>
struct ShortcutRows;
template <>
struct ShortcutRows<float> {
  static constexpr int floor = 0;
};
template <>
struct ShortcutRows<double> {
  static constexpr int floor = 512;
};
template <typename T>
__host__ __device__ inline bool shortcut_row(int r) {
  return (r & (kRefSwath - 1)) >= ShortcutRows<T>::floor;
}

template <typename T>
struct Num;
template <>
struct Num<float> {
  // "max" sentinel of the reference (limits.hpp:40-43) for absent predecessors
  static __device__ __forceinline__ float big() { return FLT_MAX; }
  static __device__ __forceinline__ float quiet_nan() { return __int_as_float(0x7fc00000); }
  static __device__ __forceinline__ float cell(float d, float m) { return __fmaf_rn(d, d, m); }
  static __device__ __forceinline__ float min2(float a, float b) { return fminf(a, b); }
  static __device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
  }
};
// Costs are never NaN and never -0 (they start at +0 or d*d and only grow), so
// a compare-and-select minimum gives the same bits as fmin without fmin's NaN
// handling, which costs several extra instructions per call in double.
template <>
struct Num<double> {
  static __device__ __forceinline__ double big() { return DBL_MAX; }
  static __device__ __forceinline__ double quiet_nan() {
    return __longlong_as_double(0x7ff8000000000000ll);
  }
  static __device__ __forceinline__ double cell(double d, double m) { return __fma_rn(d, d, m); }
  static __device__ __forceinline__ double min2(double a, double b) { return b < a ? b : a; }
  static __device__ __forceinline__ double min3(double a, double b, double c) {
    return min2(min2(a, b), c);
  }
};

// Inputs of one swath sweep for one pair.
template <typename T>
struct SwathJob {
  const T *x;         // first series (rows), length m
  const T *y;         // second series (columns), length n
  int m, n;
  int c0;             // first column of this swath
  int r0;             // first computed row: 0, or 1 with open start (row 0 is all zeros)
  const T *edge_in;   // C[r][c0-1] for r in [r0, m), or nullptr for the first swath
  T *edge_out;        // receives C[r][c_last] for r in [r0, m), or nullptr
  bool open_end;
  bool free_diag0;    // column c0 is a reference swath-left column (c0 % 1024 == 0, c0 > 0)
  bool track = false;  // keep the right edge's shortcut minimum and last-row value (EdgeStat)
  T corner_init;      // diagonal input of lane 0 at its first row
  T *stage;           // this warp's kStageElems elements of shared memory
};

// The right-edge column's open-end shortcut figures (valid in lane 31 when the
// job tracks them): the minimum over the rows ShortcutRows selects and the
// value on the last row.
template <typename T>
struct EdgeStat {
  T emin, etop;
};

// Staging of lane 0's row inputs: in the steady state the whole warp copies
// the x values and left-edge costs of the next 64 rows (one chunk, 32 steps)
// into shared memory with cp.async, one chunk ahead, so that lane 0 reads
// them from shared memory instead of waiting on L2.  Two slots of
// [x[64] | edge[64]] per warp.
constexpr int kChunkRows = 64;
constexpr int kStageElems = 2 * 2 * kChunkRows;

__device__ __forceinline__ void cp_async_elem(void *smem, const void *gmem, int bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// A lane's column values y[c] of the swath, and the differences x - y[c] of
// a step's two rows.  For float the values are kept as packed pairs of
// adjacent columns, and one sub.rn.f32x2 gives the differences of two
// columns (each half rounds as sub.rn.f32, so the bits are those of x - y).
// The differences of a row must be asked for in increasing column order, in
// fully unrolled code (the column index is then a constant).
template <typename T, int R>
struct YCols {
  T v[R];
  __device__ __forceinline__ void load(const T *y, int c, int n) {
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = (c + j < n) ? y[c + j] : T(0);
  }
  __device__ __forceinline__ T get(int j) const { return v[j]; }
};
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
template <int H>
__device__ __forceinline__ float half_f32x2(unsigned long long p) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(p));
  return H ? hi : lo;
}
__device__ __forceinline__ unsigned long long sub_f32x2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
template <int R>
struct YCols<float, R> {
  static_assert(R % 2 == 0, "columns come in pairs");
  unsigned long long p[R / 2];
  __device__ __forceinline__ void load(const float *y, int c, int n) {
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
      const int j = c + 2 * i;
      p[i] = pack_f32x2(j < n ? y[j] : 0.f, j + 1 < n ? y[j + 1] : 0.f);
    }
  }
  __device__ __forceinline__ float get(int j) const {
    return (j & 1) ? half_f32x2<1>(p[j / 2]) : half_f32x2<0>(p[j / 2]);
  }
};

template <typename T, int R>
struct RowDiffs {
  T xa, xb;
  __device__ __forceinline__ RowDiffs(T a, T b) : xa(a), xb(b) {}
  __device__ __forceinline__ T a(const YCols<T, R> &y, int j) const { return xa - y.get(j); }
  __device__ __forceinline__ T b(const YCols<T, R> &y, int j) const { return xb - y.get(j); }
};
template <int R>
struct RowDiffs<float, R> {
  unsigned long long xa2, xb2, pa = 0, pb = 0;  // pa, pb: the row's current column pair
  __device__ __forceinline__ RowDiffs(float a, float b)
      : xa2(pack_f32x2(a, a)), xb2(pack_f32x2(b, b)) {}
  __device__ __forceinline__ float a(const YCols<float, R> &y, int j) {
    if ((j & 1) == 0) pa = sub_f32x2(xa2, y.p[j / 2]);
    return (j & 1) ? half_f32x2<1>(pa) : half_f32x2<0>(pa);
  }
  __device__ __forceinline__ float b(const YCols<float, R> &y, int j) {
    if ((j & 1) == 0) pb = sub_f32x2(xb2, y.p[j / 2]);
    return (j & 1) ? half_f32x2<1>(pb) : half_f32x2<0>(pb);
  }
};

// One cell: the open-end top-row rule when TOP (the right move is free,
// dtw.hpp:196-200; at a reference swath-left column the diagonal is free too,
// dtw.hpp:179-185), the White-Neely cost otherwise.
template <typename T>
__device__ __forceinline__ T cell_rule(T d, T up, T diag, T left, bool top, bool fd) {
  const T v = Num<T>::cell(d, Num<T>::min3(up, diag, left));
  const T vt = fd ? Num<T>::min3(Num<T>::cell(d, up), diag, left)
                  : Num<T>::min2(Num<T>::cell(d, Num<T>::min2(up, diag)), left);
  return top ? vt : v;
}

// Two rows per step for one lane: row a = ra and row b = ra + 1, row b one
// column behind row a, so that the two dependency chains (left to right within
// a row) interleave.  col[j] holds C[ra-1][c_j] on entry and C[ra+1][c_j] on
// exit.  la / lb: costs of rows a / b one column left of the lane's first
// column; dg: cost of row a-1 there.  Returns C[ra][c_last] (row a's last
// column, needed by the next lane).  MASKED steps may hold lanes outside
// [r0, m); with TOP they may also hold the open-end top row (top_a / top_b),
// without it the caller guarantees they do not (no open end in this sweep).
template <typename T, int R, bool MASKED, bool TOP = true>
__device__ __forceinline__ T step_rows2(T (&col)[R], const YCols<T, R> &yv, T xa, T xb, T la,
                                        T lb, T dg, bool act_a, bool act_b, bool top_a,
                                        bool top_b, bool fd0) {
  T a_left = la, a_diag = dg;
  T b_left = lb, b_diag = la;
  RowDiffs<T, R> df(xa, xb);
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const T up = col[j];
    const T da = df.a(yv, j);
    T va;
    if (MASKED && TOP) {
      va = cell_rule<T>(da, up, a_diag, a_left, top_a, j == 0 && fd0);
      va = act_a ? va : up;
    } else if (MASKED) {
      va = Num<T>::cell(da, Num<T>::min3(up, a_diag, a_left));
      va = act_a ? va : up;
    } else {
      va = Num<T>::cell(da, Num<T>::min3(up, a_diag, a_left));
    }
    a_diag = up;
    a_left = va;
    const T db = df.b(yv, j);
    T vb;
    if (MASKED && TOP) {
      vb = cell_rule<T>(db, va, b_diag, b_left, top_b, j == 0 && fd0);
      vb = act_b ? vb : va;
    } else if (MASKED) {
      vb = Num<T>::cell(db, Num<T>::min3(va, b_diag, b_left));
      vb = act_b ? vb : va;
    } else {
      vb = Num<T>::cell(db, Num<T>::min3(va, b_diag, b_left));
    }
    b_diag = va;
    b_left = vb;
    col[j] = vb;
  }
  return a_left;
}

// The unmasked step of step_rows2 in skewed order: row b's cell of column
// j - 1 comes after row a's cell of column j.  Row a at column j reads
// C[ra-1][c_{j-1}] (the old col[j-1]) as its diagonal, so in this order the
// old col[j-1] is dead before row b writes the new col[j-1], and the new value
// can take the old one's register; in column order every new col[j] would sit
// in the register of its left neighbour and the whole column would rotate back
// at the end of each step.  Same cells, same arithmetic, same results.
template <typename T, int R>
__device__ __forceinline__ T step_rows2_steady(T (&col)[R], const YCols<T, R> &yv, T xa, T xb,
                                               T la, T lb, T dg) {
  T a_left = la, a_diag = dg;
  T b_left = lb, b_diag = la;
  RowDiffs<T, R> df(xa, xb);
  T va_prev;
  {
    const T up = col[0];
    va_prev = Num<T>::cell(df.a(yv, 0), Num<T>::min3(up, a_diag, a_left));
    a_diag = up;
    a_left = va_prev;
  }
#pragma unroll
  for (int j = 1; j < R; ++j) {
    const T up = col[j];
    const T va = Num<T>::cell(df.a(yv, j), Num<T>::min3(up, a_diag, a_left));
    a_diag = up;
    a_left = va;
    const T vb = Num<T>::cell(df.b(yv, j - 1), Num<T>::min3(va_prev, b_diag, b_left));
    b_diag = va_prev;
    b_left = vb;
    col[j - 1] = vb;
    va_prev = va;
  }
  col[R - 1] = Num<T>::cell(df.b(yv, R - 1), Num<T>::min3(va_prev, b_diag, b_left));
  return a_left;
}

template <typename T>
struct Pair2;
template <>
struct Pair2<float> {
  using V = float2;
};
template <>
struct Pair2<double> {
  using V = double2;
};

// Hand-off of swath-edge rows between warps.  NoGate: the edge buffer is the
// warp's own (written by the same warp's previous swath), nothing to wait for.
// A gate with kActive set makes lane 0 call wait_in(k) before it reads edge
// rows [0, k) and lane 31 call publish(k) once rows [0, k) are stored.
struct NoGate {
  static constexpr bool kActive = false;
  __device__ __forceinline__ void wait_in(int) {}
  __device__ __forceinline__ void publish(int) {}
};
constexpr int kPublishSteps = 64;  // lane 31 publishes every 64 steps (128 rows)

// Row checkpoints (the stripe-mode forward pass): the full cost row
// r = r0 + k*K - 1 (k >= 1, K = 2^shift >= 2) of this swath's columns is
// stored at q + (k - 1) * stride + (c - c0) -- q points at this swath's first
// column.  K is even, so these rows are always the second row of a lane's
// step pair.
template <typename T>
struct CkptOut {
  T *q;
  unsigned long long stride;
  int shift;
};

// Sweeps one swath.  On return col[] holds, per lane, the costs of the last
// row m-1 at the lane's columns.  Swath-edge buffers are indexed by r - r0,
// two rows per 8/16-byte access.  Returns the right edge's EdgeStat (lane 31;
// the big value unless TRACK and job.track).
template <typename T, int R, typename Gate = NoGate, bool CKPT = false, bool TRACK = true>
__device__ __forceinline__ EdgeStat<T> sweep_swath(const SwathJob<T> &job, T (&col)[R],
                                                   Gate gate = Gate(),
                                                   CkptOut<T> ckpt = CkptOut<T>{nullptr, 0, 1}) {
  using V2 = typename Pair2<T>::V;
  const int lane = threadIdx.x & 31;
  const int m = job.m;
  const int r0 = job.r0;
  YCols<T, R> yv;
  yv.load(job.y, job.c0 + lane * R, job.n);
  // Row r0 - 1 is the boundary: the virtual row above the matrix (absent,
  // "max") or, with open start, the all-zero row 0.
  const T init = r0 ? T(0) : Num<T>::big();
#pragma unroll
  for (int j = 0; j < R; ++j) col[j] = init;

  const bool has_in = job.edge_in != nullptr;
  const bool has_out = job.edge_out != nullptr;
  const int rows = m - r0;
  const int total = (rows + 1) / 2 + 31;  // wavefront steps including fill and drain
  const bool lane0 = lane == 0, lane31 = lane == 31;
  const bool oe_top = job.open_end && m >= 2;  // a single-row matrix has no open-end rule
  const bool fd0 = job.free_diag0 && lane0;
  const int last_x = m - 1, last_e = rows > 0 ? rows - 1 : 0;

  T xa_cur = T(0), xb_cur = T(0), a_last = init;
  T dg = lane0 ? job.corner_init : init;
  const bool track = TRACK && job.track && lane31;
  EdgeStat<T> st{Num<T>::big(), Num<T>::big()};
  auto note = [&](int r, T v) {
    if (shortcut_row<T>(r)) st.emin = Num<T>::min2(st.emin, v);
    if (r == m - 1) st.etop = v;
  };

  // lane 0's inputs of step t: x of rows a, b and the left-edge costs of rows a, b
  auto fetch = [&](int t, T &xa, T &xb, T &ea, T &eb) {
    const int k = 2 * t;  // ra - r0
    const int ka = k < last_e ? k : last_e, kb = k + 1 < last_e ? k + 1 : last_e;
    const int ia = r0 + k < last_x ? r0 + k : last_x;
    const int ib = r0 + k + 1 < last_x ? r0 + k + 1 : last_x;
    xa = job.x[ia];
    xb = job.x[ib];
    if (has_in) {
      if (Gate::kActive) gate.wait_in(rows > 0 ? kb + 1 : 0);
      ea = job.edge_in[ka];
      eb = job.edge_in[kb];
    } else {
      ea = eb = Num<T>::big();
    }
  };

  auto store_ckpt = [&](int ra) {
    const int kk = ra - r0 + 2;
    if ((kk & ((1 << ckpt.shift) - 1)) == 0) {
      T *dst = ckpt.q + (unsigned long long)((kk >> ckpt.shift) - 1) * ckpt.stride + lane * R;
#pragma unroll
      for (int j = 0; j < R; ++j) dst[j] = col[j];
    }
  };

  auto masked_step = [&](int t) {
    const int ra = r0 + 2 * (t - lane);
    T xa = __shfl_up_sync(kFull, xa_cur, 1);
    T xb = __shfl_up_sync(kFull, xb_cur, 1);
    T la = __shfl_up_sync(kFull, a_last, 1);
    T lb = __shfl_up_sync(kFull, col[R - 1], 1);
    if (lane0) fetch(t, xa, xb, la, lb);
    const T diag = dg;
    dg = lb;
    const bool act_a = ra >= r0 && ra < m, act_b = ra + 1 >= r0 && ra + 1 < m;
    if (oe_top)
      a_last = step_rows2<T, R, true, true>(col, yv, xa, xb, la, lb, diag, act_a, act_b,
                                            ra == m - 1, ra + 1 == m - 1, fd0);
    else
      a_last = step_rows2<T, R, true, false>(col, yv, xa, xb, la, lb, diag, act_a, act_b, false,
                                             false, false);
    xa_cur = xa;
    xb_cur = xb;
    if (lane31 && has_out) {
      if (act_a) job.edge_out[ra - r0] = a_last;
      if (act_b) job.edge_out[ra + 1 - r0] = col[R - 1];
    }
    if (track) {
      if (act_a) note(ra, a_last);
      if (act_b) note(ra + 1, col[R - 1]);
    }
    if (CKPT && act_b) store_ckpt(ra);
  };

  // chunk c of lane 0's rows (k = ra - r0 in [64c, 64c + 64)) into slot c % 2;
  // each lane copies rows 2*lane, 2*lane + 1 of the chunk (clamped like fetch)
  auto issue_chunk = [&](int c) {
    T *slot = job.stage + (c & 1) * (2 * kChunkRows);
    const int k = c * kChunkRows + 2 * lane;
    const int ia = r0 + k < last_x ? r0 + k : last_x;
    const int ib = r0 + k + 1 < last_x ? r0 + k + 1 : last_x;
    cp_async_elem(slot + 2 * lane, job.x + ia, sizeof(T));
    cp_async_elem(slot + 2 * lane + 1, job.x + ib, sizeof(T));
    if (has_in) {
      const int ka = k < last_e ? k : last_e, kb = k + 1 < last_e ? k + 1 : last_e;
      cp_async_elem(slot + kChunkRows + 2 * lane, job.edge_in + ka, sizeof(T));
      cp_async_elem(slot + kChunkRows + 2 * lane + 1, job.edge_in + kb, sizeof(T));
    }
    cp_async_commit();
  };
  // edge rows of chunk c must be published before any lane copies them
  auto gate_chunk = [&](int c) {
    if (Gate::kActive && has_in && lane0) {
      const int need = (c + 1) * kChunkRows;
      gate.wait_in(rows < need ? rows : need);
    }
  };
  // lane 0's staged inputs of step u
  auto staged = [&](int u, T &xa, T &xb, T &ea, T &eb) {
    const T *slot = job.stage + ((u >> 5) & 1) * (2 * kChunkRows);
    const int i = 2 * (u & 31);
    const V2 xv = *reinterpret_cast<const V2 *>(slot + i);
    xa = xv.x;
    xb = xv.y;
    if (has_in) {
      const V2 ev = *reinterpret_cast<const V2 *>(slot + kChunkRows + i);
      ea = ev.x;
      eb = ev.y;
    } else {
      ea = eb = Num<T>::big();
    }
  };

  // steady state: rows a, b of every lane in [r0, m-2]
  int steady_end = (rows - 1) / 2;  // first step at which lane 0's row b reaches m-1
  if (steady_end < 31) steady_end = 31;
  const int fill_end = total < 31 ? total : 31;
  int t = 0;
  for (; t < fill_end; ++t) masked_step(t);
  if (t < steady_end) {
    // chunks of steps t and t + 1 (the same chunk or two consecutive ones)
    const int cfirst = t >> 5;
    gate_chunk(cfirst + 1);
    __syncwarp();
    issue_chunk(cfirst);
    issue_chunk(cfirst + 1);
    cp_async_wait_all();
    __syncwarp();
    T pxa = T(0), pxb = T(0), pea = T(0), peb = T(0);
    if (lane0) staged(t, pxa, pxb, pea, peb);
    for (; t < steady_end; ++t) {
      T xa = __shfl_up_sync(kFull, xa_cur, 1);
      T xb = __shfl_up_sync(kFull, xb_cur, 1);
      T la = __shfl_up_sync(kFull, a_last, 1);
      T lb = __shfl_up_sync(kFull, col[R - 1], 1);
      if (((t + 1) & 31) == 0) {
        // step t + 1 opens chunk c1 (already copied); copy chunk c1 + 1 into
        // the slot of chunk c1 - 1, whose last read was the previous step's
        const int c1 = (t + 1) >> 5;
        cp_async_wait_all();
        gate_chunk(c1 + 1);
        __syncwarp();
        issue_chunk(c1 + 1);
      }
      {
        // lane 0 takes the staged inputs of this step and reads the next
        // step's; every lane reads the same shared words (one broadcast), so
        // no lane branches
        T nxa, nxb, nea, neb;
        staged(t + 1, nxa, nxb, nea, neb);
        xa = lane0 ? pxa : xa;
        xb = lane0 ? pxb : xb;
        la = lane0 ? pea : la;
        lb = lane0 ? peb : lb;
        pxa = nxa;
        pxb = nxb;
        pea = nea;
        peb = neb;
      }
      const T diag = dg;
      dg = lb;
      a_last = step_rows2_steady<T, R>(col, yv, xa, xb, la, lb, diag);
      xa_cur = xa;
      xb_cur = xb;
      if (CKPT) store_ckpt(r0 + 2 * (t - lane));
      if (has_out) {
        if (lane31) {
          V2 v;
          v.x = a_last;
          v.y = col[R - 1];
          *reinterpret_cast<V2 *>(job.edge_out + 2 * (t - 31)) = v;
        }
        if (Gate::kActive && ((t - 31) % kPublishSteps) == kPublishSteps - 1 && lane31)
          gate.publish(2 * (t - 31) + 2);
      }
      if (track) {
        const int ra = r0 + 2 * (t - 31);
        note(ra, a_last);
        note(ra + 1, col[R - 1]);
      }
    }
    // the next swath reuses the slots: no copy may still be in flight
    cp_async_wait_all();
    __syncwarp();
  }
  for (; t < total; ++t) masked_step(t);
  if (Gate::kActive && lane31 && has_out) gate.publish(rows);
  return st;
}

// Reads the cost at absolute column cabs (which must lie in this swath) from
// the lane that owns it; every lane returns the value.
template <typename T, int R>
__device__ __forceinline__ T pick_column(const T (&col)[R], int c0, int cabs) {
  const int rel = cabs - c0;
  const int owner = rel / R, reg = rel - owner * R;
  T v = col[0];
#pragma unroll
  for (int j = 1; j < R; ++j) v = (j == reg) ? col[j] : v;
  return __shfl_sync(kFull, v, owner);
}

}  // namespace odba
