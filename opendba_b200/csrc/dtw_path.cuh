// Path-recording variant of the swath sweep in dtw_device.cuh, for the DBA
// round (DBAUpdate's DTWDistance launches with a path matrix, dba.hpp:589-617).
//
// Each cell also records the reference's move choice (dtw.hpp:202-227):
//   if (diag > up) move = (up > right) ? RIGHT : UP
//   else           move = (diag > right) ? RIGHT : DIAGONAL
// over the three candidate costs rounded separately (fma(d, d, pred), or the
// free predecessor on the open-end top row).  Ties therefore resolve
// DIAGONAL > UP > RIGHT, i.e. move = DIAGONAL if diag == min, else UP if
// up == min, else RIGHT.  Two bits per cell are kept as two bit planes: D
// (the diagonal candidate equals the minimum) and U (the up candidate does),
// each set by one compare and one predicated OR of an immediate; decode_move
// applies the priority.  The codes the reference derives from position alone
// (row 0, (0, 0), the open-end OPEN_RIGHT) are rebuilt by the backtrack.
//
// Path layout per swath: step t, lane l, row slot s (0 = row a, 1 = row b)
// at 64-bit word ((t * 32 + l) * 2 + s); bit j holds register j's D bit and
// bit 32 + j its U bit.  A warp writes 512 contiguous bytes per step.
#pragma once

#include "dtw_device.cuh"

namespace odba {

// Swath hand-off of the path sweep.  The next swath's warp can run no closer
// behind this one than the rows it must see published: lane 31 publishes
// every kPathPublishSteps steps, and lane 0's rows of chunk c + 1 are gated
// and copied kPathIssueStep steps into chunk c (a chunk is 32 steps), which
// leaves 32 - kPathIssueStep steps for the copies to land.  A member's
// swaths form a chain, so the lag per hand-off adds up over its swaths.
constexpr int kPathPublishSteps = 16;
constexpr int kPathIssueStep = 24;
static_assert(kPathIssueStep >= 0 && kPathIssueStep < 31, "chunk c + 1 is issued inside chunk c");

// Sets bit J of w if a == b: one compare and one predicated OR of an
// immediate (no select, no shifted constant in a register).
template <int J>
__device__ __forceinline__ void or_bit_if_eq(unsigned &w, float a, float b) {
  asm("{\n\t.reg .pred p;\n\tsetp.eq.f32 p, %1, %2;\n\t@p or.b32 %0, %0, %3;\n\t}"
      : "+r"(w)
      : "f"(a), "f"(b), "n"(1u << J));
}
template <int J>
__device__ __forceinline__ void or_bit_if_eq(unsigned &w, double a, double b) {
  asm("{\n\t.reg .pred p;\n\tsetp.eq.f64 p, %1, %2;\n\t@p or.b32 %0, %0, %3;\n\t}"
      : "+r"(w)
      : "d"(a), "d"(b), "n"(1u << J));
}

// Move codes the sweep records (dtw.hpp:10-16).
constexpr int kMoveDiag = 1, kMoveRight = 2, kMoveUp = 3;

// The move of register j from its step word (DIAGONAL > UP > RIGHT).
__device__ __forceinline__ int decode_move(unsigned long long w, int j) {
  if ((w >> j) & 1ull) return kMoveDiag;
  return ((w >> (32 + j)) & 1ull) ? kMoveUp : kMoveRight;
}

// One cell with its move bits.  top: open-end top row (right free); fd: the
// reference's swath-left column on that row (diagonal free too).
template <typename T, bool MASKED, int J>
__device__ __forceinline__ T path_cell(T d, T up, T diag, T left, bool top, bool fd, unsigned &pd,
                                       unsigned &pu) {
  const T uv = Num<T>::cell(d, up);
  T dv = Num<T>::cell(d, diag);
  T rv = Num<T>::cell(d, left);
  if (MASKED) {
    rv = top ? left : rv;
    dv = (top && fd) ? diag : dv;
  }
  const T v = Num<T>::min3(uv, dv, rv);
  or_bit_if_eq<J>(pd, dv, v);
  or_bit_if_eq<J>(pu, uv, v);
  return v;
}

template <typename T, int R, bool MASKED, int J = 0>
struct PathCols {
  // Column J of one step: the cells of rows a and b.
  static __device__ __forceinline__ void run(T (&col)[R], const YCols<T, R> &yv,
                                             RowDiffs<T, R> &df, T &a_left, T &a_diag, T &b_left,
                                             T &b_diag, bool act_a, bool act_b, bool top_a,
                                             bool top_b, bool fd0, unsigned &da, unsigned &ua,
                                             unsigned &db, unsigned &ub) {
    if constexpr (J < R) {
      const T up = col[J];
      T va = path_cell<T, MASKED, J>(df.a(yv, J), up, a_diag, a_left, top_a,
                                     J == 0 && fd0, da, ua);
      if (MASKED) va = act_a ? va : up;
      a_diag = up;
      a_left = va;
      T vb = path_cell<T, MASKED, J>(df.b(yv, J), va, b_diag, b_left, top_b,
                                     J == 0 && fd0, db, ub);
      if (MASKED) vb = act_b ? vb : va;
      b_diag = va;
      b_left = vb;
      col[J] = vb;
      PathCols<T, R, MASKED, J + 1>::run(col, yv, df, a_left, a_diag, b_left, b_diag, act_a,
                                         act_b, top_a, top_b, fd0, da, ua, db, ub);
    }
  }
};

template <typename T, int R, bool MASKED>
__device__ __forceinline__ T step_rows2_path(T (&col)[R], const YCols<T, R> &yv, T xa, T xb, T la,
                                             T lb, T dg, bool act_a, bool act_b, bool top_a,
                                             bool top_b, bool fd0, unsigned long long &wa,
                                             unsigned long long &wb) {
  T a_left = la, a_diag = dg;
  T b_left = lb, b_diag = la;
  unsigned da = 0u, ua = 0u, db = 0u, ub = 0u;
  RowDiffs<T, R> df(xa, xb);
  PathCols<T, R, MASKED, 0>::run(col, yv, df, a_left, a_diag, b_left, b_diag, act_a, act_b,
                                 top_a, top_b, fd0, da, ua, db, ub);
  wa = (unsigned long long)da | ((unsigned long long)ua << 32);
  wb = (unsigned long long)db | ((unsigned long long)ub << 32);
  return a_left;
}

// The unmasked path step in skewed order (see step_rows2_steady in
// dtw_device.cuh): row b's cell of column J - 1 after row a's cell of column
// J, so each new col value can take the register of the old one.
template <typename T, int R, int J>
struct PathColsSkew {
  static __device__ __forceinline__ void run(T (&col)[R], const YCols<T, R> &yv,
                                             RowDiffs<T, R> &df, T &a_left, T &a_diag, T &b_left,
                                             T &b_diag, T &va_prev, unsigned &da, unsigned &ua,
                                             unsigned &db, unsigned &ub) {
    if constexpr (J < R) {
      const T up = col[J];
      const T va =
          path_cell<T, false, J>(df.a(yv, J), up, a_diag, a_left, false, false, da, ua);
      a_diag = up;
      a_left = va;
      const T vb = path_cell<T, false, J - 1>(df.b(yv, J - 1), va_prev, b_diag, b_left,
                                              false, false, db, ub);
      b_diag = va_prev;
      b_left = vb;
      col[J - 1] = vb;
      va_prev = va;
      PathColsSkew<T, R, J + 1>::run(col, yv, df, a_left, a_diag, b_left, b_diag, va_prev, da, ua,
                                     db, ub);
    }
  }
};

template <typename T, int R>
__device__ __forceinline__ T step_rows2_path_steady(T (&col)[R], const YCols<T, R> &yv, T xa,
                                                    T xb, T la, T lb, T dg,
                                                    unsigned long long &wa,
                                                    unsigned long long &wb) {
  T a_left = la, a_diag = dg;
  T b_left = lb, b_diag = la;
  unsigned da = 0u, ua = 0u, db = 0u, ub = 0u;
  RowDiffs<T, R> df(xa, xb);
  T va_prev;
  {
    const T up = col[0];
    va_prev = path_cell<T, false, 0>(df.a(yv, 0), up, a_diag, a_left, false, false, da, ua);
    a_diag = up;
    a_left = va_prev;
  }
  PathColsSkew<T, R, 1>::run(col, yv, df, a_left, a_diag, b_left, b_diag, va_prev, da, ua, db, ub);
  col[R - 1] = path_cell<T, false, R - 1>(df.b(yv, R - 1), va_prev, b_diag, b_left, false,
                                          false, db, ub);
  wa = (unsigned long long)da | ((unsigned long long)ua << 32);
  wb = (unsigned long long)db | ((unsigned long long)ub << 32);
  return a_left;
}

struct PathOut {
  unsigned long long *words;  // this swath's move words, (steps * 32 * 2) of them
  bool track_min;             // record min / top of this swath's right-edge column
};

// A tile of a swath (stripe-mode recompute): rows [job.r0, job.m) only, the
// row below the tile given by col_init (this lane's R columns start at
// col_init + lane * R), and the open-end top row at top_row.  top_left, if
// set, replaces the left-edge value of the top row (the recomputed top row of
// the swath to the left, where that row is not the matrix's last).  The
// default is a whole swath: col_init null (the boundary row), top_row =
// job.m - 1, the stored left edge throughout.
template <typename T>
struct TileIn {
  const T *col_init;
  int top_row;
  const T *top_left = nullptr;
  // a band of a swath handing its last row to the band above: this lane's R
  // columns at row_out + lane * R, and (with a left edge) the edge's value
  // on that row, the next band's corner, at corner_out
  T *row_out = nullptr;
  T *corner_out = nullptr;
};

// Sweeps one swath recording moves.  Same wavefront as sweep_swath; in
// addition lane 31 keeps the minimum of the right-edge column it spills over
// the rows ShortcutRows selects, and its top-row value (for the reference's
// open-end shortcut, dtw.hpp:74-129).
template <typename T, int R, typename Gate = NoGate>
__device__ __forceinline__ void sweep_swath_path(const SwathJob<T> &job, const PathOut &po,
                                                 T (&col)[R], T &edge_min, T &edge_top,
                                                 TileIn<T> tile = TileIn<T>{nullptr, -1},
                                                 Gate gate = Gate()) {
  const int lane = threadIdx.x & 31;
  const int m = job.m;
  const int r0 = job.r0;
  YCols<T, R> yv;
  yv.load(job.y, job.c0 + lane * R, job.n);
  const T init = r0 ? T(0) : Num<T>::big();
  if (tile.col_init) {
    const T *src = tile.col_init + lane * R;
#pragma unroll
    for (int j = 0; j < R; ++j) col[j] = src[j];
  } else {
#pragma unroll
    for (int j = 0; j < R; ++j) col[j] = init;
  }
  const int top = tile.top_row >= 0 ? tile.top_row : m - 1;

  const bool has_in = job.edge_in != nullptr;
  const bool has_out = job.edge_out != nullptr;
  const int rows = m - r0;
  const int total = (rows + 1) / 2 + 31;
  const bool lane0 = lane == 0, lane31 = lane == 31;
  const bool oe_top = job.open_end && top >= 1;
  const bool fd0 = job.free_diag0 && lane0;
  const int last_x = m - 1, last_e = rows > 0 ? rows - 1 : 0;
  T emin = Num<T>::big(), etop = Num<T>::big();

  T xa_cur = T(0), xb_cur = T(0), a_last = init;
  T dg = lane0 ? job.corner_init : init;
  const T top_left = (tile.top_left && lane0) ? *tile.top_left : T(0);

  auto fetch = [&](int t, T &xa, T &xb, T &ea, T &eb) {
    const int k = 2 * t;
    const int ka = k < last_e ? k : last_e, kb = k + 1 < last_e ? k + 1 : last_e;
    const int ia = r0 + k < last_x ? r0 + k : last_x;
    const int ib = r0 + k + 1 < last_x ? r0 + k + 1 : last_x;
    xa = job.x[ia];
    xb = job.x[ib];
    if (has_in) {
      if (Gate::kActive) gate.wait_in(rows > 0 ? kb + 1 : 0);
      ea = job.edge_in[ka];
      eb = job.edge_in[kb];
      if (tile.top_left) {
        // the top row is the tile's last, always in the masked drain
        if (r0 + k == top) ea = top_left;
        if (r0 + k + 1 == top) eb = top_left;
      }
    } else {
      ea = eb = Num<T>::big();
    }
  };

  // rows outside [r0, m) are not stored: in a tile they belong to a
  // neighbouring tile
  auto store_words = [&](int t, unsigned long long wa, unsigned long long wb, bool act_a,
                         bool act_b) {
    if (act_a && act_b) {
      ulonglong2 w;
      w.x = wa;
      w.y = wb;
      reinterpret_cast<ulonglong2 *>(po.words)[t * 32 + lane] = w;
    } else {
      if (act_a) po.words[(size_t(t) * 32 + lane) * 2] = wa;
      if (act_b) po.words[(size_t(t) * 32 + lane) * 2 + 1] = wb;
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
    unsigned long long wa, wb;
    a_last = step_rows2_path<T, R, true>(col, yv, xa, xb, la, lb, diag, act_a, act_b,
                                         oe_top && ra == top, oe_top && ra + 1 == top, fd0, wa, wb);
    xa_cur = xa;
    xb_cur = xb;
    store_words(t, wa, wb, act_a, act_b);
    if (lane31) {
      if (act_a) {
        if (has_out) job.edge_out[ra - r0] = a_last;
        if (shortcut_row<T>(ra)) emin = Num<T>::min2(emin, a_last);
        if (ra == top) etop = a_last;
      }
      if (act_b) {
        if (has_out) job.edge_out[ra + 1 - r0] = col[R - 1];
        if (shortcut_row<T>(ra + 1)) emin = Num<T>::min2(emin, col[R - 1]);
        if (ra + 1 == top) etop = col[R - 1];
      }
    }
  };

  // Steady state as in sweep_swath: lane 0's rows staged in shared memory one
  // 64-row chunk ahead by the whole warp (cp.async), no masks, no top row.
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
  auto staged = [&](int u, T &xa, T &xb, T &ea, T &eb) {
    using V2 = typename Pair2<T>::V;
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

  int steady_end = (rows - 1) / 2;  // first step at which lane 0's row b reaches the last row
  if (steady_end < 31) steady_end = 31;
  const int fill_end = total < 31 ? total : 31;
  int t = 0;
  for (; t < fill_end; ++t) masked_step(t);
  if (t < steady_end) {
    using V2 = typename Pair2<T>::V;
    const int cfirst = t >> 5;
    gate_chunk(cfirst + 1);
    __syncwarp();
    issue_chunk(cfirst);
    issue_chunk(cfirst + 1);
    cp_async_wait_all();
    __syncwarp();
    T pxa = T(0), pxb = T(0), pea = T(0), peb = T(0);
    if (lane0) staged(t, pxa, pxb, pea, peb);
    int issued = cfirst + 1;  // the last chunk copied
    for (; t < steady_end; ++t) {
      T xa = __shfl_up_sync(kFull, xa_cur, 1);
      T xb = __shfl_up_sync(kFull, xb_cur, 1);
      T la = __shfl_up_sync(kFull, a_last, 1);
      T lb = __shfl_up_sync(kFull, col[R - 1], 1);
      if ((t & 31) == kPathIssueStep && (t >> 5) + 1 > issued) {
        // chunk t / 32 + 1 into the slot chunk t / 32 - 1 left (read by
        // lane 0 before this step; the gate's __syncwarp orders those reads
        // before the copies)
        issued = (t >> 5) + 1;
        gate_chunk(issued);
        __syncwarp();
        issue_chunk(issued);
      }
      if (((t + 1) & 31) == 0) {
        // chunk (t + 1) / 32 landed, for lane 0's read of step t + 1 below
        cp_async_wait_all();
        __syncwarp();
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
      unsigned long long wa, wb;
      a_last = step_rows2_path_steady<T, R>(col, yv, xa, xb, la, lb, diag, wa, wb);
      xa_cur = xa;
      xb_cur = xb;
      ulonglong2 w;
      w.x = wa;
      w.y = wb;
      reinterpret_cast<ulonglong2 *>(po.words)[t * 32 + lane] = w;
      // lane 31's edge rows and shortcut minimum; the conditions on t are
      // the same in every lane, and the minimum is kept in every lane (only
      // lane 31's is read)
      if (has_out) {
        if (lane31) {
          V2 v;
          v.x = a_last;
          v.y = col[R - 1];
          *reinterpret_cast<V2 *>(job.edge_out + 2 * (t - 31)) = v;
        }
        if (Gate::kActive && ((t - 31) % kPathPublishSteps) == kPathPublishSteps - 1 && lane31)
          gate.publish(2 * (t - 31) + 2);
      }
      const int ra = r0 + 2 * (t - 31);
      if (shortcut_row<T>(ra)) emin = Num<T>::min2(emin, a_last);
      if (shortcut_row<T>(ra + 1)) emin = Num<T>::min2(emin, col[R - 1]);
    }
    // the next swath reuses the slots: no copy may still be in flight
    cp_async_wait_all();
    __syncwarp();
  }
  for (; t < total; ++t) masked_step(t);
  if (Gate::kActive && lane31 && has_out) gate.publish(rows);
  if (tile.row_out) {
    T *dst = tile.row_out + lane * R;
#pragma unroll
    for (int j = 0; j < R; ++j) dst[j] = col[j];
  }
  // lane 0's last fetch read the left edge's last row (clamped to it)
  if (tile.corner_out && has_in && lane0) *tile.corner_out = dg;
  edge_min = __shfl_sync(kFull, emin, 31);
  edge_top = __shfl_sync(kFull, etop, 31);
}

}  // namespace odba
