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
// registers.  At step t lane l works on row r = r0 + t - l, so lane l needs
// from lane l-1 the cost of the same row one column to the left (produced one
// step earlier) -- one shuffle per step carries it.  The swath's left edge is
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

template <typename T>
struct Num;
template <>
struct Num<float> {
  // "max" sentinel of the reference (limits.hpp:40-43) for absent predecessors
  static __device__ __forceinline__ float big() { return FLT_MAX; }
  static __device__ __forceinline__ float cell(float d, float m) { return __fmaf_rn(d, d, m); }
  static __device__ __forceinline__ float min2(float a, float b) { return fminf(a, b); }
  static __device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
  }
};
template <>
struct Num<double> {
  static __device__ __forceinline__ double big() { return DBL_MAX; }
  static __device__ __forceinline__ double cell(double d, double m) { return __fma_rn(d, d, m); }
  static __device__ __forceinline__ double min2(double a, double b) { return fmin(a, b); }
  static __device__ __forceinline__ double min3(double a, double b, double c) {
    return fmin(fmin(a, b), c);
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
  T corner_init;      // diagonal input of lane 0 at its first row
};

// One wavefront step for one lane.  col[j] holds C[r-1][c_j] on entry and
// C[r][c_j] on exit.  MASKED steps may hold lanes outside [r0, m) (fill and
// drain of the wavefront) and the top row, where the open-end rules apply.
template <typename T, int R, bool MASKED>
__device__ __forceinline__ void step_cells(T (&col)[R], const T (&yv)[R], T xin, T left, T diag,
                                           bool active, bool top, bool free_diag0) {
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const T up = col[j];
    const T d = xin - yv[j];
    T v = Num<T>::cell(d, Num<T>::min3(up, diag, left));
    if (MASKED) {
      // top row with open end: the right move is free (dtw.hpp:196-200); at a
      // reference swath-left column the diagonal is free too (dtw.hpp:179-185)
      T vt = (j == 0 && free_diag0) ? Num<T>::min3(Num<T>::cell(d, up), diag, left)
                                    : Num<T>::min2(Num<T>::cell(d, Num<T>::min2(up, diag)), left);
      v = top ? vt : v;
      v = active ? v : up;
    }
    diag = up;
    left = v;
    col[j] = v;
  }
}

// Sweeps one swath.  On return col[] holds, per lane, the costs of the last
// row m-1 at the lane's columns (rows beyond m-1 are never applied).
template <typename T, int R>
__device__ __forceinline__ void sweep_swath(const SwathJob<T> &job, T (&col)[R]) {
  const int lane = threadIdx.x & 31;
  const int m = job.m;
  const int r0 = job.r0;
  T yv[R];
  {
    const int cl = job.c0 + lane * R;
#pragma unroll
    for (int j = 0; j < R; ++j) yv[j] = (cl + j < job.n) ? job.y[cl + j] : T(0);
  }
  // Row r0 - 1 is the boundary: the virtual row above the matrix (absent,
  // "max") or, with open start, the all-zero row 0.
  const T init = r0 ? T(0) : Num<T>::big();
#pragma unroll
  for (int j = 0; j < R; ++j) col[j] = init;

  const bool has_in = job.edge_in != nullptr;
  const bool has_out = job.edge_out != nullptr;
  const int total = (m - r0) + 31;  // wavefront steps including fill and drain
  const bool lane0 = lane == 0, lane31 = lane == 31;
  const bool oe_top = job.open_end && m >= 2;  // a single-row matrix has no open-end rule
  const bool fd0 = job.free_diag0 && lane0;

  T xcur = T(0);
  T left_prev = lane0 ? job.corner_init : init;

  auto lane0_inputs = [&](int r, T &x, T &e) {
    const int rc = r < m ? r : m - 1;
    x = job.x[rc];
    e = has_in ? job.edge_in[rc] : Num<T>::big();
  };

  auto masked_step = [&](int t) {
    const int r = r0 + t - lane;
    T xin = __shfl_up_sync(kFull, xcur, 1);
    T lin = __shfl_up_sync(kFull, col[R - 1], 1);
    if (lane0) lane0_inputs(r, xin, lin);
    const T diag = left_prev;
    left_prev = lin;
    xcur = xin;
    const bool active = (r >= r0) && (r < m);
    const bool top = oe_top && (r == m - 1);
    step_cells<T, R, true>(col, yv, xin, lin, diag, active, top, fd0);
    if (lane31 && has_out && active) job.edge_out[r] = col[R - 1];
  };

  const int steady_end = (m - 1 - r0) > 31 ? (m - 1 - r0) : 31;
  const int fill_end = total < 31 ? total : 31;
  int t = 0;
  for (; t < fill_end; ++t) masked_step(t);

  // Steady state: every lane holds a row in [r0, m-2]; no masks, no top row.
  // Lane 0's inputs are prefetched four steps ahead.
  if (t + 4 <= steady_end) {
    T qx[4], qe[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      qx[k] = T(0);
      qe[k] = T(0);
    }
    if (lane0) {
#pragma unroll
      for (int k = 0; k < 4; ++k) lane0_inputs(r0 + t + k, qx[k], qe[k]);
    }
    for (; t + 4 <= steady_end; t += 4) {
      T nx[4], ne[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        nx[k] = T(0);
        ne[k] = T(0);
      }
      if (lane0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) lane0_inputs(r0 + t + 4 + k, nx[k], ne[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        T xin = __shfl_up_sync(kFull, xcur, 1);
        T lin = __shfl_up_sync(kFull, col[R - 1], 1);
        if (lane0) {
          xin = qx[k];
          lin = qe[k];
        }
        const T diag = left_prev;
        left_prev = lin;
        xcur = xin;
        step_cells<T, R, false>(col, yv, xin, lin, diag, true, false, false);
        if (lane31 && has_out) job.edge_out[r0 + t + k - 31] = col[R - 1];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        qx[k] = nx[k];
        qe[k] = ne[k];
      }
    }
  }
  for (; t < total; ++t) masked_step(t);
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
