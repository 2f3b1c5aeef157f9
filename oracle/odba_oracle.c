/* CPU oracle for the OpenDBA hot path -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A restatement in plain C of what the reference computes, used only as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
 * Compiled with -ffp-contract=off so that "fma_mode" alone decides whether a
 * DTW cell is rounded as one fused multiply-add or as a product then a sum.
 *
 * Reference sources followed (paths within the reference project):
 *   DTW cell rule, step pattern, swath quirks   dtw.hpp:131-239
 *   open-end shortcut                           dtw.hpp:74-129
 *   pair distance epilogue                      dtw.hpp:116-125, 242-257
 *   medoid sums of squares and argmin           dba.hpp:186-351
 *   backtrack / centroid pile-up                dba.hpp:374-423
 *   DBA round mean and delta                    dba.hpp:817-836
 *   path file line order                        io_utils.hpp:287-323
 *   stripe-mode round (odba_stripe.inc)         dba.hpp:515-763, dtw.hpp:74-239
 *   z-normalisation                             gpu_utils.hpp:34-170
 */
#include "odba_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <limits.h>
#include <string.h>

/* The reference's swath width: blockDim.x of every DTWDistance launch
 * (maxThreadsPerBlock, cuda_utils.hpp:42-57, forced to 1024 in DBAUpdate at
 * dba.hpp:455-457).  Its open-end rules depend on it (dtw.hpp:74, 172-200). */
#define SWATH 1024

static const int kMoveI[7] = {-1, -1, 0, -1, 0, 0, 0}; /* dtw.hpp:20 */
static const int kMoveJ[7] = {-1, -1, -1, 0, -1, -1, -1}; /* dtw.hpp:21 */

/* The open-end shortcut's column minimum (dtw.hpp:83-105) is read from one
 * shared word that all 32 lanes of warp 0 store their partial minimum to; lane
 * l's partial covers the rows r with r % 1024 >= 32*l.  On the B200 the
 * reference's float build reads lane 0's store (the full minimum) and its
 * double build lane 16's (rows with r % 1024 >= 512), as its stripe-mode and
 * open-end runs show (tests/golden/ref/stripe_*). */
static int g_shortcut_lane[2] = {0, 16}; /* float, double */
#define SHORTCUT_LANE_f32 g_shortcut_lane[0]
#define SHORTCUT_LANE_f64 g_shortcut_lane[1]

void oracle_set_shortcut_lanes(int lane_f32, int lane_f64) {
  g_shortcut_lane[0] = lane_f32;
  g_shortcut_lane[1] = lane_f64;
}

#define DEFINE_ORACLE(T, SFX, FMA, TMAX)                                                        \
  static inline T add_dd_##SFX(T acc, T d, int fma_mode) {                                     \
    if (fma_mode) return FMA(d, d, acc);                                                       \
    T dd = d * d;                                                                              \
    return acc + dd;                                                                           \
  }                                                                                            \
                                                                                               \
  /* Full cost matrix sweep, row by row.  Keeps two rows; optionally stores moves, every    \
   * cost (costs[r*n+c]) and the per-swath-boundary column minima the open-end shortcut      \
   * needs.  Returns C[m-1][n-1]. */                                                           \
  static T sweep_##SFX(const T *first, size_t m, const T *second, size_t n, int os, int oe,     \
                       int fma_mode, unsigned char *path, T *bmin, T *btop, T *costs) {        \
    T *prev = (T *)malloc(sizeof(T) * n);                                                      \
    T *cur = (T *)malloc(sizeof(T) * n);                                                       \
    size_t nb = n / SWATH + 1;                                                                 \
    if (bmin)                                                                                  \
      for (size_t k = 0; k < nb; ++k) bmin[k] = TMAX;                                          \
    for (size_t r = 0; r < m; ++r) {                                                           \
      const T x = first[r];                                                                    \
      for (size_t c = 0; c < n; ++c) {                                                         \
        T d = x - second[c];                                                                   \
        T v;                                                                                   \
        unsigned char mv;                                                                      \
        if (r == 0) {                                                                          \
          /* row 0 is run serially by thread 0 (dtw.hpp:131-156) */                            \
          T left = (c == 0) ? (T)0 : cur[c - 1];                                               \
          v = os ? left : add_dd_##SFX(left, d, fma_mode);                                     \
          mv = (c == 0) ? (os ? ORACLE_NIL_OPEN_RIGHT : ORACLE_NIL)                            \
                        : (os ? ORACLE_OPEN_RIGHT : ORACLE_RIGHT);                             \
        } else {                                                                               \
          T up = add_dd_##SFX(prev[c], d, fma_mode);                                           \
          T right = TMAX, diag = TMAX;                                                         \
          int used_open = 0;                                                                   \
          if (c == 0) {                                                                        \
            /* left edge of the whole matrix: up only (dtw.hpp:172-186) */                     \
          } else if (c % SWATH == 0) {                                                         \
            /* left column of a later swath, fed from the spilled boundary */                  \
            right = cur[c - 1];                                                                \
            diag = prev[c - 1];                                                                \
            if (r < m - 1 || !oe) {                                                            \
              right = add_dd_##SFX(right, d, fma_mode);                                        \
              diag = add_dd_##SFX(diag, d, fma_mode);                                          \
            } else {                                                                           \
              used_open = 1; /* top row, open end: right AND diagonal free */                  \
            }                                                                                  \
          } else {                                                                             \
            right = add_dd_##SFX(cur[c - 1], d, fma_mode);                                     \
            diag = add_dd_##SFX(prev[c - 1], d, fma_mode);                                     \
            if (oe && r == m - 1) {                                                            \
              right = cur[c - 1]; /* top row, open end: right move free (dtw.hpp:196-200) */   \
              used_open = 1;                                                                   \
            }                                                                                  \
          }                                                                                    \
          /* White-Neely selection, tie priority DIAGONAL > UP > RIGHT (dtw.hpp:202-227) */    \
          if (diag > up) {                                                                     \
            if (up > right) {                                                                  \
              v = right;                                                                       \
              mv = used_open ? ORACLE_OPEN_RIGHT : ORACLE_RIGHT;                               \
            } else {                                                                           \
              v = up;                                                                          \
              mv = ORACLE_UP;                                                                  \
            }                                                                                  \
          } else {                                                                             \
            if (diag > right) {                                                                \
              v = right;                                                                       \
              mv = used_open ? ORACLE_OPEN_RIGHT : ORACLE_RIGHT;                               \
            } else {                                                                           \
              v = diag;                                                                        \
              mv = ORACLE_DIAGONAL;                                                            \
            }                                                                                  \
          }                                                                                    \
        }                                                                                      \
        cur[c] = v;                                                                            \
        if (path) path[r * n + c] = mv;                                                        \
        if (costs) costs[r * n + c] = v;                                                       \
        if (bmin && (c + 1) % SWATH == 0) {                                                    \
          size_t k = (c + 1) / SWATH;                                                          \
          if ((r % SWATH) >= (size_t)(32 * SHORTCUT_LANE_##SFX) && v < bmin[k]) bmin[k] = v;   \
          if (r == m - 1) btop[k] = v;                                                         \
        }                                                                                      \
      }                                                                                        \
      T *t = prev;                                                                             \
      prev = cur;                                                                              \
      cur = t;                                                                                 \
    }                                                                                          \
    T last = prev[n - 1];                                                                      \
    free(prev);                                                                                \
    free(cur);                                                                                 \
    return last;                                                                               \
  }                                                                                            \
                                                                                               \
  /* First swath start at which the open-end shortcut fires (dtw.hpp:74-129), or 0. */         \
  static size_t shortcut_col_##SFX(size_t m, size_t n, int os, int oe, const T *bmin,          \
                                   const T *btop) {                                            \
    if (!oe || os) return 0;                                                                   \
    for (size_t c0 = SWATH; c0 < n; c0 += SWATH) {                                             \
      if (c0 <= m) continue;                                                                   \
      size_t k = c0 / SWATH;                                                                   \
      if (btop[k] == bmin[k]) return c0;                                                       \
    }                                                                                          \
    return 0;                                                                                  \
  }                                                                                            \
                                                                                               \
  int oracle_dtw_pair_##SFX(const T *first, size_t m, const T *second, size_t n, int os,       \
                            int oe, int fma_mode, T *dist_out, unsigned char *path) {          \
    if (m == 0 || n == 0) return -1;                                                           \
    size_t nb = n / SWATH + 1;                                                                 \
    T *bmin = (T *)malloc(sizeof(T) * nb);                                                     \
    T *btop = (T *)calloc(nb, sizeof(T));                                                      \
    T last = sweep_##SFX(first, m, second, n, os, oe, fma_mode, path, bmin, btop, NULL);       \
    size_t c0 = shortcut_col_##SFX(m, n, os, oe, bmin, btop);                                  \
    if (path && c0)                                                                            \
      for (size_t c = c0; c < n; ++c) path[(m - 1) * n + c] = ORACLE_OPEN_RIGHT;               \
    const T frozen = c0 ? btop[c0 / SWATH] : (T)0;                                             \
    free(bmin);                                                                                \
    free(btop);                                                                                \
    if (dist_out) {                                                                            \
      /* Where the shortcut fires the distance is the top-row value it freezes (dtw.hpp:113,  \
       * 121): the full sweep's corner when its minimum covers the whole column, but not     \
       * always with the double build's partial minimum; a single-row matrix reads the       \
       * sentinel it has just written. */                                                      \
      if (c0 && m == 1) {                                                                      \
        *dist_out = (T)(sqrtf((float)TMAX) / (float)m);                                        \
      } else if (c0) {                                                                         \
        *dist_out = (T)(sqrtf((float)frozen) / (float)m);                                      \
      } else if ((oe && !os) || (!oe && os)) {                                                 \
        *dist_out = (T)(sqrtf((float)last) / (float)m);                                        \
      } else {                                                                                 \
        *dist_out = (T)sqrtf((float)last);                                                     \
      }                                                                                        \
    }                                                                                          \
    return 0;                                                                                  \
  }                                                                                            \
                                                                                               \
  int oracle_pairwise_##SFX(const T *series, const uint64_t *offsets, const uint64_t *lens,    \
                            int n, int os, int oe, int fma_mode, T *out,                       \
                            const int64_t *pair_list, int64_t n_list, int threads) {           \
    int64_t npairs = (int64_t)n * (n - 1) / 2;                                                 \
    int64_t *row_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));          \
    int64_t *col_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));          \
    int64_t p = 0;                                                                             \
    for (int s = 0; s + 1 < n; ++s)                                                            \
      for (int j = s + 1; j < n; ++j) {                                                        \
        row_of[p] = s;                                                                         \
        col_of[p] = j;                                                                         \
        ++p;                                                                                   \
      }                                                                                        \
    int64_t count = pair_list ? n_list : npairs;                                               \
    if (threads > 0) omp_set_num_threads(threads);                                             \
    _Pragma("omp parallel for schedule(dynamic, 1)") for (int64_t q = 0; q < count; ++q) {     \
      int64_t idx = pair_list ? pair_list[q] : q;                                              \
      int64_t s = row_of[idx], j = col_of[idx];                                                \
      T dv;                                                                                    \
      oracle_dtw_pair_##SFX(series + offsets[s], lens[s], series + offsets[j], lens[j], os,     \
                            oe, fma_mode, &dv, NULL);                                          \
      out[idx] = dv;                                                                           \
    }                                                                                          \
    free(row_of);                                                                              \
    free(col_of);                                                                              \
    return 0;                                                                                  \
  }                                                                                            \
                                                                                               \
  int oracle_medoid_##SFX(const T *dists, int n, const uint64_t *lens, T *sos_out) {           \
    T *sos = (T *)calloc((size_t)n, sizeof(T));                                                \
    size_t off = 0;                                                                            \
    for (int s = 0; s + 1 < n; ++s) {                                                          \
      for (int j = s + 1; j < n; ++j) {                                                        \
        T d = dists[off + (size_t)(j - s - 1)];                                                \
        d = d * d;                                                                             \
        sos[s] = sos[s] + d;                                                                   \
        sos[j] = sos[j] + d;                                                                   \
      }                                                                                        \
      off += (size_t)(n - s - 1);                                                              \
    }                                                                                          \
    int medoid = -1;                                                                           \
    if (n > 2) {                                                                               \
      T lowest = TMAX;                                                                         \
      for (int i = 0; i < n; ++i)                                                              \
        if (sos[i] < lowest) {                                                                 \
          medoid = i;                                                                          \
          lowest = sos[i];                                                                     \
        }                                                                                      \
    } else if (n == 2) {                                                                       \
      medoid = lens[0] > lens[1] ? 0 : 1;                                                      \
    } else if (n == 1) {                                                                       \
      medoid = 0;                                                                              \
    }                                                                                          \
    if (sos_out) memcpy(sos_out, sos, sizeof(T) * (size_t)n);                                  \
    free(sos);                                                                                 \
    return medoid;                                                                             \
  }                                                                                            \
                                                                                               \
  /* Orientation of one member against the centroid (dba.hpp:497-501, 598-616). */             \
  static void orient_##SFX(const T *centroid, size_t Lc, const T *seq, size_t len, int oe,     \
                           const T **first, size_t *m, const T **second, size_t *n,            \
                           int *flip) {                                                        \
    *flip = (oe && Lc < len) ? 1 : 0;                                                          \
    if (*flip) {                                                                               \
      *first = centroid, *m = Lc, *second = seq, *n = len;                                     \
    } else {                                                                                   \
      *first = seq, *m = len, *second = centroid, *n = Lc;                                     \
    }                                                                                          \
  }                                                                                            \
                                                                                               \
  double oracle_dba_update_##SFX(const T *centroid, size_t Lc, const T *series,                \
                                 const uint64_t *offsets, const uint64_t *lens, int n, int os, \
                                 int oe, int fma_mode, T *mean_out, uint32_t *counts_out,      \
                                 T *sums_out) {                                                \
    T *sums = (T *)calloc(Lc, sizeof(T));                                                      \
    uint32_t *counts = (uint32_t *)calloc(Lc, sizeof(uint32_t));                               \
    for (int k = 0; k < n; ++k) {                                                              \
      const T *seq = series + offsets[k];                                                      \
      const T *first, *second;                                                                 \
      size_t m, nn;                                                                            \
      int flip;                                                                                \
      orient_##SFX(centroid, Lc, seq, lens[k], oe, &first, &m, &second, &nn, &flip);           \
      unsigned char *path = (unsigned char *)calloc(m * nn, 1);                                \
      oracle_dtw_pair_##SFX(first, m, second, nn, os, oe, fma_mode, NULL, path);               \
      long i = (long)m - 1, j = (long)nn - 1;                                                  \
      unsigned char mv = path[i * nn + j];                                                     \
      while (j >= 0 && mv != ORACLE_NIL && mv != ORACLE_NIL_OPEN_RIGHT) {                      \
        if (mv != ORACLE_OPEN_RIGHT) {                                                         \
          size_t t = flip ? (size_t)i : (size_t)j;                                             \
          sums[t] = sums[t] + seq[flip ? j : i];                                               \
          counts[t]++;                                                                         \
        }                                                                                      \
        i += kMoveI[mv];                                                                       \
        j += kMoveJ[mv];                                                                       \
        mv = path[i * nn + j];                                                                 \
      }                                                                                        \
      if (mv != ORACLE_NIL_OPEN_RIGHT) {                                                       \
        sums[0] = sums[0] + seq[0];                                                            \
        counts[0]++;                                                                           \
      }                                                                                        \
      free(path);                                                                              \
    }                                                                                          \
    double max_delta = 0.0;                                                                    \
    for (size_t t = 0; t < Lc; ++t) {                                                          \
      T mean = sums[t] / (T)counts[t];                                                         \
      if (mean_out) mean_out[t] = mean;                                                        \
      double delta = fabs((double)(centroid[t] - mean));                                       \
      if (delta > max_delta) max_delta = delta;                                                \
    }                                                                                          \
    if (counts_out) memcpy(counts_out, counts, sizeof(uint32_t) * Lc);                         \
    if (sums_out) memcpy(sums_out, sums, sizeof(T) * Lc);                                      \
    free(sums);                                                                                \
    free(counts);                                                                              \
    return max_delta;                                                                          \
  }                                                                                            \
                                                                                               \
  int64_t oracle_path_triples_##SFX(const T *centroid, size_t Lc, const T *seq, size_t len,    \
                                    int os, int oe, int fma_mode, int64_t *triples,            \
                                    int64_t cap) {                                             \
    const T *first, *second;                                                                   \
    size_t m, nn;                                                                              \
    int flip;                                                                                  \
    orient_##SFX(centroid, Lc, seq, len, oe, &first, &m, &second, &nn, &flip);                 \
    unsigned char *path = (unsigned char *)calloc(m * nn, 1);                                  \
    oracle_dtw_pair_##SFX(first, m, second, nn, os, oe, fma_mode, NULL, path);                 \
    long i = (long)m - 1, j = (long)nn - 1;                                                    \
    unsigned char mv = path[i * nn + j];                                                       \
    int64_t k = 0;                                                                             \
    while (mv != ORACLE_NIL && mv != ORACLE_NIL_OPEN_RIGHT) {                                  \
      if (k >= cap) {                                                                          \
        free(path);                                                                            \
        return -1;                                                                             \
      }                                                                                        \
      triples[3 * k] = i, triples[3 * k + 1] = j, triples[3 * k + 2] = mv;                     \
      ++k;                                                                                     \
      i += kMoveI[mv];                                                                         \
      j += kMoveJ[mv];                                                                         \
      mv = path[i * nn + j];                                                                   \
    }                                                                                          \
    if (k >= cap) {                                                                            \
      free(path);                                                                              \
      return -1;                                                                               \
    }                                                                                          \
    triples[3 * k] = i, triples[3 * k + 1] = j, triples[3 * k + 2] = mv;                       \
    ++k;                                                                                       \
    free(path);                                                                                \
    return k;                                                                                  \
  }                                                                                            \
                                                                                               \
  /* Shuffle-down tree of one 32-lane warp as the reference's calc_sums runs it              \
   * (gpu_utils.hpp:47-49): lane i adds lane i+16, then i+8, ..., result in lane 0. */        \
  static T warp_tree_##SFX(T *v) {                                                             \
    for (int off = 16; off > 0; off /= 2)                                                      \
      for (int i = 0; i < off; ++i) v[i] = v[i] + v[i + off];                                  \
    return v[0];                                                                               \
  }

static double warp_tree_dbl(double *v) {
  for (int off = 16; off > 0; off /= 2)
    for (int i = 0; i < off; ++i) v[i] = v[i] + v[i + off];
  return v[0];
}

DEFINE_ORACLE(float, f32, fmaf, FLT_MAX)
DEFINE_ORACLE(double, f64, fma, DBL_MAX)

/* stripe-mode DBA round (dba.hpp:515-763), once per value type */
#define ST float
#define SNAME(x) x##_f32
#define STMAX FLT_MAX
#include "odba_stripe.inc"
#undef ST
#undef SNAME
#undef STMAX
#define ST double
#define SNAME(x) x##_f64
#define STMAX DBL_MAX
#include "odba_stripe.inc"
#undef ST
#undef SNAME
#undef STMAX

#define DEFINE_ZNORM(T, SFX)                                                                   \
  int oracle_znorm_##SFX(T *series, const uint64_t *offsets, const uint64_t *lens, int n,      \
                         double *means, double *sigmas) {                                      \
    for (int s = 0; s < n; ++s) {                                                              \
      T *x = series + offsets[s];                                                              \
      size_t len = lens[s];                                                                    \
      size_t chunks = (len + 1023) / 1024;                                                     \
      /* calc_sums: per-1024 chunk tree in T, chunks accumulated in order */                  \
      T sum = 0;                                                                               \
      for (size_t ch = 0; ch < chunks; ++ch) {                                                 \
        T warps[32];                                                                           \
        for (int w = 0; w < 32; ++w) {                                                         \
          T v[32];                                                                             \
          for (int l = 0; l < 32; ++l) {                                                       \
            size_t pos = ch * 1024 + (size_t)w * 32 + l;                                       \
            v[l] = pos < len ? x[pos] : (T)0;                                                  \
          }                                                                                    \
          warps[w] = warp_tree_##SFX(v);                                                       \
        }                                                                                      \
        sum = sum + warp_tree_##SFX(warps);                                                    \
      }                                                                                        \
      /* calc_sum_of_squares: (x - sum/len)^2 in double, same trees */                         \
      double ss = 0;                                                                           \
      double mean_for_ss = (double)sum / (double)len;                                          \
      for (size_t ch = 0; ch < chunks; ++ch) {                                                 \
        double warps[32];                                                                      \
        for (int w = 0; w < 32; ++w) {                                                         \
          double v[32];                                                                        \
          for (int l = 0; l < 32; ++l) {                                                       \
            size_t pos = ch * 1024 + (size_t)w * 32 + l;                                       \
            double t = 0;                                                                      \
            if (pos < len) {                                                                   \
              t = (double)x[pos] - mean_for_ss;                                                \
              t = t * t;                                                                       \
            }                                                                                  \
            v[l] = t;                                                                          \
          }                                                                                    \
          warps[w] = warp_tree_dbl(v);                                                         \
        }                                                                                      \
        ss = ss + warp_tree_dbl(warps);                                                        \
      }                                                                                        \
      /* rescale_sequences (gpu_utils.hpp:110-129) */                                          \
      double mean = (double)sum / (double)len;                                                 \
      double sd = sqrt(ss / (double)len);                                                      \
      if (means) means[s] = mean;                                                              \
      if (sigmas) sigmas[s] = sd;                                                              \
      if (sd == 0) sd = 1;                                                                     \
      for (size_t i = 0; i < len; ++i) {                                                       \
        double q = ((double)x[i] - mean) / sd;                                                 \
        x[i] = (T)(0.0 + q * 1.0);                                                             \
      }                                                                                        \
    }                                                                                          \
    return 0;                                                                                  \
  }

DEFINE_ZNORM(float, f32)
DEFINE_ZNORM(double, f64)

/* Distance-only restatement used as the timed CPU baseline.  Same arithmetic
 * as sweep_*: below the top row the reference's swath-left rule equals the
 * interior rule, so rows are one tight fused-multiply-add / min loop; the top
 * row keeps the open-end rules.  Checked equal to oracle_pairwise_* by the tests. */
#define DEFINE_FAST(T, SFX, FMA, FMIN, TMAX)                                                   \
  static T fast_pair_##SFX(const T *x, size_t m, const T *y, size_t n, int os, int oe, T *prev, \
                           T *cur) {                                                           \
    size_t r0 = os ? 1 : 0;                                                                    \
    T init = os ? (T)0 : TMAX;                                                                 \
    for (size_t c = 0; c < n; ++c) prev[c] = init;                                             \
    for (size_t r = r0; r < m; ++r) {                                                          \
      const T xr = x[r];                                                                       \
      T left = TMAX;                                                                           \
      T diag = (r == 0) ? (T)0 : TMAX;                                                         \
      if (oe && m >= 2 && r == m - 1) {                                                        \
        for (size_t c = 0; c < n; ++c) {                                                       \
          const T up = prev[c];                                                                \
          const T d = xr - y[c];                                                               \
          T v;                                                                                 \
          if (c > 0 && c % SWATH == 0)                                                         \
            v = FMIN(FMIN(FMA(d, d, up), diag), left);                                         \
          else                                                                                 \
            v = FMIN(FMA(d, d, FMIN(up, diag)), left);                                         \
          diag = up;                                                                           \
          left = v;                                                                            \
          cur[c] = v;                                                                          \
        }                                                                                      \
      } else {                                                                                 \
        for (size_t c = 0; c < n; ++c) {                                                       \
          const T up = prev[c];                                                                \
          const T d = xr - y[c];                                                               \
          const T v = FMA(d, d, FMIN(FMIN(up, diag), left));                                   \
          diag = up;                                                                           \
          left = v;                                                                            \
          cur[c] = v;                                                                          \
        }                                                                                      \
      }                                                                                        \
      T *t = prev;                                                                             \
      prev = cur;                                                                              \
      cur = t;                                                                                 \
    }                                                                                          \
    return prev[n - 1];                                                                        \
  }                                                                                            \
                                                                                               \
  int oracle_pairwise_fast_##SFX(const T *series, const uint64_t *offsets,                     \
                                 const uint64_t *lens, int n, int os, int oe, T *out,          \
                                 const int64_t *pair_list, int64_t n_list, int threads) {      \
    int64_t npairs = (int64_t)n * (n - 1) / 2;                                                 \
    int64_t *row_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));          \
    int64_t *col_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));          \
    int64_t p = 0;                                                                             \
    uint64_t maxlen = 1;                                                                       \
    for (int s = 0; s < n; ++s)                                                                \
      if (lens[s] > maxlen) maxlen = lens[s];                                                  \
    for (int s = 0; s + 1 < n; ++s)                                                            \
      for (int j = s + 1; j < n; ++j) {                                                        \
        row_of[p] = s;                                                                         \
        col_of[p] = j;                                                                         \
        ++p;                                                                                   \
      }                                                                                        \
    int64_t count = pair_list ? n_list : npairs;                                               \
    if (threads > 0) omp_set_num_threads(threads);                                             \
    _Pragma("omp parallel") {                                                                  \
      T *a = (T *)malloc(sizeof(T) * maxlen);                                                  \
      T *b = (T *)malloc(sizeof(T) * maxlen);                                                  \
      _Pragma("omp for schedule(dynamic, 1)") for (int64_t q = 0; q < count; ++q) {            \
        int64_t idx = pair_list ? pair_list[q] : q;                                            \
        int64_t s = row_of[idx], j = col_of[idx];                                              \
        size_t m = lens[s], nn = lens[j];                                                      \
        T corner = fast_pair_##SFX(series + offsets[s], m, series + offsets[j], nn, os, oe, a, \
                                   b);                                                         \
        float v;                                                                               \
        if (m == 1 && oe && !os && nn > SWATH)                                                 \
          v = sqrtf((float)TMAX) / (float)m;                                                   \
        else if ((oe && !os) || (!oe && os))                                                   \
          v = sqrtf((float)corner) / (float)m;                                                 \
        else                                                                                   \
          v = sqrtf((float)corner);                                                            \
        out[idx] = (T)v;                                                                       \
      }                                                                                        \
      free(a);                                                                                 \
      free(b);                                                                                 \
    }                                                                                          \
    free(row_of);                                                                              \
    free(col_of);                                                                              \
    return 0;                                                                                  \
  }

DEFINE_FAST(float, f32, fmaf, fminf, FLT_MAX)
DEFINE_FAST(double, f64, fma, fmin, DBL_MAX)

/* FP64 reference distances: the recurrence, tie order, swath rules and
 * open-end shortcut of the reference (dtw.hpp:74-239) evaluated in double
 * whatever the result type, with the epilogue's square root and division in
 * double too (the reference takes sqrtf even for double, dtw.hpp:116-125,
 * 242-257).  Not a parity target: it states how far the float and double
 * results are from FP64 arithmetic.  for_f32 picks the shortcut lane and the
 * one-row sentinel of the float build, else those of the double build. */
int oracle_pairwise_fp64ref(const double *series, const uint64_t *offsets, const uint64_t *lens,
                            int n, int os, int oe, int for_f32, double *out,
                            const int64_t *pair_list, int64_t n_list, int threads) {
  int64_t npairs = (int64_t)n * (n - 1) / 2;
  int64_t count = pair_list ? n_list : npairs;
  int64_t *row_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));
  int64_t *col_of = (int64_t *)malloc(sizeof(int64_t) * (npairs > 0 ? npairs : 1));
  int64_t p = 0;
  uint64_t maxlen = 1;
  for (int s = 0; s < n; ++s)
    if (lens[s] > maxlen) maxlen = lens[s];
  for (int s = 0; s + 1 < n; ++s)
    for (int j = s + 1; j < n; ++j) {
      row_of[p] = s;
      col_of[p] = j;
      ++p;
    }
  const int saved_lane = g_shortcut_lane[1];
  g_shortcut_lane[1] = for_f32 ? g_shortcut_lane[0] : saved_lane; /* read by sweep_f64 */
  const double sentinel = for_f32 ? (double)FLT_MAX : DBL_MAX;
  const int shortcut = oe && !os;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
  {
    double *a = (double *)malloc(sizeof(double) * maxlen);
    double *b = (double *)malloc(sizeof(double) * maxlen);
#pragma omp for schedule(dynamic, 1)
    for (int64_t q = 0; q < count; ++q) {
      int64_t idx = pair_list ? pair_list[q] : q;
      int64_t s = row_of[idx], j = col_of[idx];
      const double *x = series + offsets[s], *y = series + offsets[j];
      size_t m = lens[s], nn = lens[j];
      double value;
      if (shortcut) {
        size_t nb = nn / SWATH + 1;
        double *bmin = (double *)malloc(sizeof(double) * nb);
        double *btop = (double *)calloc(nb, sizeof(double));
        double last = sweep_f64(x, m, y, nn, os, oe, 1, NULL, bmin, btop, NULL);
        size_t c0 = shortcut_col_f64(m, nn, os, oe, bmin, btop);
        if (c0 && m == 1)
          value = sqrt(sentinel) / (double)m;
        else
          value = sqrt(c0 ? btop[c0 / SWATH] : last) / (double)m;
        free(bmin);
        free(btop);
      } else {
        double corner = fast_pair_f64(x, m, y, nn, os, oe, a, b);
        value = os && !oe ? sqrt(corner) / (double)m : sqrt(corner);
      }
      out[idx] = value;
    }
    free(a);
    free(b);
  }
  g_shortcut_lane[1] = saved_lane;
  free(row_of);
  free(col_of);
  return 0;
}

/* ---- k-segmentation (segmentation.hpp:48-337 kernel, 340-583 host) ---------
 * One "block" = raw_samples_per_threadblock = 256 * dw samples of one series,
 * processed as the reference's 256-thread block does, thread by thread.
 * Where the reference races (the even-span median of a 2-sample segment
 * reads the first sample of the next segment while that segment is being
 * sorted), the sorted value is used.  smem is the device's opt-in shared
 * memory per block; it sets the DP extent e. */
static unsigned char seg_quant(double v) {
  /* float -> unsigned char conversion on the GPU clamps to [0, 255], NaN -> 0 */
  if (!(v == v)) return 0;
  if (v <= 0.0) return 0;
  if (v >= 255.0) return 255;
  return (unsigned char)v;
}

#define DEFINE_SEG(T, SFX, TMAX, TMIN)                                                         \
  static void seg_block_##SFX(const T *series, long orig_N, int by, int spb, int k_max,      \
                              int minseg, int smem, T *out_medians) {                        \
    const int dw = (minseg + 2) / 3;                                                         \
    const int N = ((long)(by + 1) * spb > orig_N) ? (int)(orig_N % spb) : spb;              \
    int expected_k = k_max;                                                                  \
    if ((long)(by + 1) * spb > orig_N) {                                                     \
      int per = (spb + k_max - 1) / k_max;                                                   \
      expected_k = ((int)(orig_N % spb) + per - 1) / per;                                     \
    }                                                                                        \
    const int N_ds = N / dw;                                                                 \
    const T *x = series + (long)by * spb;                                                    \
    T ds[256];                                                                               \
    for (int t = 0; t < 256; ++t) ds[t] = 0;                                                 \
    for (int t = 0; t < 256; ++t) {                                                          \
      if (t * dw <= N - dw) {                                                                \
        T acc = 0;                                                                           \
        int num = 0;                                                                         \
        for (int i = 0; i < dw && dw * t + t + i < N; i++) {                                 \
          acc = acc + x[dw * t + i];                                                         \
          num++;                                                                             \
        }                                                                                    \
        ds[t] = acc / (T)num;                                                                \
      }                                                                                      \
    }                                                                                        \
    /* warp shuffle-down reductions with "if (tmp < val) val = tmp" (cuda_utils.hpp:20-40) */ \
    T wmax[8], wmin[8];                                                                      \
    for (int w = 0; w < 8; ++w) {                                                            \
      T vmax[32], vmin[32];                                                                  \
      for (int l = 0; l < 32; ++l) {                                                         \
        int t = w * 32 + l;                                                                  \
        vmax[l] = t < N_ds ? ds[t] : TMIN;                                                   \
        vmin[l] = t < N_ds ? ds[t] : TMAX;                                                   \
      }                                                                                      \
      for (int off = 16; off > 0; off /= 2) {                                                \
        T nmax[32], nmin[32];                                                                \
        for (int l = 0; l < 32; ++l) {                                                       \
          T a = l + off < 32 ? vmin[l + off] : vmin[l];                                      \
          T b = l + off < 32 ? vmax[l + off] : vmax[l];                                      \
          nmin[l] = (a < vmin[l]) ? a : vmin[l];                                             \
          nmax[l] = (b > vmax[l]) ? b : vmax[l];                                             \
        }                                                                                    \
        memcpy(vmin, nmin, sizeof(vmin));                                                    \
        memcpy(vmax, nmax, sizeof(vmax));                                                    \
      }                                                                                      \
      wmax[w] = vmax[0];                                                                     \
      wmin[w] = vmin[0];                                                                     \
    }                                                                                        \
    const int nw = N_ds / 32;                                                                \
    T gmax, gmin;                                                                            \
    {                                                                                        \
      T vmax[32], vmin[32];                                                                  \
      for (int l = 0; l < 32; ++l) {                                                         \
        vmax[l] = l < nw ? wmax[l] : TMIN;                                                   \
        vmin[l] = l < nw ? wmin[l] : TMAX;                                                   \
      }                                                                                      \
      for (int off = 16; off > 0; off /= 2) {                                                \
        T nmax[32], nmin[32];                                                                \
        for (int l = 0; l < 32; ++l) {                                                       \
          T a = l + off < 32 ? vmin[l + off] : vmin[l];                                      \
          T b = l + off < 32 ? vmax[l + off] : vmax[l];                                      \
          nmin[l] = (a < vmin[l]) ? a : vmin[l];                                             \
          nmax[l] = (b > vmax[l]) ? b : vmax[l];                                             \
        }                                                                                    \
        memcpy(vmin, nmin, sizeof(vmin));                                                    \
        memcpy(vmax, nmax, sizeof(vmax));                                                    \
      }                                                                                      \
      gmax = vmax[0];                                                                        \
      gmin = vmin[0];                                                                        \
    }                                                                                        \
    /* only thread 0 repoints T_min at the block minimum (segmentation.hpp:144-148); the    \
     * others read slot N_ds/32 of the max array: warp 0's minimum, or with fewer than two  \
     * full warps the value thread 0 wrote there */                                          \
    T others_min = nw >= 2 ? wmin[0] : (nw == 1 ? gmin : gmax);                             \
    unsigned char q[256];                                                                    \
    for (int t = 0; t < N_ds; ++t) {                                                         \
      T mn = t == 0 ? gmin : others_min;                                                     \
      T frac = (ds[t] - mn) / (gmax - mn + 1);                                               \
      q[t] = seg_quant(256.0 * (double)frac);                                                \
    }                                                                                        \
    /* prefix sums give every SUMS / SQUARES entry (no 16-bit wrap for <= 256 samples) */   \
    unsigned P[257], Q[257];                                                                 \
    P[0] = Q[0] = 0;                                                                         \
    for (int t = 0; t < N_ds; ++t) {                                                         \
      P[t + 1] = P[t] + q[t];                                                                \
      Q[t + 1] = Q[t] + (unsigned)q[t] * q[t];                                               \
    }                                                                                        \
    /* DP extent from the reference's shared-memory layout (segmentation.hpp:96-162) */     \
    int e = 1;                                                                               \
    if (N_ds > 0) {                                                                          \
      long off_opt = ((long)(k_max + 1) * 2 + 3) / 4 * 4;                                    \
      long off_ksd = off_opt + (long)(N_ds + 1) * 4;                                         \
      long off_ds = (off_ksd + 2L * (N_ds + 1) * 4 + sizeof(T) - 1) / sizeof(T) * sizeof(T); \
      long off_sq = (off_ds + (long)(N_ds + 2) * sizeof(T) + 3) / 4 * 4;                     \
      e = (int)((smem - off_sq) / ((long)N_ds * 6));                                         \
    }                                                                                        \
    /* 1-based DIST(l, r): SQUARES - SUMS*SUMS/len, unsigned minus int (int product wraps) */ \
    unsigned *ksd0 = (unsigned *)calloc(N_ds + 2, sizeof(unsigned));                         \
    unsigned *ksd1 = (unsigned *)calloc(N_ds + 2, sizeof(unsigned));                         \
    unsigned short *kpath = (unsigned short *)calloc((size_t)(k_max + 1) * (N_ds + 2), 2);  \
    unsigned short bp[260];                                                                  \
    int smallest_noisy = expected_k + 1;                                                     \
    int test_k = (expected_k + 1) / 2;                                                       \
    int delta = test_k / 2;                                                                  \
    int exitf = 0;                                                                           \
    while (!exitf) {                                                                         \
      for (int t = 0; t < N_ds; ++t) {                                                       \
        int n1 = t + 1;                                                                      \
        if (n1 <= e) {                                                                       \
          unsigned s = P[n1] - P[0];                                                         \
          unsigned sq = Q[n1] - Q[0];                                                        \
          int ms = (int)((unsigned)(s * s)) / n1;                                            \
          ksd1[n1] = sq - (unsigned)ms;                                                      \
        } else {                                                                             \
          ksd1[n1] = INT_MAX / 2;                                                            \
        }                                                                                    \
        if (t < test_k) kpath[(size_t)t * (N_ds + 2) + t] = (unsigned short)(test_k - 1);    \
      }                                                                                      \
      for (int p = 2; p <= test_k; ++p) {                                                    \
        unsigned *prev = (p % 2) ? ksd0 : ksd1;                                              \
        unsigned *cur = (p % 2) ? ksd1 : ksd0;                                               \
        for (int n = p; n <= N_ds; ++n) {                                                    \
          int lo = (n - e + 1 > p) ? n - e + 1 : p;                                          \
          int minval = INT_MAX, minidx = -1;                                                 \
          for (int idx = lo, start = lo; idx - start < e && idx <= n; idx++) {               \
            unsigned s = P[n] - P[idx - 1];                                                  \
            unsigned sq = Q[n] - Q[idx - 1];                                                 \
            int len = n - idx + 1;                                                           \
            int ms = (int)((unsigned)(s * s)) / len;                                         \
            unsigned opt = prev[idx - 1] + (sq - (unsigned)ms);                              \
            if (opt < (unsigned)minval) {                                                    \
              minval = (int)opt;                                                             \
              minidx = idx;                                                                  \
            }                                                                                \
          }                                                                                  \
          cur[n] = (unsigned)minval;                                                         \
          kpath[(size_t)(p - 1) * (N_ds + 2) + (n - 1)] = (unsigned short)((unsigned short)minidx - 1); \
        }                                                                                    \
      }                                                                                      \
      bp[test_k] = (unsigned short)N_ds;                                                     \
      for (int p = test_k - 1; p >= 1; p--) {                                                \
        int col = bp[p + 1] - 1;                                                             \
        bp[p] = (col >= 0 && col < N_ds + 2) ? kpath[(size_t)p * (N_ds + 2) + col] : 0;      \
      }                                                                                      \
      bp[0] = 0;                                                                             \
      int noisy = 0;                                                                         \
      for (int i = 1; i <= test_k; i++)                                                      \
        if ((int)bp[i] - (int)bp[i - 1] < minseg / dw) noisy = 1;                            \
      if (delta == 0 || test_k + delta > k_max) {                                            \
        exitf = 1;                                                                           \
      } else if (test_k != 1 && noisy) {                                                     \
        smallest_noisy = test_k;                                                             \
        test_k -= delta;                                                                     \
      } else {                                                                               \
        if (test_k == 1 || smallest_noisy == test_k + 1)                                     \
          exitf = 1;                                                                         \
        else                                                                                 \
          test_k += delta;                                                                   \
      }                                                                                      \
      delta = (delta + 1) / 2;                                                               \
    }                                                                                        \
    /* medians: segments sorted, then the reference's quirky middle pick */                 \
    T *od = (T *)calloc((size_t)spb + 2, sizeof(T));                                         \
    for (int i = 0; i < spb && (long)by * spb + i < orig_N; ++i) od[i] = x[i];               \
    for (int t = test_k + 1; t <= k_max; ++t) out_medians[t - 1] = TMAX;                     \
    for (int t = 1; t <= test_k; ++t) {                                                      \
      int rb = bp[t] * dw;                                                                   \
      if (rb > N) rb = N;                                                                    \
      int lb = bp[t - 1] * dw;                                                               \
      for (int i = lb; i < rb - 1; ++i)                                                      \
        for (int j = i + 1; j < rb; ++j)                                                     \
          if (od[i] > od[j]) {                                                               \
            T tmp = od[i];                                                                   \
            od[i] = od[j];                                                                   \
            od[j] = tmp;                                                                     \
          }                                                                                  \
    }                                                                                        \
    for (int t = 1; t <= test_k; ++t) {                                                      \
      int rb = bp[t] * dw;                                                                   \
      if (rb > N) rb = N;                                                                    \
      int lb = bp[t - 1] * dw;                                                               \
      if ((lb - rb) % 2)                                                                     \
        out_medians[t - 1] = od[(lb + rb) / 2];                                              \
      else                                                                                   \
        out_medians[t - 1] = (od[(lb + rb) / 2] + od[(lb + rb) / 2 + 1]) / 2;                \
    }                                                                                        \
    free(ksd0);                                                                              \
    free(ksd1);                                                                              \
    free(kpath);                                                                             \
    free(od);                                                                                \
  }                                                                                          \
                                                                                             \
  int64_t oracle_segment_##SFX(const T *series, const uint64_t *offsets, const uint64_t *lens,  \
                               int n, int minseg, int prefix_skip, int smem, T *out,          \
                               uint64_t *out_lens) {                                          \
    const int dw = (minseg + 2) / 3;                                                         \
    const int spb = 256 * dw;                                                                \
    const int k_max = (int)((256 + ((float)minseg) / dw - 1) / (((float)minseg) / dw));      \
    int64_t written = 0;                                                                     \
    for (int s = 0; s < n; ++s) {                                                            \
      const long L = (long)lens[s];                                                          \
      const int nb = (int)((L + spb - 1) / spb);                                             \
      size_t cap = (size_t)k_max * nb;                                                       \
      T *seg = (T *)malloc(sizeof(T) * (cap ? cap : 1));                                     \
      for (int by = 0; by < nb; ++by)                                                        \
        seg_block_##SFX(series + offsets[s], L, by, spb, k_max, minseg, smem,               \
                        seg + (size_t)by * k_max);                                           \
      /* host post-processing (segmentation.hpp:492-573) */                                  \
      T epsilon = TMAX;                                                                      \
      T previous = seg[0];                                                                   \
      for (size_t j = 1; j < cap; ++j) {                                                     \
        T current = seg[j];                                                                  \
        if (current != TMAX && previous != TMAX &&                                           \
            ((current <= previous && previous - current < epsilon) ||                        \
             (current > previous && current - previous < epsilon))) {                        \
          if (current - previous == 0) {                                                     \
            for (size_t k = j; k < cap; k++) {                                               \
              seg[k - 1] = seg[k];                                                           \
              if (seg[k] == TMAX) break;                                                     \
            }                                                                                \
          } else {                                                                           \
            epsilon = current < previous ? (previous - current) : (current - previous);      \
          }                                                                                  \
        }                                                                                    \
        previous = current;                                                                  \
      }                                                                                      \
      int prev_undef = 0;                                                                    \
      long cursor = 0;                                                                       \
      for (size_t j = 0; j < cap; ++j) {                                                     \
        if (seg[j] == TMAX) {                                                                \
          prev_undef = 1;                                                                    \
          continue;                                                                          \
        }                                                                                    \
        if (prev_undef) {                                                                    \
          prev_undef = 0;                                                                    \
          if (cursor >= 1 && seg[cursor - 1] < seg[j] + epsilon &&                           \
              seg[cursor - 1] > seg[j] - epsilon)                                            \
            seg[cursor - 1] = (seg[cursor - 1] + seg[j]) / 2;                                \
        }                                                                                    \
        if ((size_t)cursor != j) seg[cursor] = seg[j];                                       \
        cursor++;                                                                            \
      }                                                                                      \
      if (cursor >= 1 && seg[cursor - 1] >= TMAX / 2) cursor--;                              \
      long skipped = 0;                                                                      \
      if (prefix_skip) {                                                                     \
        if (cursor <= prefix_skip) {                                                         \
          skipped = cursor - 1;                                                              \
          cursor = 1;                                                                        \
        } else {                                                                             \
          skipped = prefix_skip;                                                             \
          cursor -= prefix_skip;                                                             \
        }                                                                                    \
      }                                                                                      \
      out_lens[s] = (uint64_t)cursor;                                                        \
      memcpy(out + written, seg + skipped, sizeof(T) * (size_t)cursor);                      \
      written += cursor;                                                                     \
      free(seg);                                                                             \
    }                                                                                        \
    return written;                                                                          \
  }

DEFINE_SEG(float, f32, FLT_MAX, FLT_MIN)
DEFINE_SEG(double, f64, DBL_MAX, DBL_MIN)
