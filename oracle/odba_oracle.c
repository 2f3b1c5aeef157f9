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
 *   z-normalisation                             gpu_utils.hpp:34-170
 */
#include "odba_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* The reference's swath width: blockDim.x of every DTWDistance launch
 * (maxThreadsPerBlock, cuda_utils.hpp:42-57, forced to 1024 in DBAUpdate at
 * dba.hpp:455-457).  Its open-end rules depend on it (dtw.hpp:74, 172-200). */
#define SWATH 1024

static const int kMoveI[7] = {-1, -1, 0, -1, 0, 0, 0}; /* dtw.hpp:20 */
static const int kMoveJ[7] = {-1, -1, -1, 0, -1, -1, -1}; /* dtw.hpp:21 */

#define DEFINE_ORACLE(T, SFX, FMA, TMAX)                                                        \
  static inline T add_dd_##SFX(T acc, T d, int fma_mode) {                                     \
    if (fma_mode) return FMA(d, d, acc);                                                       \
    T dd = d * d;                                                                              \
    return acc + dd;                                                                           \
  }                                                                                            \
                                                                                               \
  /* Full cost matrix sweep, row by row.  Keeps two rows; optionally stores moves and the     \
   * per-swath-boundary column minima the open-end shortcut needs.  Returns C[m-1][n-1]. */    \
  static T sweep_##SFX(const T *first, size_t m, const T *second, size_t n, int os, int oe,     \
                       int fma_mode, unsigned char *path, T *bmin, T *btop) {                  \
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
        if (bmin && (c + 1) % SWATH == 0) {                                                    \
          size_t k = (c + 1) / SWATH;                                                          \
          if (v < bmin[k]) bmin[k] = v;                                                        \
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
    T *bmin = NULL, *btop = NULL;                                                              \
    if (path) {                                                                                \
      bmin = (T *)malloc(sizeof(T) * nb);                                                      \
      btop = (T *)calloc(nb, sizeof(T));                                                       \
    }                                                                                          \
    T last = sweep_##SFX(first, m, second, n, os, oe, fma_mode, path, bmin, btop);             \
    if (path) {                                                                                \
      size_t c0 = shortcut_col_##SFX(m, n, os, oe, bmin, btop);                                \
      if (c0)                                                                                  \
        for (size_t c = c0; c < n; ++c) path[(m - 1) * n + c] = ORACLE_OPEN_RIGHT;             \
      free(bmin);                                                                              \
      free(btop);                                                                              \
    }                                                                                          \
    if (dist_out) {                                                                            \
      /* The shortcut never changes the top-row value it freezes, so the distance is the     \
       * full sweep's corner -- except for a single-row matrix, where the shortcut reads the \
       * sentinel it has just written (dtw.hpp:113, 121). */                                   \
      if (m == 1 && oe && !os && n > SWATH) {                                                  \
        *dist_out = (T)(sqrtf((float)TMAX) / (float)m);                                        \
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
