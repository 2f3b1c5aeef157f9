/* CPU oracle for the OpenDBA hot path -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C restatement of the reference's arithmetic, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * Nothing in opendba_b200/ links or calls it.
 *
 * fma_mode selects how the reference's "cost + diff*diff" is rounded:
 *   1 = one fused multiply-add (fmaf/fma), 0 = product rounded, then sum rounded.
 * Which one nvcc emitted for the reference on sm_100a is pinned against the
 * reference's own GPU outputs (tests/golden/ref/).
 */
#ifndef ODBA_ORACLE_H
#define ODBA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Move codes of the reference's path matrix (dtw.hpp:10-16). */
#define ORACLE_NIL 255
#define ORACLE_DIAGONAL 1
#define ORACLE_RIGHT 2
#define ORACLE_UP 3
#define ORACLE_OPEN_RIGHT 4
#define ORACLE_NIL_OPEN_RIGHT 5

/* Which warp-0 lane's partial minimum the open-end shortcut check reads in
 * the float and double restatements (defaults 0 and 16, the reference's B200
 * builds); tests vary it to find inputs that tell lanes apart. */
void oracle_set_shortcut_lanes(int lane_f32, int lane_f64);

/* One pair: first (rows, length m) against second (columns, length n).
 * dist_out receives the reference's medoid-pass distance (dtw.hpp:116-125,
 * 242-257).  If path is non-NULL it receives m*n move codes, row-major
 * (path[r*n+c]), with the open-end shortcut's OPEN_RIGHT overrides applied;
 * cells the reference never computes are left as 0.  Returns 0 on success. */
int oracle_dtw_pair_f32(const float *first, size_t m, const float *second, size_t n,
                        int open_start, int open_end, int fma_mode, float *dist_out,
                        unsigned char *path);
int oracle_dtw_pair_f64(const double *first, size_t m, const double *second, size_t n,
                        int open_start, int open_end, int fma_mode, double *dist_out,
                        unsigned char *path);

/* All pairs i<j of a ragged set (series i starts at offsets[i]); out has
 * n(n-1)/2 entries in the reference's upper-triangle order (clustering.cuh:6).
 * If pair_list is non-NULL only the listed pair indices are computed (used
 * for bounded CPU-baseline samples).  threads <= 0 uses all cores. */
int oracle_pairwise_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                        int n, int open_start, int open_end, int fma_mode, float *out,
                        const int64_t *pair_list, int64_t n_list, int threads);
int oracle_pairwise_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                        int n, int open_start, int open_end, int fma_mode, double *out,
                        const int64_t *pair_list, int64_t n_list, int threads);

/* Same distances as oracle_pairwise_*, distance-only tight loop (the timed
 * CPU baseline). */
int oracle_pairwise_fast_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                             int n, int open_start, int open_end, float *out,
                             const int64_t *pair_list, int64_t n_list, int threads);
int oracle_pairwise_fast_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                             int n, int open_start, int open_end, double *out,
                             const int64_t *pair_list, int64_t n_list, int threads);

/* FP64 reference distances for stating the error of a result: the same
 * recurrence, tie order, swath rules and open-end shortcut evaluated in double
 * (series given as double), square root and division in double.  for_f32
 * selects the float build's shortcut lane and one-row sentinel. */
int oracle_pairwise_fp64ref(const double *series, const uint64_t *offsets, const uint64_t *lens,
                            int n, int open_start, int open_end, int for_f32, double *out,
                            const int64_t *pair_list, int64_t n_list, int threads);

/* Medoid selection of approximateMedoidIndices for one cluster (dba.hpp:186-351):
 * sums of squared distances accumulated in T in row-major pair order. */
int oracle_medoid_f32(const float *dists, int n, const uint64_t *lens, float *sos_out);
int oracle_medoid_f64(const double *dists, int n, const uint64_t *lens, double *sos_out);

/* One DBA round (DBAUpdate, dba.hpp:432-848, with updateCentroid dba.hpp:374-423).
 * Members are given in the order the reference processes them.  mean_out gets
 * sum/count in T, counts_out the pile-up counts, and the return value is the
 * max |old - new| in double.  If path_lens_out is non-NULL, path_lens_out[k]
 * gets the number of backtrack lines member k's path file would hold. */
double oracle_dba_update_f32(const float *centroid, size_t Lc, const float *series,
                             const uint64_t *offsets, const uint64_t *lens, int n,
                             int open_start, int open_end, int fma_mode, float *mean_out,
                             uint32_t *counts_out, float *sums_out);
double oracle_dba_update_f64(const double *centroid, size_t Lc, const double *series,
                             const uint64_t *offsets, const uint64_t *lens, int n,
                             int open_start, int open_end, int fma_mode, double *mean_out,
                             uint32_t *counts_out, double *sums_out);

/* One DBA round in the reference's stripe mode (dba.hpp:515-763), including
 * the open-end rules its stripe re-run applies at the backtrack height (see
 * odba_stripe.inc).  lane: which warp-0 lane's partial minimum the open-end
 * shortcut check reads (0: the full minimum).  Per-member path cells
 * (row, column, move) go to triples back to back (tri_counts[k] cells for
 * member k, -1 if tri_cap ran out); hazards[k] counts the walk's stripe exits
 * on row 0 past the first stripe. */
double oracle_dba_update_stripe_f32(const float *centroid, size_t Lc, const float *series,
                                    const uint64_t *offsets, const uint64_t *lens, int n,
                                    int open_start, int open_end, int fma_mode, int lane,
                                    float *mean_out, uint32_t *counts_out, int64_t *triples,
                                    int64_t tri_cap, int64_t *tri_counts, int64_t *hazards);
double oracle_dba_update_stripe_f64(const double *centroid, size_t Lc, const double *series,
                                    const uint64_t *offsets, const uint64_t *lens, int n,
                                    int open_start, int open_end, int fma_mode, int lane,
                                    double *mean_out, uint32_t *counts_out, int64_t *triples,
                                    int64_t tri_cap, int64_t *tri_counts, int64_t *hazards);

/* Backtrack of one member against the centroid, emitting the (i, j, move)
 * triples in the order the reference's path file lists them (io_utils.hpp:287-323),
 * the final anchor line included.  Returns the number of triples written, or
 * -1 if cap is too small. */
int64_t oracle_path_triples_f32(const float *centroid, size_t Lc, const float *seq, size_t len,
                                int open_start, int open_end, int fma_mode, int64_t *triples,
                                int64_t cap);
int64_t oracle_path_triples_f64(const double *centroid, size_t Lc, const double *seq, size_t len,
                                int open_start, int open_end, int fma_mode, int64_t *triples,
                                int64_t cap);

/* Z-normalisation (gpu_utils.hpp:34-170) in place, chunk partials of 1024
 * added in ascending chunk order; writes the double means and sigmas. */
int oracle_znorm_f32(float *series, const uint64_t *offsets, const uint64_t *lens, int n,
                     double *means, double *sigmas);
int oracle_znorm_f64(double *series, const uint64_t *offsets, const uint64_t *lens, int n,
                     double *means, double *sigmas);

/* k-segmentation of every series (adaptive_segmentation, segmentation.hpp:340-583)
 * with the device's opt-in shared memory per block smem; out receives the
 * concatenated segment medians, out_lens the segment counts.  Returns the
 * number of values written. */
int64_t oracle_segment_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                           int n, int minseg, int prefix_skip, int smem, float *out,
                           uint64_t *out_lens);
int64_t oracle_segment_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                           int n, int minseg, int prefix_skip, int smem, double *out,
                           uint64_t *out_lens);

#ifdef __cplusplus
}
#endif
#endif
