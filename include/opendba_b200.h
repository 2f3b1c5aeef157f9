/* opendba_b200 -- C ABI of the B200 (sm_100a) implementation of OpenDBA's
 * data-parallel hot path: the all-vs-all DTW medoid pass, z-normalisation and
 * the DBA round (DTW with warp path, backtrack, centroid update).
 *
 * The reference (Brooklynvcx/OpenDBA) has no library or FFI: its API is the
 * header-only C++ templates in dba.hpp / gpu_utils.hpp included into one
 * translation unit.  Each entry point below replaces one of those, as cited.
 * All functions return an odba_status; on failure odba_last_error() gives a
 * message (per calling thread).  Device pointers are plain CUDA device (or
 * managed) addresses; "stream" is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  No function keeps a pointer after it returns.
 *
 * Series layout on the device: the n series are concatenated in one array;
 * series i starts at element offsets[i] and has lens[i] elements (>= 1).
 * Pair distances use the reference's upper-triangle order: pair (s, j), s < j,
 * at index s*n - s*(s+1)/2 + (j - s - 1) (clustering.cuh:4-6).
 */
#ifndef OPENDBA_B200_H
#define OPENDBA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ODBA_ABI_VERSION 1

enum odba_status {
  ODBA_OK = 0,
  ODBA_ERR_INVALID_ARGUMENT = 1,
  ODBA_ERR_CUDA = 2,
  ODBA_ERR_OUT_OF_MEMORY = 3,
  ODBA_ERR_WORKSPACE_TOO_SMALL = 4,
  ODBA_ERR_UNSUPPORTED_DEVICE = 5,
  ODBA_ERR_TIMEOUT = 6,
  ODBA_ERR_IO = 7
};

int odba_abi_version(void);
const char *odba_status_string(int status);
/* Message of the last failure in the calling thread ("" if none). */
const char *odba_last_error(void);
/* ODBA_OK when the current CUDA device is a compute capability 10.x (B200) part. */
int odba_device_check(void);

/* ---- all-vs-all DTW distances (the medoid pass) ----------------------------
 * Replaces the DTWDistance launch loop of approximateMedoidIndices
 * (dba.hpp:37-161, kernel dtw.hpp:39-259) for one device.  Series s is the
 * first (row) series of pair (s, j), as in the reference.  The workspace holds
 * a work counter and swath-edge buffers.  odba_dtw_pairwise_workspace_bytes
 * depends only on the element size and the longest series and fits every
 * launch plan when there are at most as many pairs as resident warps;
 * odba_dtw_pairwise_workspace_bytes_n is the tighter size of the plan chosen
 * by default for n series (few long series: per-pair edge buffers instead of
 * per-warp ones).  A smaller workspace restricts the plans to those that fit.
 * use_open_start / use_open_end have the reference's meaning
 * (openDBA.cu:72-104), including its open-end shortcut (dtw.hpp:74-129):
 * where it fires the distance is the last-row value of that swath's left
 * edge.  The shortcut compares that value with a minimum the reference's float
 * build takes over the whole edge and its double build over the edge rows r
 * with r % 1024 >= 512 (which of its warp-0 lanes' shared stores survives, as
 * its B200 runs show); both are reproduced.  If a swath hand-off wait of the pipelined plan runs
 * out (it never does in a healthy launch), the pairs it touched read NaN and
 * the word at byte 8 of the workspace is non-zero. */
size_t odba_dtw_pairwise_workspace_bytes(int elem_size, uint64_t max_len);
size_t odba_dtw_pairwise_workspace_bytes_n(int elem_size, int n, uint64_t max_len);
int odba_dtw_pairwise_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                          int n, uint64_t max_len, int use_open_start, int use_open_end,
                          float *dists, void *workspace, size_t workspace_bytes, void *stream);
int odba_dtw_pairwise_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                          int n, uint64_t max_len, int use_open_start, int use_open_end,
                          double *dists, void *workspace, size_t workspace_bytes, void *stream);

/* ---- a range of the all-vs-all pairs (one device's share) -------------------
 * Replaces one device's part of approximateMedoidIndices' launch loop, which
 * deals the rows of the pair triangle to the devices in turn (dba.hpp:67-161).
 * Computes pairs p in [pair_begin, pair_end) of the upper triangle (reference
 * order, clustering.cuh:4-6) into dists[p] of a full-size triangle buffer;
 * other entries are not touched.  Same workspace rules as
 * odba_dtw_pairwise_*, with the pairs of the range in place of n(n-1)/2. */
int odba_dtw_pairwise_range_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                                int n, uint64_t max_len, int use_open_start, int use_open_end,
                                uint64_t pair_begin, uint64_t pair_end, float *dists,
                                void *workspace, size_t workspace_bytes, void *stream);
int odba_dtw_pairwise_range_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                                int n, uint64_t max_len, int use_open_start, int use_open_end,
                                uint64_t pair_begin, uint64_t pair_end, double *dists,
                                void *workspace, size_t workspace_bytes, void *stream);

/* ---- launch plans of the pair kernels, and their autotuner -------------------
 * No reference counterpart (the reference has one launch shape).  Every plan
 * gives the same distances bit for bit:
 *   ODBA_PLAN_WHOLE_PAIR             one warp per pair, 1024-column swaths
 *                                    (512 for double), persistent work queue;
 *   ODBA_PLAN_WHOLE_PAIR_HALF_SWATH  the same with half-width swaths;
 *   ODBA_PLAN_SWATH_PIPELINE         many warps per pair: swaths of one pair
 *                                    run on different warps, each waiting
 *                                    (bounded) on the previous swath's edge.
 * The plan is chosen per key (element size, len_bucket = floor(log2 max_len),
 * count_bucket = floor(log2 pairs)): a plan pinned with odba_tune_set; else,
 * in tuning mode (odba_tune_mode(1)), each eligible plan not yet measured for
 * the key, launch by launch; else the fastest measured plan; else a rule of
 * thumb.  odba_tune_query reports the plan the next launch would use and the
 * measured rates (pairs * max_len^2 per second, ODBA_PLAN_COUNT doubles,
 * index = plan).  odba_tune_flush waits for pending measurements;
 * odba_tune_save / odba_tune_load write and read the table as text. */
enum {
  ODBA_PLAN_AUTO = 0,
  ODBA_PLAN_WHOLE_PAIR = 1,
  ODBA_PLAN_WHOLE_PAIR_HALF_SWATH = 2,
  ODBA_PLAN_SWATH_PIPELINE = 3,
  ODBA_PLAN_COUNT = 4
};
int odba_tune_set(int elem_size, int len_bucket, int count_bucket, int plan);
int odba_tune_query(int elem_size, uint64_t max_len, uint64_t npairs, size_t workspace_bytes,
                    int *plan, double *rates);
void odba_tune_mode(int on);
int odba_tune_flush(void);
int odba_tune_save(const char *path);
int odba_tune_load(const char *path);

/* ---- row bands of the DBA round's path DTW ----------------------------------------
 * No reference counterpart (a tuning knob; results do not depend on it).
 * When a round's (member, swath) tasks are fewer than about three waves of
 * the GPU's resident warps, the path DTW cuts each member's rows into bands
 * so that the last wave of tasks is short.  n in 1..8 pins the number of
 * bands for the following launches (1: none), 0 restores the automatic
 * choice.  A workspace size queried under one setting fits launches under the
 * same setting. */
int odba_round_set_bands(int n);

/* ---- self-test of the bounded device wait --------------------------------------
 * No reference counterpart.  One warp runs the swath pipeline's wait on a
 * progress word that nothing publishes, with the given limit (at most 10 s);
 * returns ODBA_ERR_TIMEOUT when the wait ran out and raised the error word,
 * as it must. */
int odba_selftest_wait_timeout(uint64_t limit_ns, void *stream);

/* ---- DTW distances of an arbitrary pair list (batched jobs, queries) ----------
 * No single reference counterpart: the batched form of the medoid launches of
 * approximateMedoidIndices (dba.hpp:67-161) over many independent jobs, and
 * read-vs-centroid queries, in one persistent launch.  Task i aligns series
 * `first` (rows) against series `second` (columns) of the shared series table
 * and writes the reference's pair distance (dtw.hpp:116-125, 242-257) to
 * dists[out & (2^62 - 1)]; bit 62 of `out` selects open start, bit 63 open end.
 * Tasks are taken in array order (put the largest m*n first).  The workspace
 * is odba_dtw_pairwise_workspace_bytes(elem_size, max_len) with max_len the
 * longest `first` series.  series may be NULL: offsets are then element
 * addresses (device address / element size), so series in separate
 * allocations can share one launch. */
typedef struct odba_pair_task {
  uint32_t first;
  uint32_t second;
  uint64_t out;
} odba_pair_task;
int odba_dtw_pairlist_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                          const odba_pair_task *tasks, uint64_t ntasks, uint64_t max_len,
                          float *dists, void *workspace, size_t workspace_bytes, void *stream);
int odba_dtw_pairlist_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                          const odba_pair_task *tasks, uint64_t ntasks, uint64_t max_len,
                          double *dists, void *workspace, size_t workspace_bytes, void *stream);

/* ---- all-vs-all DTW distances without any device allocation -----------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory at the call site (a serving or real-time loop that forbids allocation
 * after start-up, or a host that owns the device's whole memory budget and
 * gives plugins no allocator): same inputs, outputs and results as
 * odba_dtw_pairwise_f32, but the work counter and swath-edge buffers live in a
 * fixed 64 MiB array inside the library instead of a caller workspace.
 *   - The array belongs to a module of its own.  Under CUDA's lazy module
 *     loading (the default) it is mapped by the first call on each device, so
 *     that call can itself need 64 MiB of free device memory: make it at
 *     start-up.  It stays mapped until the context ends.
 *   - Every lens[i] must be at most max_len (a pair whose first series is
 *     longer gets NaN).  max_len up to 2,097,088 samples; a larger one is
 *     rejected with ODBA_ERR_INVALID_ARGUMENT.  Series above about 4,700
 *     samples run on fewer warps than odba_dtw_pairwise_f32 (59 % of them at
 *     8,000 samples on a B200), one block of 4 warps above about 1.05 M.
 *   - Each call looks up the array's device address (cudaGetSymbolAddress)
 *     unless its stream is capturing, so a device reset between calls is
 *     fine; a call on a capturing stream needs an earlier call outside
 *     capture in the same context.  Make the first call before any stream
 *     capture.
 *   - Calls share the array: calls that overlap on the GPU (two streams, two
 *     host threads) race and must be serialized by the caller. */
int odba_dtw_pairwise_noalloc_f32(const float *series, const uint64_t *offsets,
                                  const uint64_t *lens, int n, uint64_t max_len,
                                  int use_open_start, int use_open_end, float *dists,
                                  void *stream);

/* ---- clustering of the medoid pass --------------------------------------------
 * Replaces the clustering half of approximateMedoidIndices (dba.hpp:219-343)
 * and the hclust-cpp calls it makes (hclust_fast with complete linkage,
 * cutree_k, cutree_cdist; dba.hpp:234, 248, 276).  Host memory throughout.
 * odba_complete_linkage: dists is the condensed upper triangle (n(n-1)/2
 * doubles, reference pair order); merge (2(n-1) ints, column-major (n-1) x 2)
 * and height (n-1) follow R's hclust convention (singleton x as -(x+1),
 * cluster of step k as k+1, heights ascending).  odba_cutree_k labels the n
 * leaves after the first n-k merges, clusters numbered by their lowest leaf
 * (k < 2 or k > n: one cluster); odba_cutree_cdist applies the merges below
 * height cdist.  odba_cluster_medoids_*: from the T distance triangle and the
 * lengths, the memberships and per-cluster medoids for a clustering threshold
 * cdist with the reference's meaning (1: one cluster; > 1: that many
 * clusters, raised until enough have several members; [0, 1): cut height on
 * distances scaled by the largest; negative: one cluster, the reference
 * leaves it unimplemented); medoids needs n ints. */
int odba_complete_linkage(int n, const double *dists, int *merge, double *height);
int odba_cutree_k(int n, const int *merge, int k, int *labels);
int odba_cutree_cdist(int n, const int *merge, const double *height, double cdist, int *labels);
int odba_cluster_medoids_f32(int n, const float *dists, const uint64_t *lens, double cdist,
                             int *memberships, int *medoids, int *num_clusters);
int odba_cluster_medoids_f64(int n, const double *dists, const uint64_t *lens, double cdist,
                             int *memberships, int *medoids, int *num_clusters);

/* ---- medoid from pair distances (one cluster) ------------------------------
 * Replaces the sum-of-squares and medoid choice of approximateMedoidIndices
 * (dba.hpp:186-203, 325-342).  sos (n values) and medoid (one int) are device
 * buffers; lens are the device series lengths (used when n == 2). */
int odba_medoid_f32(const float *dists, const uint64_t *lens, int n, float *sos, int *medoid,
                    void *stream);
int odba_medoid_f64(const double *dists, const uint64_t *lens, int n, double *sos, int *medoid,
                    void *stream);

/* ---- z-normalisation in place ----------------------------------------------
 * Replaces normalizeSequences<T> with refSequenceIndex < 0 (gpu_utils.hpp:132-170).
 * means / sigmas (n doubles, device) may be NULL. */
int odba_znorm_f32(float *series, const uint64_t *offsets, const uint64_t *lens, int n,
                   double *means, double *sigmas, void *stream);
int odba_znorm_f64(double *series, const uint64_t *offsets, const uint64_t *lens, int n,
                   double *means, double *sigmas, void *stream);

/* ---- one DBA round -------------------------------------------------------------
 * Replaces DBAUpdate<T> (dba.hpp:432-848) with updateCentroid (dba.hpp:374-423)
 * for the full-path (non-stripe) case: aligns every member to the centroid by
 * DTW with a recorded path, backtracks, and averages the aligned member samples
 * into new_centroid (Lc values, T) with their pile-up counts; *delta (device
 * double) receives max |centroid - new_centroid|.  Members are processed in the
 * given order, and every centroid sum is added in the reference's order, so
 * the result is bit-identical to the reference's.  h_lens is a host copy of
 * lens (it sizes the workspace).  If path_triples is non-NULL it receives, per
 * member k starting at triple sum_{i<k}(lens[i] + Lc + 1), the path as
 * (row, column, move) int32 triples in the order of the reference's path file
 * (io_utils.hpp:287-323, move codes of dtw.hpp:10-16), and path_counts[k] the
 * number of triples (-1 if the walk failed).  The path DTW may run as a swath
 * pipeline whose hand-off waits are bounded: if one ever runs out, the 32-bit
 * word at byte 8 of the workspace is non-zero after the round (it is cleared
 * at every launch; the same holds for the batched and stripe-mode rounds). */
size_t odba_dba_round_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                      uint64_t centroid_len, int use_open_start, int use_open_end);
int odba_dba_round_f32(const float *centroid, uint64_t centroid_len, const float *series,
                       const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                       int use_open_start, int use_open_end, float *new_centroid, uint32_t *counts,
                       double *delta, int32_t *path_triples, int64_t *path_counts,
                       void *workspace, size_t workspace_bytes, void *stream);
int odba_dba_round_f64(const double *centroid, uint64_t centroid_len, const double *series,
                       const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                       int use_open_start, int use_open_end, double *new_centroid,
                       uint32_t *counts, double *delta, int32_t *path_triples,
                       int64_t *path_counts, void *workspace, size_t workspace_bytes,
                       void *stream);

/* ---- one DBA round over several GPUs: ranges, then the ordered reducer --------
 * The two halves of odba_dba_round_* for a round whose members are dealt to
 * several GPUs, as DBAUpdate deals them to its devices (dba.hpp:484-486,
 * currDevice = seq_index % deviceCount) before averaging on the host
 * (dba.hpp:817-836).  odba_dba_round_ranges_*: path DTW and backtrack
 * (updateCentroid's walk, dba.hpp:374-423) of this GPU's members; ranges
 * (device, n * centroid_len pairs of int32) receives, for member k at pair
 * k * centroid_len + t, the first and last member sample index that centroid
 * index t receives ((1, 0) if none); same workspace as odba_dba_round_*.
 * odba_dba_reduce_ranges_*: from all members' ranges (members in the round's
 * order, gathered from every GPU) and the series, new_centroid, counts and
 * *delta exactly as odba_dba_round_* computes them (the sums are added in the
 * reference's order, so the result is bit-identical to the one-GPU round).
 * ranges must come from odba_dba_round_ranges_* for the same centroid and
 * members; workspace of odba_dba_reduce_workspace_bytes. */
int odba_dba_round_ranges_f32(const float *centroid, uint64_t centroid_len, const float *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int32_t *ranges,
                              void *workspace, size_t workspace_bytes, void *stream);
int odba_dba_round_ranges_f64(const double *centroid, uint64_t centroid_len, const double *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int32_t *ranges,
                              void *workspace, size_t workspace_bytes, void *stream);
size_t odba_dba_reduce_workspace_bytes(int elem_size, int n);
int odba_dba_reduce_ranges_f32(const float *centroid, uint64_t centroid_len, const float *series,
                               const uint64_t *offsets, const uint64_t *lens, int n,
                               int use_open_start, int use_open_end, const int32_t *ranges,
                               float *new_centroid, uint32_t *counts, double *delta,
                               void *workspace, size_t workspace_bytes, void *stream);
int odba_dba_reduce_ranges_f64(const double *centroid, uint64_t centroid_len, const double *series,
                               const uint64_t *offsets, const uint64_t *lens, int n,
                               int use_open_start, int use_open_end, const int32_t *ranges,
                               double *new_centroid, uint32_t *counts, double *delta,
                               void *workspace, size_t workspace_bytes, void *stream);

/* ---- one DBA round in stripe mode ------------------------------------------------
 * Replaces DBAUpdate<T>'s stripe mode (dba.hpp:515-763), used by the
 * reference when a member's path matrix does not fit in device memory.  Same
 * arguments and results as the reference's stripe mode, but no member's path
 * is ever held whole: the forward pass keeps every swath's right edge and
 * every ckpt_rows-th cost row (a power of two; 0 = 4096), and the backtrack
 * recomputes, 1024-column stripe by stripe from the right, the tiles of
 * ckpt_rows rows below the path in parallel.  Workspace for the longest
 * member m and centroid length Lc (rows x columns after the open-end flip):
 * about (Lc/1024 * m + m/ckpt_rows * Lc) values plus m * 256 bytes (float;
 * double swaths are 512 wide) -- 80 GB for 4 M x 4 M in float with the
 * default, where a full path needs 4 TB.  In global and open-start alignment
 * the results equal odba_dba_round_* bit for bit.  With an open end they
 * follow the reference's stripe re-run, which sees the backtrack height H as
 * the first sequence's length (dba.hpp:700-721): the open-end top-row rule
 * acts on row H-1, and the shortcut (dtw.hpp:74-129) is checked on the stored
 * edge's rows below H, so paths and means differ from the full-path round. */
size_t odba_dba_round_stripe_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                             uint64_t centroid_len, int use_open_start,
                                             int use_open_end, int ckpt_rows);
int odba_dba_round_stripe_f32(const float *centroid, uint64_t centroid_len, const float *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int ckpt_rows,
                              float *new_centroid, uint32_t *counts, double *delta,
                              int32_t *path_triples, int64_t *path_counts, void *workspace,
                              size_t workspace_bytes, void *stream);
int odba_dba_round_stripe_f64(const double *centroid, uint64_t centroid_len, const double *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int ckpt_rows,
                              double *new_centroid, uint32_t *counts, double *delta,
                              int32_t *path_triples, int64_t *path_counts, void *workspace,
                              size_t workspace_bytes, void *stream);

/* ---- prefix chop -----------------------------------------------------------------
 * Replaces the alignment and path walk of chopPrefixFromSequences<T>
 * (dba.hpp:1191-1395): every series is aligned to the leader (prefix,
 * P samples, on the rows) with open-end DTW and a recorded path; walking the
 * path back from the end cell past the run of OPEN_RIGHT moves along the top
 * row gives the chop position (chop_positions[k], the first column kept;
 * -1 if the walk failed), and histograms[k * P + i] counts the path cells
 * from there to (0, 0) on leader row i.  Device buffers; h_lens is a host copy
 * of lens.  The caller normalises the leader and the series first (as the
 * reference does when it normalises) and cuts the series. */
size_t odba_prefix_chop_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                        uint64_t prefix_len);
int odba_prefix_chop_f32(const float *prefix, uint64_t prefix_len, const float *series,
                         const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                         int64_t *chop_positions, int32_t *histograms, void *workspace,
                         size_t workspace_bytes, void *stream);
int odba_prefix_chop_f64(const double *prefix, uint64_t prefix_len, const double *series,
                         const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                         int64_t *chop_positions, int32_t *histograms, void *workspace,
                         size_t workspace_bytes, void *stream);

/* ---- one DBA round for many jobs at once ---------------------------------------
 * No single reference counterpart: DBAUpdate<T> (dba.hpp:432-848) for many
 * independent averaging jobs in one launch sequence (no host synchronization
 * inside, so it can be captured in a CUDA graph and replayed every round).
 * Job J: centroid centroids[centroid_offsets[J] .. + centroid_lens[J]),
 * job_flags[J] bit 0 open start, bit 1 open end, bit 2 active (inactive jobs
 * are skipped and keep their outputs), members job_member_begin[J] ..
 * job_member_end[J]-1 of the member list, in the order their samples are
 * added (the reference's member order).  Member k is series member_series[k]
 * of the series table and belongs to job member_job[k].  member_order
 * (optional) is the order in which members are aligned (longest first keeps
 * the tail short); it does not change any result.  Outputs per job at the
 * job's centroid offset: means, counts; deltas[J] = max |centroid - mean|.
 * The h_* arrays are host copies that size the workspace: only jobs whose
 * h_job_flags have bit 2 set take path and range space, so a large set of
 * jobs can run in waves with a workspace sized for one wave (the device flags
 * of a launch must then activate no job outside the sizing set).  Results
 * equal one odba_dba_round_* call per job, bit for bit.  series may be NULL,
 * with offsets as element addresses (see odba_dtw_pairlist_*). */
size_t odba_dba_batch_workspace_bytes(int elem_size, const uint64_t *h_member_lens,
                                      const int *h_member_job, int nmem,
                                      const uint64_t *h_centroid_lens, const int *h_job_flags,
                                      int njobs);
int odba_dba_batch_round_f32(const float *centroids, const uint64_t *centroid_offsets,
                             const int *centroid_lens, const int *job_flags,
                             const int *job_member_begin, const int *job_member_end, int njobs,
                             int max_centroid_len, const float *series, const uint64_t *offsets,
                             const uint64_t *lens, const int *member_series,
                             const int *member_job, const int *member_order, int nmem,
                             const uint64_t *h_member_lens, const int *h_member_job,
                             const uint64_t *h_centroid_lens, const int *h_job_flags,
                             float *means, uint32_t *counts, double *deltas, int32_t *path_triples,
                             int64_t *path_counts, void *workspace, size_t workspace_bytes,
                             void *stream);
int odba_dba_batch_round_f64(const double *centroids, const uint64_t *centroid_offsets,
                             const int *centroid_lens, const int *job_flags,
                             const int *job_member_begin, const int *job_member_end, int njobs,
                             int max_centroid_len, const double *series, const uint64_t *offsets,
                             const uint64_t *lens, const int *member_series,
                             const int *member_job, const int *member_order, int nmem,
                             const uint64_t *h_member_lens, const int *h_member_job,
                             const uint64_t *h_centroid_lens, const int *h_job_flags,
                             double *means, uint32_t *counts, double *deltas,
                             int32_t *path_triples, int64_t *path_counts, void *workspace,
                             size_t workspace_bytes, void *stream);

/* ---- k-segmentation ------------------------------------------------------------
 * Replaces the kernel part of adaptive_segmentation<T> (adaptive_device_segmentation,
 * segmentation.hpp:48-337; launch segmentation.hpp:440-463).  Every block of
 * 256*ceil(min_segment_length/3) samples of every series gets k_max median slots
 * (k_max = ceil(256 / (min_segment_length / ceil(min_segment_length/3))) as the
 * reference computes it); unused slots hold the type's max.  medians must hold
 * odba_segment_capacity(h_lens, n, min_segment_length) values, series first, then
 * blocks in order.  The host-side merge of block edges and sentinel removal
 * (segmentation.hpp:486-578) is done by adaptive_segmentation<T> in opendba.hpp.
 * The workspace holds n 64-bit offsets. */
size_t odba_segment_capacity(const uint64_t *h_lens, int n, int min_segment_length);
size_t odba_segment_workspace_bytes(int n);
int odba_segment_blocks_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                            const uint64_t *h_lens, int n, int min_segment_length, float *medians,
                            void *workspace, size_t workspace_bytes, void *stream);
int odba_segment_blocks_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                            const uint64_t *h_lens, int n, int min_segment_length, double *medians,
                            void *workspace, size_t workspace_bytes, void *stream);

/* ---- host-buffer medoid pass (end to end) ------------------------------------
 * What performDBA does between its sort and the DBA rounds for one cluster
 * (dba.hpp:902-928 with approximateMedoidIndices): copies the concatenated
 * host series to the device, optionally z-normalises them, computes all pair
 * distances and the medoid, and copies the distances (n(n-1)/2), the medoid
 * index and, when norm != 0, the per-series means and sigmas back.  Host
 * buffers may be pageable or pinned; h_means / h_sigmas may be NULL. */
int odba_medoid_pass_host_f32(const float *h_series, const uint64_t *h_lens, int n,
                              int use_open_start, int use_open_end, int norm, float *h_dists,
                              int *h_medoid, double *h_means, double *h_sigmas, void *stream);
int odba_medoid_pass_host_f64(const double *h_series, const uint64_t *h_lens, int n,
                              int use_open_start, int use_open_end, int norm, double *h_dists,
                              int *h_medoid, double *h_means, double *h_sigmas, void *stream);

/* ---- whole pipeline (the C++ façade in opendba.hpp, callable over FFI) --------
 * odba_perform_dba_*: performDBA<T> (dba.hpp:863-1189) on host series
 * (sorted, z-normalised and truncated in place like the reference does), with
 * algo_mode CLUSTER_ONLY (1), CONSENSUS_ONLY (2) or CLUSTER_AND_CONSENSUS (3);
 * writes <prefix>.pair_dists.txt, <prefix>.avg.txt, per-cluster path and
 * checkpoint files.  odba_setup_and_run: setupAndRun<T> (openDBA.cuh:13-200)
 * for elem_size 4 (float) or 8 (double): reads text / binary / TSV files,
 * optionally segments them, then runs performDBA.  Like the reference, these
 * end the process with its exit codes (exit_codes.hpp) on fatal input/output
 * errors; otherwise they return ODBA_OK.
 * odba_segment_host_*: adaptive_segmentation<T> (segmentation.hpp:340-583) on
 * concatenated host series; h_out needs odba_segment_capacity(...) values and
 * receives each series' segment medians back to back, h_out_lens the counts. */
int odba_perform_dba_f32(float **sequences, int num_sequences, size_t *lengths, char **names,
                         int use_open_start, int use_open_end, const char *output_prefix,
                         int norm, double cdist, int algo_mode);
int odba_perform_dba_f64(double **sequences, int num_sequences, size_t *lengths, char **names,
                         int use_open_start, int use_open_end, const char *output_prefix,
                         int norm, double cdist, int algo_mode);
int odba_setup_and_run(int elem_size, const char *seqprefix_file, char **files, int num_files,
                       const char *output_prefix, int read_mode, int use_open_start,
                       int use_open_end, const char *min_segment_length, int norm, double cdist,
                       int prefix_start, int prefix_length, int is_short);
int odba_segment_host_f32(const float *h_series, const uint64_t *h_lens, int n,
                          int min_segment_length, int prefix_skip, float *h_out,
                          uint64_t *h_out_lens);
int odba_segment_host_f64(const double *h_series, const uint64_t *h_lens, int n,
                          int min_segment_length, int prefix_skip, double *h_out,
                          uint64_t *h_out_lens);

/* ---- many DBA jobs: batched or plain ---------------------------------------------
 * No single reference counterpart: each job is what performDBA<T> computes for
 * one cluster (cdist 1, CLUSTER_AND_CONSENSUS, no files; dba.hpp:863-1146) for
 * the series job_begin[j] .. job_end[j]-1 of the concatenated host input (jobs
 * contiguous and in order), with job_flags[j] bit 0 open start, bit 1 open end.
 * batched != 0: all pairs of all jobs in one length-sorted launch, and each DBA
 * round for every unconverged job as one CUDA-graph replay; batched == 0: job
 * by job through the single-job entry points (the drop-in path).  Both give the
 * same results.  Outputs per job: h_medoids[j] (index within the job's input
 * order), its centroid at h_centroids[h_centroid_offsets[j]] with the medoid's
 * length (capacity: the sum over jobs of the longest series), rounds run and
 * the last delta.  max_rounds <= 0 means the reference's 250.  Returns
 * ODBA_ERR_TIMEOUT if a swath hand-off wait ran out on the device. */
int odba_dba_jobs_f32(const float *h_series, const uint64_t *h_lens, const int *job_begin,
                      const int *job_end, const int *job_flags, int njobs, int norm,
                      int max_rounds, int batched, int *h_medoids, uint64_t *h_centroid_offsets,
                      float *h_centroids, int *h_rounds, double *h_deltas, void *stream);
int odba_dba_jobs_f64(const double *h_series, const uint64_t *h_lens, const int *job_begin,
                      const int *job_end, const int *job_flags, int njobs, int norm,
                      int max_rounds, int batched, int *h_medoids, uint64_t *h_centroid_offsets,
                      double *h_centroids, int *h_rounds, double *h_deltas, void *stream);

/* ---- serving loop with continuous batching -----------------------------------
 * No reference counterpart.  A server owns a worker thread on one device that
 * batches whatever requests are admitted: each iteration runs one pair-list
 * launch (every admitted query's pairs, every job's medoid pairs) and one
 * batched DBA round (every job in its round stage); requests that arrive
 * meanwhile join the next iteration; requests are admitted in arrival order
 * while the estimated device memory of all admitted work stays under
 * hbm_budget_bytes (one request is always admitted).  Centroids added with
 * odba_server_add_centroid stay resident.  A query aligns each of nreads reads
 * (first series) to each listed centroid (second series) and returns nreads x
 * ncentroids pair distances, row-major; a job is performDBA for one cluster
 * (see odba_dba_jobs_*) and returns the centroid.  Results do not depend on
 * what else was batched.  submit returns a request id (> 0) or -status; poll
 * returns 0 running, 1 done, -status failed; wait blocks up to timeout_s;
 * take copies the result out (capacity in elements) and forgets the request. */
void *odba_server_create(int elem_size, size_t hbm_budget_bytes, int device);
void odba_server_destroy(void *server);
int odba_server_add_centroid(void *server, const void *h_centroid, uint64_t len);
int64_t odba_server_submit_query(void *server, const void *h_reads, const uint64_t *h_read_lens,
                                 int nreads, const int *centroid_ids, int ncentroids, int flags);
int64_t odba_server_submit_job(void *server, const void *h_series, const uint64_t *h_lens, int n,
                               int flags, int norm);
int odba_server_poll(void *server, int64_t request);
int odba_server_wait(void *server, int64_t request, double timeout_s);
int odba_server_take(void *server, int64_t request, void *h_out, uint64_t capacity,
                     uint64_t *out_len, int *medoid, int *rounds, double *latency_s);
int odba_server_stats(void *server, uint64_t *iterations, uint64_t *cells, double *busy_s);

#ifdef __cplusplus
}
#endif

#endif /* OPENDBA_B200_H */
