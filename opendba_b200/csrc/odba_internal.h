// Internal declarations shared by the CUDA translation units of
// libopendba_b200.so.  Nothing here is part of the public C ABI
// (include/opendba_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "opendba_b200.h"

namespace odba {

// Records a failure in the calling thread's error slot and returns status.
int fail(int status, const char *msg);
// Checks cudaGetLastError() after a launch; returns ODBA_OK or ODBA_ERR_CUDA.
int check_launch(const char *what);
// Returns ODBA_OK if the current device is a compute capability 10.x part.
int require_sm100();

template <typename T>
size_t pairwise_workspace_bytes(uint64_t max_len);
template <typename T>
int pairwise_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                    uint64_t max_len, int os, int oe, T *dists, void *workspace, size_t ws_bytes,
                    cudaStream_t stream);

template <typename T>
int pairwise_range_launch(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                          uint64_t max_len, int os, int oe, unsigned long long pbeg,
                          unsigned long long pend, T *dists, void *workspace, size_t ws_bytes,
                          cudaStream_t stream);
template <typename T>
size_t pairwise_workspace_bytes_n(unsigned long long npairs, uint64_t max_len);

// Autotuner of the pair kernels' launch plan (ODBA_PLAN_*).
int tune_set(int elem_size, int len_bucket, int count_bucket, int plan);
int tune_query(int elem_size, uint64_t max_len, unsigned long long npairs, size_t ws_bytes, int *plan,
               double *rates);
void tune_mode(int on);
int tune_flush();
int tune_save(const char *path);
int tune_load(const char *path);
// Runs the swath pipeline's bounded wait on a word nothing publishes.
int gate_selftest(unsigned long long limit_ns, cudaStream_t stream);

template <typename T>
int pairlist_launch(const T *series, const uint64_t *offsets, const uint64_t *lens,
                    const odba_pair_task *tasks, unsigned long long ntasks, uint64_t max_len,
                    T *dists, void *workspace, size_t ws_bytes, cudaStream_t stream);

// Complete linkage and dendrogram cuts (clustering.cpp, host code).
void complete_linkage(int n, double *D, int *merge, double *height);
void cut_tree_k(int n, const int *merge, int k, int *labels);
void cut_tree_height(int n, const int *merge, const double *height, double cdist, int *labels);
template <typename T>
int cluster_and_medoids(int n, const T *dists, const uint64_t *lens, double cdist, int *memberships,
                        int *medoids);

template <typename T>
int medoid_launch(const T *dists, const uint64_t *lens, int n, T *sos, int *medoid,
                  cudaStream_t stream);

template <typename T>
int znorm_launch(T *series, const uint64_t *offsets, const uint64_t *lens, int n, double *means,
                 double *sigmas, cudaStream_t stream);

template <typename T>
size_t dba_round_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe);
template <typename T>
int dba_round_launch(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                     const uint64_t *lens, const uint64_t *h_lens, int n, int os, int oe, T *mean,
                     uint32_t *counts, double *delta, int32_t *triples, int64_t *triple_counts,
                     void *ws, size_t ws_bytes, cudaStream_t stream);

template <typename T>
int dba_round_ranges_launch(const T *centroid, uint64_t Lc, const T *series,
                            const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                            int n, int os, int oe, int2 *ranges_out, void *ws, size_t ws_bytes,
                            cudaStream_t stream);
template <typename T>
size_t dba_reduce_workspace_bytes(int n);
// Row bands of the round's swath pipeline: n in 1..8 pins the count, 0 lets
// each launch choose it.  Returns the previous setting.
int dba_round_bands(int n);
template <typename T>
int dba_reduce_ranges_launch(const T *centroid, uint64_t Lc, const T *series,
                             const uint64_t *offsets, const uint64_t *lens, int n, int os, int oe,
                             const int2 *ranges, T *mean, uint32_t *counts, double *delta, void *ws,
                             size_t ws_bytes, cudaStream_t stream);

template <typename T>
size_t dba_round_stripe_workspace_bytes(const uint64_t *h_lens, int n, uint64_t Lc, int os, int oe,
                                        int ckpt_rows);
template <typename T>
int dba_round_stripe_launch(const T *centroid, uint64_t Lc, const T *series,
                            const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                            int n, int os, int oe, int ckpt_rows, T *mean, uint32_t *counts,
                            double *delta, int32_t *triples, int64_t *triple_counts, void *ws,
                            size_t ws_bytes, cudaStream_t stream);

template <typename T>
size_t prefix_chop_workspace_bytes(const uint64_t *h_lens, int n, uint64_t P);
template <typename T>
int prefix_chop_launch(const T *prefix, uint64_t P, const T *series, const uint64_t *offsets,
                       const uint64_t *lens, const uint64_t *h_lens, int n, long long *chop,
                       int *hist, void *ws, size_t ws_bytes, cudaStream_t stream);

template <typename T>
size_t dba_batch_workspace_bytes(const uint64_t *h_mlens, const int *h_mjob, int nmem,
                                 const uint64_t *h_clen, const int *h_flags, int njobs);
template <typename T>
int dba_batch_launch(const T *centroids, const unsigned long long *coff, const int *clen,
                     const int *jflags, const int *mbeg, const int *mend, int njobs, int max_clen,
                     const T *series, const uint64_t *offsets, const uint64_t *lens,
                     const int *mseries, const int *mjob, const int *order, int nmem,
                     const uint64_t *h_mlens, const int *h_mjob, const uint64_t *h_clen,
                     const int *h_flags, T *means, uint32_t *counts, double *deltas,
                     int32_t *triples, int64_t *triple_counts, void *ws, size_t ws_bytes,
                     cudaStream_t stream);

void segment_params(int minseg, int *dw, int *spb, int *k_max);
template <typename T>
int segment_blocks(const T *series, const uint64_t *offsets, const uint64_t *lens,
                   const uint64_t *h_lens, int n, int minseg, T *medians, void *ws,
                   size_t ws_bytes, cudaStream_t stream);

}  // namespace odba
