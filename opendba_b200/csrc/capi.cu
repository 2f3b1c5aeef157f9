// The extern "C" surface of libopendba_b200.so (include/opendba_b200.h):
// argument validation, error reporting and the host-buffer entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "odba_internal.h"

namespace odba {

namespace {
thread_local char g_err[512] = "";
}

int fail(int status, const char *msg) {
  std::snprintf(g_err, sizeof(g_err), "%s", msg);
  return status;
}

int check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return ODBA_OK;
  char buf[400];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  return fail(e == cudaErrorMemoryAllocation ? ODBA_ERR_OUT_OF_MEMORY : ODBA_ERR_CUDA, buf);
}

int require_sm100() {
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
    return fail(ODBA_ERR_CUDA, "no CUDA device available");
  if (major != 10) return fail(ODBA_ERR_UNSUPPORTED_DEVICE, "requires a compute capability 10.x (sm_100a) device");
  return ODBA_OK;
}

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  char buf[400];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  return fail(e == cudaErrorMemoryAllocation ? ODBA_ERR_OUT_OF_MEMORY : ODBA_ERR_CUDA, buf);
}

#define ODBA_CUDA(call, what)                       \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

template <typename T>
int pairwise_checked(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                     uint64_t max_len, int os, int oe, T *dists, void *ws, size_t ws_bytes,
                     void *stream) {
  if (n < 0 || (n >= 2 && (!series || !offsets || !lens || !dists || !ws)))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or negative series count");
  if (max_len == 0 || max_len > (1ull << 31))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "max_len must be in [1, 2^31]");
  if (int rc = require_sm100()) return rc;
  return pairwise_launch<T>(series, offsets, lens, n, max_len, os ? 1 : 0, oe ? 1 : 0, dists, ws,
                            ws_bytes, static_cast<cudaStream_t>(stream));
}

template <typename T>
int pairwise_range_checked(const T *series, const uint64_t *offsets, const uint64_t *lens, int n,
                           uint64_t max_len, int os, int oe, uint64_t pbeg, uint64_t pend, T *dists,
                           void *ws, size_t ws_bytes, void *stream) {
  const unsigned long long npairs = n > 1 ? (unsigned long long)n * (n - 1) / 2 : 0;
  if (pbeg > pend || pend > npairs)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "pair range outside the upper triangle");
  if (n < 0 || (pend > pbeg && (!series || !offsets || !lens || !dists || !ws)))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or negative series count");
  if (max_len == 0 || max_len > (1ull << 31))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "max_len must be in [1, 2^31]");
  if (int rc = require_sm100()) return rc;
  return pairwise_range_launch<T>(series, offsets, lens, n, max_len, os ? 1 : 0, oe ? 1 : 0, pbeg,
                                  pend, dists, ws, ws_bytes, static_cast<cudaStream_t>(stream));
}

template <typename T>
int medoid_pass_host(const T *h_series, const uint64_t *h_lens, int n, int os, int oe, int norm,
                     T *h_dists, int *h_medoid, double *h_means, double *h_sigmas, void *stream_v) {
  if (n < 1 || !h_series || !h_lens || !h_medoid || (n >= 2 && !h_dists))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  if (int rc = require_sm100()) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
  std::vector<uint64_t> offs(n);
  uint64_t total = 0, max_len = 0;
  for (int i = 0; i < n; ++i) {
    if (h_lens[i] == 0) return fail(ODBA_ERR_INVALID_ARGUMENT, "every series needs at least one sample");
    offs[i] = total;
    total += h_lens[i];
    if (h_lens[i] > max_len) max_len = h_lens[i];
  }
  const size_t npairs = size_t(n) * (n - 1) / 2;
  const size_t ws_bytes = pairwise_workspace_bytes_n<T>(npairs, max_len);
  // one device allocation: series | offsets | lens | dists | sos | means | sigmas | medoid | workspace
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_series = up((total + 16) * sizeof(T)), b_meta = up(n * sizeof(uint64_t)),
               b_d = up((npairs + 1) * sizeof(T)), b_sos = up(n * sizeof(T)),
               b_mv = up(n * sizeof(double)), b_med = 256;
  const size_t bytes = b_series + 2 * b_meta + b_d + b_sos + 2 * b_mv + b_med + ws_bytes;
  char *base = nullptr;
  ODBA_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&base), bytes, stream), "device allocation");
  T *d_series = reinterpret_cast<T *>(base);
  uint64_t *d_offs = reinterpret_cast<uint64_t *>(base + b_series);
  uint64_t *d_lens = reinterpret_cast<uint64_t *>(base + b_series + b_meta);
  T *d_dists = reinterpret_cast<T *>(base + b_series + 2 * b_meta);
  T *d_sos = reinterpret_cast<T *>(base + b_series + 2 * b_meta + b_d);
  double *d_means = reinterpret_cast<double *>(base + b_series + 2 * b_meta + b_d + b_sos);
  double *d_sigmas = d_means + b_mv / sizeof(double);
  int *d_medoid = reinterpret_cast<int *>(base + b_series + 2 * b_meta + b_d + b_sos + 2 * b_mv);
  void *d_ws = base + b_series + 2 * b_meta + b_d + b_sos + 2 * b_mv + b_med;
  int rc = ODBA_OK;
  unsigned wait_err = 0;
  auto run = [&]() -> int {
    ODBA_CUDA(cudaMemcpyAsync(d_series, h_series, total * sizeof(T), cudaMemcpyHostToDevice, stream),
              "series upload");
    ODBA_CUDA(cudaMemcpyAsync(d_offs, offs.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, stream),
              "offsets upload");
    ODBA_CUDA(cudaMemcpyAsync(d_lens, h_lens, n * sizeof(uint64_t), cudaMemcpyHostToDevice, stream),
              "lengths upload");
    if (norm) {
      if (int r = znorm_launch<T>(d_series, d_offs, d_lens, n, d_means, d_sigmas, stream)) return r;
    }
    if (n >= 2) {
      if (int r = pairwise_launch<T>(d_series, d_offs, d_lens, n, max_len, os ? 1 : 0, oe ? 1 : 0,
                                     d_dists, d_ws, ws_bytes, stream))
        return r;
    }
    if (int r = medoid_launch<T>(d_dists, d_lens, n, d_sos, d_medoid, stream)) return r;
    if (n >= 2)
      ODBA_CUDA(cudaMemcpyAsync(h_dists, d_dists, npairs * sizeof(T), cudaMemcpyDeviceToHost, stream),
                "distance download");
    ODBA_CUDA(cudaMemcpyAsync(h_medoid, d_medoid, sizeof(int), cudaMemcpyDeviceToHost, stream),
              "medoid download");
    if (norm && h_means)
      ODBA_CUDA(cudaMemcpyAsync(h_means, d_means, n * sizeof(double), cudaMemcpyDeviceToHost, stream),
                "means download");
    if (norm && h_sigmas)
      ODBA_CUDA(cudaMemcpyAsync(h_sigmas, d_sigmas, n * sizeof(double), cudaMemcpyDeviceToHost, stream),
                "sigmas download");
    if (n >= 2)
      ODBA_CUDA(cudaMemcpyAsync(&wait_err, static_cast<char *>(d_ws) + 8, sizeof(unsigned),
                                cudaMemcpyDeviceToHost, stream),
                "error word download");
    ODBA_CUDA(cudaStreamSynchronize(stream), "medoid pass");
    if (wait_err) return fail(ODBA_ERR_TIMEOUT, "a swath hand-off wait ran out in the pair kernel");
    return ODBA_OK;
  };
  rc = run();
  cudaFreeAsync(base, stream);
  if (rc == ODBA_OK) ODBA_CUDA(cudaStreamSynchronize(stream), "medoid pass teardown");
  return rc;
}

template <typename T>
int dba_round_checked(const T *centroid, uint64_t Lc, const T *series,
                             const uint64_t *offsets, const uint64_t *lens,
                             const uint64_t *h_lens, int n, int os, int oe, T *mean,
                             uint32_t *counts, double *delta, int32_t *triples,
                             int64_t *triple_counts, void *ws, size_t ws_bytes, void *stream,
                             int ckpt_rows = -1) {
  if (n < 1 || Lc == 0 || !centroid || !series || !offsets || !lens || !h_lens || !mean ||
      !counts || !delta || !ws)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer, empty centroid or no members");
  if ((triples == nullptr) != (triple_counts == nullptr))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "path triples and their counts go together");
  for (int k = 0; k < n; ++k)
    if (h_lens[k] == 0 || h_lens[k] > (1ull << 30))
      return fail(ODBA_ERR_INVALID_ARGUMENT, "member lengths must be in [1, 2^30]");
  if (Lc > (1ull << 30)) return fail(ODBA_ERR_INVALID_ARGUMENT, "centroid too long");
  if (int rc = require_sm100()) return rc;
  if (ckpt_rows >= 0)
    return dba_round_stripe_launch<T>(centroid, Lc, series, offsets, lens, h_lens, n, os ? 1 : 0,
                                      oe ? 1 : 0, ckpt_rows, mean, counts, delta, triples,
                                      triple_counts, ws, ws_bytes, static_cast<cudaStream_t>(stream));
  return dba_round_launch<T>(centroid, Lc, series, offsets, lens, h_lens, n, os ? 1 : 0,
                             oe ? 1 : 0, mean, counts, delta, triples, triple_counts, ws,
                             ws_bytes, static_cast<cudaStream_t>(stream));
}

template <typename T>
int dba_ranges_checked(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                       const uint64_t *lens, const uint64_t *h_lens, int n, int os, int oe,
                       int32_t *ranges, void *ws, size_t ws_bytes, void *stream) {
  if (n < 1 || Lc == 0 || !centroid || !series || !offsets || !lens || !h_lens || !ranges || !ws)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer, empty centroid or no members");
  for (int k = 0; k < n; ++k)
    if (h_lens[k] == 0 || h_lens[k] > (1ull << 30))
      return fail(ODBA_ERR_INVALID_ARGUMENT, "member lengths must be in [1, 2^30]");
  if (Lc > (1ull << 30)) return fail(ODBA_ERR_INVALID_ARGUMENT, "centroid too long");
  if (int rc = require_sm100()) return rc;
  return dba_round_ranges_launch<T>(centroid, Lc, series, offsets, lens, h_lens, n, os ? 1 : 0,
                                    oe ? 1 : 0, reinterpret_cast<int2 *>(ranges), ws, ws_bytes,
                                    static_cast<cudaStream_t>(stream));
}

template <typename T>
int dba_reduce_checked(const T *centroid, uint64_t Lc, const T *series, const uint64_t *offsets,
                       const uint64_t *lens, int n, int os, int oe, const int32_t *ranges, T *mean,
                       uint32_t *counts, double *delta, void *ws, size_t ws_bytes, void *stream) {
  if (n < 1 || Lc == 0 || !centroid || !series || !offsets || !lens || !ranges || !mean ||
      !counts || !delta || !ws)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer, empty centroid or no members");
  if (Lc > (1ull << 30)) return fail(ODBA_ERR_INVALID_ARGUMENT, "centroid too long");
  if (int rc = require_sm100()) return rc;
  return dba_reduce_ranges_launch<T>(centroid, Lc, series, offsets, lens, n, os ? 1 : 0, oe ? 1 : 0,
                                     reinterpret_cast<const int2 *>(ranges), mean, counts, delta, ws,
                                     ws_bytes, static_cast<cudaStream_t>(stream));
}

template <typename T>
int prefix_chop_checked(const T *prefix, uint64_t P, const T *series, const uint64_t *offsets,
                               const uint64_t *lens, const uint64_t *h_lens, int n, int64_t *chop,
                               int32_t *hist, void *ws, size_t ws_bytes, void *stream) {
  if (n < 1 || P == 0 || !prefix || !series || !offsets || !lens || !h_lens || !chop || !hist || !ws)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer, empty prefix or no series");
  if (P > (1ull << 30)) return fail(ODBA_ERR_INVALID_ARGUMENT, "prefix too long");
  for (int k = 0; k < n; ++k)
    if (h_lens[k] == 0 || h_lens[k] > (1ull << 30))
      return fail(ODBA_ERR_INVALID_ARGUMENT, "series lengths must be in [1, 2^30]");
  if (int rc = require_sm100()) return rc;
  return prefix_chop_launch<T>(prefix, P, series, offsets, lens, h_lens, n,
                               reinterpret_cast<long long *>(chop), hist, ws, ws_bytes,
                               static_cast<cudaStream_t>(stream));
}

}  // namespace
}  // namespace odba

using namespace odba;

extern "C" {

int odba_abi_version(void) { return ODBA_ABI_VERSION; }

const char *odba_status_string(int status) {
  switch (status) {
    case ODBA_OK: return "ok";
    case ODBA_ERR_INVALID_ARGUMENT: return "invalid argument";
    case ODBA_ERR_CUDA: return "CUDA error";
    case ODBA_ERR_OUT_OF_MEMORY: return "out of device memory";
    case ODBA_ERR_WORKSPACE_TOO_SMALL: return "workspace too small";
    case ODBA_ERR_UNSUPPORTED_DEVICE: return "unsupported device";
    case ODBA_ERR_TIMEOUT: return "timed out";
    case ODBA_ERR_IO: return "I/O error";
    default: return "unknown status";
  }
}

const char *odba_last_error(void) { return odba::g_err; }

int odba_device_check(void) { return require_sm100(); }

size_t odba_dtw_pairwise_workspace_bytes(int elem_size, uint64_t max_len) {
  if (elem_size == 8) return pairwise_workspace_bytes<double>(max_len);
  return pairwise_workspace_bytes<float>(max_len);
}

size_t odba_dtw_pairwise_workspace_bytes_n(int elem_size, int n, uint64_t max_len) {
  const unsigned long long npairs = n > 1 ? (unsigned long long)n * (n - 1) / 2 : 0;
  if (elem_size == 8) return pairwise_workspace_bytes_n<double>(npairs, max_len);
  return pairwise_workspace_bytes_n<float>(npairs, max_len);
}

int odba_tune_set(int elem_size, int len_bucket, int count_bucket, int plan) {
  return tune_set(elem_size, len_bucket, count_bucket, plan);
}

int odba_tune_query(int elem_size, uint64_t max_len, uint64_t npairs, size_t workspace_bytes,
                    int *plan, double *rates) {
  return tune_query(elem_size, max_len, npairs, workspace_bytes, plan, rates);
}

void odba_tune_mode(int on) { tune_mode(on); }

int odba_tune_flush(void) { return tune_flush(); }

int odba_tune_save(const char *path) {
  if (!path) return fail(ODBA_ERR_INVALID_ARGUMENT, "null path");
  return tune_save(path);
}

int odba_tune_load(const char *path) {
  if (!path) return fail(ODBA_ERR_INVALID_ARGUMENT, "null path");
  return tune_load(path);
}

int odba_selftest_wait_timeout(uint64_t limit_ns, void *stream) {
  return gate_selftest(limit_ns, static_cast<cudaStream_t>(stream));
}

int odba_dtw_pairwise_range_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                                int n, uint64_t max_len, int use_open_start, int use_open_end,
                                uint64_t pair_begin, uint64_t pair_end, float *dists,
                                void *workspace, size_t workspace_bytes, void *stream) {
  return pairwise_range_checked<float>(series, offsets, lens, n, max_len, use_open_start,
                                       use_open_end, pair_begin, pair_end, dists, workspace,
                                       workspace_bytes, stream);
}

int odba_dtw_pairwise_range_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                                int n, uint64_t max_len, int use_open_start, int use_open_end,
                                uint64_t pair_begin, uint64_t pair_end, double *dists,
                                void *workspace, size_t workspace_bytes, void *stream) {
  return pairwise_range_checked<double>(series, offsets, lens, n, max_len, use_open_start,
                                        use_open_end, pair_begin, pair_end, dists, workspace,
                                        workspace_bytes, stream);
}

int odba_dtw_pairwise_f32(const float *series, const uint64_t *offsets, const uint64_t *lens, int n,
                          uint64_t max_len, int use_open_start, int use_open_end, float *dists,
                          void *workspace, size_t workspace_bytes, void *stream) {
  return pairwise_checked<float>(series, offsets, lens, n, max_len, use_open_start, use_open_end,
                                 dists, workspace, workspace_bytes, stream);
}

int odba_dtw_pairwise_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                          int n, uint64_t max_len, int use_open_start, int use_open_end,
                          double *dists, void *workspace, size_t workspace_bytes, void *stream) {
  return pairwise_checked<double>(series, offsets, lens, n, max_len, use_open_start, use_open_end,
                                  dists, workspace, workspace_bytes, stream);
}

int odba_medoid_f32(const float *dists, const uint64_t *lens, int n, float *sos, int *medoid,
                    void *stream) {
  if (n < 1 || !lens || !sos || !medoid || (n >= 2 && !dists))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  if (int rc = require_sm100()) return rc;
  return medoid_launch<float>(dists, lens, n, sos, medoid, static_cast<cudaStream_t>(stream));
}

int odba_medoid_f64(const double *dists, const uint64_t *lens, int n, double *sos, int *medoid,
                    void *stream) {
  if (n < 1 || !lens || !sos || !medoid || (n >= 2 && !dists))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty input");
  if (int rc = require_sm100()) return rc;
  return medoid_launch<double>(dists, lens, n, sos, medoid, static_cast<cudaStream_t>(stream));
}

int odba_znorm_f32(float *series, const uint64_t *offsets, const uint64_t *lens, int n,
                   double *means, double *sigmas, void *stream) {
  if (n < 0 || (n > 0 && (!series || !offsets || !lens)))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or negative series count");
  if (int rc = require_sm100()) return rc;
  return znorm_launch<float>(series, offsets, lens, n, means, sigmas, static_cast<cudaStream_t>(stream));
}

int odba_znorm_f64(double *series, const uint64_t *offsets, const uint64_t *lens, int n,
                   double *means, double *sigmas, void *stream) {
  if (n < 0 || (n > 0 && (!series || !offsets || !lens)))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or negative series count");
  if (int rc = require_sm100()) return rc;
  return znorm_launch<double>(series, offsets, lens, n, means, sigmas, static_cast<cudaStream_t>(stream));
}

int odba_medoid_pass_host_f32(const float *h_series, const uint64_t *h_lens, int n,
                              int use_open_start, int use_open_end, int norm, float *h_dists,
                              int *h_medoid, double *h_means, double *h_sigmas, void *stream) {
  return medoid_pass_host<float>(h_series, h_lens, n, use_open_start, use_open_end, norm, h_dists,
                                 h_medoid, h_means, h_sigmas, stream);
}

int odba_medoid_pass_host_f64(const double *h_series, const uint64_t *h_lens, int n,
                              int use_open_start, int use_open_end, int norm, double *h_dists,
                              int *h_medoid, double *h_means, double *h_sigmas, void *stream) {
  return medoid_pass_host<double>(h_series, h_lens, n, use_open_start, use_open_end, norm, h_dists,
                                  h_medoid, h_means, h_sigmas, stream);
}

int odba_dtw_pairlist_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                          const odba_pair_task *tasks, uint64_t ntasks, uint64_t max_len,
                          float *dists, void *workspace, size_t workspace_bytes, void *stream) {
  if (ntasks && (!offsets || !lens || !tasks || !dists || !workspace))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer");
  if (max_len == 0 || max_len > (1ull << 31)) return fail(ODBA_ERR_INVALID_ARGUMENT, "max_len must be in [1, 2^31]");
  if (int rc = require_sm100()) return rc;
  return pairlist_launch<float>(series, offsets, lens, tasks, ntasks, max_len, dists, workspace,
                                workspace_bytes, static_cast<cudaStream_t>(stream));
}

int odba_dtw_pairlist_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                          const odba_pair_task *tasks, uint64_t ntasks, uint64_t max_len,
                          double *dists, void *workspace, size_t workspace_bytes, void *stream) {
  if (ntasks && (!offsets || !lens || !tasks || !dists || !workspace))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer");
  if (max_len == 0 || max_len > (1ull << 31)) return fail(ODBA_ERR_INVALID_ARGUMENT, "max_len must be in [1, 2^31]");
  if (int rc = require_sm100()) return rc;
  return pairlist_launch<double>(series, offsets, lens, tasks, ntasks, max_len, dists, workspace,
                                 workspace_bytes, static_cast<cudaStream_t>(stream));
}

size_t odba_dba_round_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                      uint64_t centroid_len, int use_open_start, int use_open_end) {
  if (n < 1 || !h_lens || centroid_len == 0) return 0;
  if (elem_size == 8)
    return dba_round_workspace_bytes<double>(h_lens, n, centroid_len, use_open_start, use_open_end);
  return dba_round_workspace_bytes<float>(h_lens, n, centroid_len, use_open_start, use_open_end);
}

int odba_dba_round_f32(const float *centroid, uint64_t centroid_len, const float *series,
                       const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                       int use_open_start, int use_open_end, float *new_centroid, uint32_t *counts,
                       double *delta, int32_t *path_triples, int64_t *path_counts,
                       void *workspace, size_t workspace_bytes, void *stream) {
  return dba_round_checked<float>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                  use_open_start, use_open_end, new_centroid, counts, delta,
                                  path_triples, path_counts, workspace, workspace_bytes, stream);
}

int odba_dba_round_f64(const double *centroid, uint64_t centroid_len, const double *series,
                       const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                       int use_open_start, int use_open_end, double *new_centroid,
                       uint32_t *counts, double *delta, int32_t *path_triples,
                       int64_t *path_counts, void *workspace, size_t workspace_bytes,
                       void *stream) {
  return dba_round_checked<double>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                   use_open_start, use_open_end, new_centroid, counts, delta,
                                   path_triples, path_counts, workspace, workspace_bytes, stream);
}

int odba_dba_round_ranges_f32(const float *centroid, uint64_t centroid_len, const float *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int32_t *ranges,
                              void *workspace, size_t workspace_bytes, void *stream) {
  return dba_ranges_checked<float>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                   use_open_start, use_open_end, ranges, workspace, workspace_bytes,
                                   stream);
}

int odba_dba_round_ranges_f64(const double *centroid, uint64_t centroid_len, const double *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int32_t *ranges,
                              void *workspace, size_t workspace_bytes, void *stream) {
  return dba_ranges_checked<double>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                    use_open_start, use_open_end, ranges, workspace, workspace_bytes,
                                    stream);
}

int odba_round_set_bands(int n) {
  if (n < 0 || n > 8) return fail(ODBA_ERR_INVALID_ARGUMENT, "band count must be 0..8");
  dba_round_bands(n);
  return ODBA_OK;
}

size_t odba_dba_reduce_workspace_bytes(int elem_size, int n) {
  if (n < 1) return 0;
  return elem_size == 8 ? dba_reduce_workspace_bytes<double>(n) : dba_reduce_workspace_bytes<float>(n);
}

int odba_dba_reduce_ranges_f32(const float *centroid, uint64_t centroid_len, const float *series,
                               const uint64_t *offsets, const uint64_t *lens, int n,
                               int use_open_start, int use_open_end, const int32_t *ranges,
                               float *new_centroid, uint32_t *counts, double *delta,
                               void *workspace, size_t workspace_bytes, void *stream) {
  return dba_reduce_checked<float>(centroid, centroid_len, series, offsets, lens, n, use_open_start,
                                   use_open_end, ranges, new_centroid, counts, delta, workspace,
                                   workspace_bytes, stream);
}

int odba_dba_reduce_ranges_f64(const double *centroid, uint64_t centroid_len, const double *series,
                               const uint64_t *offsets, const uint64_t *lens, int n,
                               int use_open_start, int use_open_end, const int32_t *ranges,
                               double *new_centroid, uint32_t *counts, double *delta,
                               void *workspace, size_t workspace_bytes, void *stream) {
  return dba_reduce_checked<double>(centroid, centroid_len, series, offsets, lens, n,
                                    use_open_start, use_open_end, ranges, new_centroid, counts, delta,
                                    workspace, workspace_bytes, stream);
}

size_t odba_dba_round_stripe_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                             uint64_t centroid_len, int use_open_start,
                                             int use_open_end, int ckpt_rows) {
  if (n < 1 || !h_lens || centroid_len == 0) return 0;
  const int os = use_open_start ? 1 : 0, oe = use_open_end ? 1 : 0;
  if (elem_size == 8)
    return dba_round_stripe_workspace_bytes<double>(h_lens, n, centroid_len, os, oe, ckpt_rows);
  return dba_round_stripe_workspace_bytes<float>(h_lens, n, centroid_len, os, oe, ckpt_rows);
}

int odba_dba_round_stripe_f32(const float *centroid, uint64_t centroid_len, const float *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int ckpt_rows,
                              float *new_centroid, uint32_t *counts, double *delta,
                              int32_t *path_triples, int64_t *path_counts, void *workspace,
                              size_t workspace_bytes, void *stream) {
  if (ckpt_rows < 0) return fail(ODBA_ERR_INVALID_ARGUMENT, "checkpoint rows must be >= 0");
  return dba_round_checked<float>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                  use_open_start, use_open_end, new_centroid, counts, delta,
                                  path_triples, path_counts, workspace, workspace_bytes, stream,
                                  ckpt_rows);
}

int odba_dba_round_stripe_f64(const double *centroid, uint64_t centroid_len, const double *series,
                              const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens,
                              int n, int use_open_start, int use_open_end, int ckpt_rows,
                              double *new_centroid, uint32_t *counts, double *delta,
                              int32_t *path_triples, int64_t *path_counts, void *workspace,
                              size_t workspace_bytes, void *stream) {
  if (ckpt_rows < 0) return fail(ODBA_ERR_INVALID_ARGUMENT, "checkpoint rows must be >= 0");
  return dba_round_checked<double>(centroid, centroid_len, series, offsets, lens, h_lens, n,
                                   use_open_start, use_open_end, new_centroid, counts, delta,
                                   path_triples, path_counts, workspace, workspace_bytes, stream,
                                   ckpt_rows);
}

size_t odba_prefix_chop_workspace_bytes(int elem_size, const uint64_t *h_lens, int n,
                                        uint64_t prefix_len) {
  if (n < 1 || !h_lens || prefix_len == 0) return 0;
  if (elem_size == 8) return prefix_chop_workspace_bytes<double>(h_lens, n, prefix_len);
  return prefix_chop_workspace_bytes<float>(h_lens, n, prefix_len);
}

int odba_prefix_chop_f32(const float *prefix, uint64_t prefix_len, const float *series,
                         const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                         int64_t *chop_positions, int32_t *histograms, void *workspace,
                         size_t workspace_bytes, void *stream) {
  return prefix_chop_checked<float>(prefix, prefix_len, series, offsets, lens, h_lens, n,
                                    chop_positions, histograms, workspace, workspace_bytes, stream);
}

int odba_prefix_chop_f64(const double *prefix, uint64_t prefix_len, const double *series,
                         const uint64_t *offsets, const uint64_t *lens, const uint64_t *h_lens, int n,
                         int64_t *chop_positions, int32_t *histograms, void *workspace,
                         size_t workspace_bytes, void *stream) {
  return prefix_chop_checked<double>(prefix, prefix_len, series, offsets, lens, h_lens, n,
                                     chop_positions, histograms, workspace, workspace_bytes, stream);
}

size_t odba_dba_batch_workspace_bytes(int elem_size, const uint64_t *h_member_lens,
                                      const int *h_member_job, int nmem,
                                      const uint64_t *h_centroid_lens, const int *h_job_flags,
                                      int njobs) {
  if (nmem < 1 || njobs < 1 || !h_member_lens || !h_member_job || !h_centroid_lens || !h_job_flags)
    return 0;
  if (elem_size == 8)
    return dba_batch_workspace_bytes<double>(h_member_lens, h_member_job, nmem, h_centroid_lens,
                                             h_job_flags, njobs);
  return dba_batch_workspace_bytes<float>(h_member_lens, h_member_job, nmem, h_centroid_lens,
                                          h_job_flags, njobs);
}

#define ODBA_BATCH_ROUND(SFX, T)                                                               \
  int odba_dba_batch_round_##SFX(                                                              \
      const T *centroids, const uint64_t *centroid_offsets, const int *centroid_lens,          \
      const int *job_flags, const int *job_member_begin, const int *job_member_end, int njobs, \
      int max_centroid_len, const T *series, const uint64_t *offsets, const uint64_t *lens,    \
      const int *member_series, const int *member_job, const int *member_order, int nmem,      \
      const uint64_t *h_member_lens, const int *h_member_job, const uint64_t *h_centroid_lens, \
      const int *h_job_flags, T *means, uint32_t *counts, double *deltas, int32_t *path_triples, \
      int64_t *path_counts, void *workspace, size_t workspace_bytes, void *stream) {           \
    if (njobs < 1 || nmem < 1 || max_centroid_len < 1 || !centroids || !centroid_offsets ||    \
        !centroid_lens || !job_flags || !job_member_begin || !job_member_end ||                \
        !offsets || !lens || !member_series || !member_job || !h_member_lens ||                \
        !h_member_job || !h_centroid_lens || !h_job_flags || !means || !counts || !deltas ||   \
        !workspace)                                                                            \
      return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or empty batch");                   \
    if ((path_triples == nullptr) != (path_counts == nullptr))                                 \
      return fail(ODBA_ERR_INVALID_ARGUMENT, "path triples and their counts go together");     \
    for (int k = 0; k < nmem; ++k)                                                             \
      if (h_member_lens[k] == 0 || h_member_lens[k] > (1ull << 30) || h_member_job[k] < 0 ||   \
          h_member_job[k] >= njobs)                                                            \
        return fail(ODBA_ERR_INVALID_ARGUMENT, "bad member length or job index");              \
    if (int rc = require_sm100()) return rc;                                                   \
    return dba_batch_launch<T>(                                                                \
        centroids, reinterpret_cast<const unsigned long long *>(centroid_offsets),             \
        centroid_lens, job_flags, job_member_begin, job_member_end, njobs, max_centroid_len,   \
        series, offsets, lens, member_series, member_job, member_order, nmem, h_member_lens,    \
        h_member_job, h_centroid_lens, h_job_flags, means, counts, deltas, path_triples,        \
        path_counts, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));           \
  }
ODBA_BATCH_ROUND(f32, float)
ODBA_BATCH_ROUND(f64, double)
#undef ODBA_BATCH_ROUND

size_t odba_segment_capacity(const uint64_t *h_lens, int n, int min_segment_length) {
  if (n < 1 || !h_lens || min_segment_length < 1) return 0;
  int dw, spb, k_max;
  segment_params(min_segment_length, &dw, &spb, &k_max);
  size_t c = 0;
  for (int i = 0; i < n; ++i) c += size_t((h_lens[i] + spb - 1) / spb) * size_t(k_max);
  return c;
}

size_t odba_segment_workspace_bytes(int n) { return n > 0 ? size_t(n) * 8 + 256 : 256; }

int odba_segment_blocks_f32(const float *series, const uint64_t *offsets, const uint64_t *lens,
                            const uint64_t *h_lens, int n, int min_segment_length, float *medians,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (n < 0 || (n > 0 && (!series || !offsets || !lens || !h_lens || !medians || !workspace)) ||
      min_segment_length < 1)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or minimum segment length below 1");
  if (int rc = require_sm100()) return rc;
  return segment_blocks<float>(series, offsets, lens, h_lens, n, min_segment_length, medians,
                               workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int odba_segment_blocks_f64(const double *series, const uint64_t *offsets, const uint64_t *lens,
                            const uint64_t *h_lens, int n, int min_segment_length, double *medians,
                            void *workspace, size_t workspace_bytes, void *stream) {
  if (n < 0 || (n > 0 && (!series || !offsets || !lens || !h_lens || !medians || !workspace)) ||
      min_segment_length < 1)
    return fail(ODBA_ERR_INVALID_ARGUMENT, "null pointer or minimum segment length below 1");
  if (int rc = require_sm100()) return rc;
  return segment_blocks<double>(series, offsets, lens, h_lens, n, min_segment_length, medians,
                                workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
