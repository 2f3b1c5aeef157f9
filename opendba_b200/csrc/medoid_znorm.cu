// Medoid selection and z-normalisation kernels.
//
// Medoid (approximateMedoidIndices, dba.hpp:186-351, one cluster): the
// reference accumulates every series' sum of squared distances in T on the
// host, walking the upper triangle row by row, so series k receives first the
// pairs (s, k), s < k, in order, then its own row (k, j), j > k.  One thread
// per series replays exactly that order (products and sums rounded separately,
// as the host code does), then one block picks the first index with the
// strictly smallest sum; two members pick the longer one, ties to the second.
//
// Z-normalisation (normalizeSequences, gpu_utils.hpp:34-170): per series, per
// 1024-sample chunk a shuffle-down tree per warp and the same tree over the 32
// warp partials; the sum in T, the squared residuals in double; population
// sigma, 0 -> 1; x <- (T)(0 + ((x - mean)/sigma) * 1).  The reference adds the
// chunk partials with atomics in arrival order; here they are added in
// ascending chunk order, so the result is run-to-run reproducible (and equals
// the reference's whenever the series has at most 1024 samples).
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "dtw_device.cuh"
#include "odba_internal.h"

namespace odba {

namespace {

__device__ __forceinline__ long long row_start_ll(long long s, long long n) {
  return s * n - s * (s + 1) / 2;
}

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

template <typename T>
__global__ void sos_kernel(const T *dists, int n, T *sos) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  T acc = T(0);
  for (int s = 0; s < k; ++s) {
    const T d = dists[row_start_ll(s, n) + (k - s - 1)];
    acc = add_rn(acc, mul_rn(d, d));
  }
  const long long base = row_start_ll(k, n);
  for (int j = k + 1; j < n; ++j) {
    const T d = dists[base + (j - k - 1)];
    acc = add_rn(acc, mul_rn(d, d));
  }
  sos[k] = acc;
}

template <typename T>
__global__ void argmin_kernel(const T *sos, const uint64_t *lens, int n, int *medoid) {
  __shared__ T sv[1024];
  __shared__ int si[1024];
  T best = Num<T>::big();
  int bi = -1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const T v = sos[i];
    if (v < best) {  // strictly smaller; NaN never wins (dba.hpp:327-335)
      best = v;
      bi = i;
    }
  }
  sv[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      const T ov = sv[threadIdx.x + w];
      const int oi = si[threadIdx.x + w];
      const int mi = si[threadIdx.x];
      if (oi >= 0 && (mi < 0 || ov < sv[threadIdx.x] || (ov == sv[threadIdx.x] && oi < mi))) {
        sv[threadIdx.x] = ov;
        si[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int m = si[0];
    if (n == 2) m = lens[0] > lens[1] ? 0 : 1;  // dba.hpp:336-339
    if (n == 1) m = 0;
    *medoid = m;
  }
}

// Shuffle-down tree of calc_sums (gpu_utils.hpp:47-49); lane 0 holds the sum.
template <typename T>
__device__ __forceinline__ T warp_tree(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = add_rn(v, __shfl_down_sync(kFull, v, off));
  return v;
}

// Tree sum of one 1024-sample chunk as calc_sums / calc_sum_of_squares do it.
template <typename A>
__device__ __forceinline__ A block_tree(A v, A *ws) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_tree(v);
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  A r = A(0);
  if (wid == 0) r = warp_tree(ws[lane]);
  __syncthreads();
  return r;  // valid in thread 0
}

template <typename T>
__global__ void __launch_bounds__(1024) znorm_kernel(T *series, const uint64_t *offsets,
                                                     const uint64_t *lens, double *means,
                                                     double *sigmas) {
  __shared__ T wsum[32];
  __shared__ double wss[32];
  __shared__ double stats[2];
  T *x = series + offsets[blockIdx.x];
  const uint64_t len = lens[blockIdx.x];
  const uint64_t chunks = (len + 1023) / 1024;
  T sum = T(0);
  for (uint64_t ch = 0; ch < chunks; ++ch) {
    const uint64_t pos = ch * 1024 + threadIdx.x;
    const T v = pos < len ? x[pos] : T(0);
    const T cs = block_tree<T>(v, wsum);
    if (threadIdx.x == 0) sum = add_rn(sum, cs);
  }
  if (threadIdx.x == 0) stats[0] = double(sum) / double(len);
  __syncthreads();
  const double mean = stats[0];
  double ss = 0.0;
  for (uint64_t ch = 0; ch < chunks; ++ch) {
    const uint64_t pos = ch * 1024 + threadIdx.x;
    double t = 0.0;
    if (pos < len) {
      t = __dadd_rn(double(x[pos]), -mean);
      t = __dmul_rn(t, t);
    }
    const double cs = block_tree<double>(t, wss);
    if (threadIdx.x == 0) ss = __dadd_rn(ss, cs);
  }
  if (threadIdx.x == 0) {
    const double sd = __dsqrt_rn(__ddiv_rn(ss, double(len)));
    if (means) means[blockIdx.x] = mean;
    if (sigmas) sigmas[blockIdx.x] = sd;
    stats[1] = sd == 0.0 ? 1.0 : sd;
  }
  __syncthreads();
  const double sd = stats[1];
  for (uint64_t pos = threadIdx.x; pos < len; pos += blockDim.x) {
    const double q = __ddiv_rn(__dadd_rn(double(x[pos]), -mean), sd);
    x[pos] = T(__dadd_rn(0.0, __dmul_rn(q, 1.0)));
  }
}

}  // namespace

template <typename T>
int medoid_launch(const T *dists, const uint64_t *lens, int n, T *sos, int *medoid,
                  cudaStream_t stream) {
  if (n < 1) return fail(ODBA_ERR_INVALID_ARGUMENT, "medoid needs at least one series");
  sos_kernel<T><<<(n + 127) / 128, 128, 0, stream>>>(dists, n, sos);
  argmin_kernel<T><<<1, 1024, 0, stream>>>(sos, lens, n, medoid);
  return check_launch("medoid kernels");
}

template <typename T>
int znorm_launch(T *series, const uint64_t *offsets, const uint64_t *lens, int n, double *means,
                 double *sigmas, cudaStream_t stream) {
  if (n < 1) return ODBA_OK;
  znorm_kernel<T><<<n, 1024, 0, stream>>>(series, offsets, lens, means, sigmas);
  return check_launch("z-normalisation kernel");
}

template int medoid_launch<float>(const float *, const uint64_t *, int, float *, int *, cudaStream_t);
template int medoid_launch<double>(const double *, const uint64_t *, int, double *, int *,
                                   cudaStream_t);
template int znorm_launch<float>(float *, const uint64_t *, const uint64_t *, int, double *,
                                 double *, cudaStream_t);
template int znorm_launch<double>(double *, const uint64_t *, const uint64_t *, int, double *,
                                  double *, cudaStream_t);

}  // namespace odba
