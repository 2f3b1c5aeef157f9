// Adaptive k-segmentation (adaptive_device_segmentation, segmentation.hpp:48-337).
//
// One 256-thread CTA per block of 256*dw raw samples (dw = ceil(minseg/3)):
// down-average by dw, 8-bit quantise against the block's range, then the
// Bellman k-segment DP on integer squared errors, with a binary search on k
// for the largest k whose segments are all at least minseg/dw long, and the
// segment medians of the raw samples.
//
// Differences in structure, not in results:
//  * DP row p depends only on row p-1, so all n of a row are computed at once
//    (one thread per n, each scanning its <= e candidates in increasing order,
//    first strict minimum wins) -- the reference runs every n through thread 0
//    with two barriers per n.
//  * The sum / square tables are prefix sums (the reference's 16-bit sums never
//    wrap for <= 256 samples of at most 255), and the whole backtrack table
//    stays in shared memory instead of a global working buffer.
//  * The DP extent e is computed from the reference's shared-memory layout and
//    the device's opt-in shared memory per block (segmentation.hpp:162, 458-461).
// Kept as the reference computes them: the down-averaging loop bound (which
// averages zero samples -- NaN -- for the upper part of a block), the
// FLT_MIN/partial-warp rules of the min/max reduction, the block minimum that
// only thread 0 sees, the saturating 8-bit conversion, the wrapping int product
// in DIST, and the even-span median pick (segmentation.hpp:327-332).  Where the
// reference races (a 2-sample segment's median reads the first sample of the
// next segment while that one is being sorted) the sorted value is used.
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>

#include "dtw_device.cuh"
#include "odba_internal.h"

namespace odba {

namespace {

template <typename T>
struct SegLim;
template <>
struct SegLim<float> {
  static __device__ __forceinline__ float lo() { return FLT_MIN; }
  static __device__ __forceinline__ float hi() { return FLT_MAX; }
};
template <>
struct SegLim<double> {
  static __device__ __forceinline__ double lo() { return DBL_MIN; }
  static __device__ __forceinline__ double hi() { return DBL_MAX; }
};

// warpReduceMin / warpReduceMax of cuda_utils.hpp:20-40
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const T o = __shfl_down_sync(kFull, v, off);
    if (o < v) v = o;
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const T o = __shfl_down_sync(kFull, v, off);
    if (o > v) v = o;
  }
  return v;
}

struct SegParams {
  int spb, k_max, minseg, dw, smem_optin;
};

// DP extent from the reference's dynamic shared-memory layout.
template <typename T>
__device__ __forceinline__ int dp_extent(int k_max, int N_ds, int smem) {
  if (N_ds <= 0) return 1;
  const long off_opt = ((long)(k_max + 1) * 2 + 3) / 4 * 4;
  const long off_ksd = off_opt + (long)(N_ds + 1) * 4;
  const long off_ds = (off_ksd + 2L * (N_ds + 1) * 4 + (long)sizeof(T) - 1) / (long)sizeof(T) * (long)sizeof(T);
  const long off_sq = (off_ds + (long)(N_ds + 2) * (long)sizeof(T) + 3) / 4 * 4;
  return int((smem - off_sq) / ((long)N_ds * 6));
}

template <typename T>
__global__ void __launch_bounds__(256) segment_kernel(const T *series, const uint64_t *offsets,
                                                      const uint64_t *lens,
                                                      const unsigned long long *seg_base,
                                                      SegParams sp, T *medians) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int s = blockIdx.x, by = blockIdx.y;
  const long orig_N = long(lens[s]);
  const int spb = sp.spb, dw = sp.dw, k_max = sp.k_max;
  if ((long)by * spb >= orig_N) return;
  const T *x = series + offsets[s] + (long)by * spb;
  T *out = medians + seg_base[s] + (unsigned long long)by * k_max;

  const bool partial = (long)(by + 1) * spb > orig_N;
  const int N = partial ? int(orig_N % spb) : spb;
  int expected_k = k_max;
  if (partial) {
    const int per = (spb + k_max - 1) / k_max;
    expected_k = (int(orig_N % spb) + per - 1) / per;
  }
  const int N_ds = N / dw;
  const int e = dp_extent<T>(k_max, N_ds, sp.smem_optin);

  // shared memory carve-up
  const int W = N_ds + 2;
  T *od = reinterpret_cast<T *>(smem_raw);                                // spb raw samples + 2
  unsigned *P = reinterpret_cast<unsigned *>(od + spb + 2);                // 257 prefix sums
  unsigned *Q = P + 257;                                                   // 257 prefix squares
  unsigned *ksd0 = Q + 257;                                                // W
  unsigned *ksd1 = ksd0 + W;                                               // W
  unsigned short *bp = reinterpret_cast<unsigned short *>(ksd1 + W);       // k_max + 2
  unsigned short *kpath = bp + (k_max + 2);                                // (k_max + 1) * W
  __shared__ T wmaxs[8], wmins[8];
  __shared__ T gstat[2];
  __shared__ unsigned char q[256];
  __shared__ int ctrl[4];

  // 1. down-average, with the reference's loop bound (segmentation.hpp:111-120)
  T dsv = T(0);
  if (t * dw <= N - dw) {
    T acc = T(0);
    int num = 0;
    for (int i = 0; i < dw && dw * t + t + i < N; i++) {
      acc = acc + x[dw * t + i];
      num++;
    }
    dsv = acc / T(num);
  }
  // 2. block range (segmentation.hpp:124-150)
  T vmax = t < N_ds ? dsv : SegLim<T>::lo();
  T vmin = t < N_ds ? dsv : SegLim<T>::hi();
  vmin = warp_min(vmin);
  vmax = warp_max(vmax);
  const int nw = N_ds / 32;
  if (lane == 0 && wid < nw) {
    wmaxs[wid] = vmax;
    wmins[wid] = vmin;
  }
  __syncthreads();
  if (wid == 0) {
    T a = lane < nw ? wmaxs[lane] : SegLim<T>::lo();
    a = warp_max(a);
    T b = lane < nw ? wmins[lane] : SegLim<T>::hi();
    b = warp_min(b);
    if (lane == 0) {
      gstat[0] = a;
      gstat[1] = b;
    }
  }
  __syncthreads();
  const T gmax = gstat[0];
  // thread 0 sees the block minimum; the others read slot nw of the max array
  const T others_min = nw >= 2 ? wmins[0] : (nw == 1 ? gstat[1] : gmax);
  const T mn = t == 0 ? gstat[1] : others_min;
  // 3. quantise (segmentation.hpp:168)
  if (t < N_ds) q[t] = (unsigned char)(256.0 * ((dsv - mn) / (gmax - mn + 1)));
  __syncthreads();
  if (t == 0) {
    unsigned a = 0, b = 0;
    P[0] = 0;
    Q[0] = 0;
    for (int i = 0; i < N_ds; ++i) {
      a += q[i];
      b += unsigned(q[i]) * q[i];
      P[i + 1] = a;
      Q[i + 1] = b;
    }
    ctrl[0] = (expected_k + 1) / 2;      // test_k
    ctrl[1] = ctrl[0] / 2;               // delta
    ctrl[2] = expected_k + 1;            // smallest noisy k found
    ctrl[3] = 0;                         // exit
  }
  __syncthreads();

  // 4. DP with the binary search on k (segmentation.hpp:190-336)
  while (!ctrl[3]) {
    const int test_k = ctrl[0];
    for (int n1 = t + 1; n1 <= N_ds; n1 += blockDim.x) {
      if (n1 <= e) {
        const unsigned sm = P[n1], sq = Q[n1];
        const int ms = int(unsigned(sm * sm)) / n1;
        ksd1[n1] = sq - unsigned(ms);
      } else {
        ksd1[n1] = INT_MAX / 2;
      }
    }
    if (t < N_ds && t < test_k) kpath[t * W + t] = (unsigned short)(test_k - 1);
    __syncthreads();
    for (int p = 2; p <= test_k; ++p) {
      const unsigned *prev = (p & 1) ? ksd0 : ksd1;
      unsigned *cur = (p & 1) ? ksd1 : ksd0;
      for (int n = p + t; n <= N_ds; n += blockDim.x) {
        const int lo = (n - e + 1 > p) ? n - e + 1 : p;
        int minval = INT_MAX, minidx = -1;
        const unsigned Pn = P[n], Qn = Q[n];
        for (int idx = lo; idx <= n; ++idx) {
          const unsigned sm = Pn - P[idx - 1];
          const unsigned sq = Qn - Q[idx - 1];
          const int ms = int(unsigned(sm * sm)) / (n - idx + 1);
          const unsigned opt = prev[idx - 1] + (sq - unsigned(ms));
          if (opt < unsigned(minval)) {
            minval = int(opt);
            minidx = idx;
          }
        }
        cur[n] = unsigned(minval);
        kpath[(p - 1) * W + (n - 1)] = (unsigned short)((unsigned short)minidx - 1);
      }
      __syncthreads();
    }
    if (t == 0) {
      bp[test_k] = (unsigned short)N_ds;
      for (int p = test_k - 1; p >= 1; p--) {
        const int col = bp[p + 1] - 1;
        bp[p] = (col >= 0 && col < W) ? kpath[p * W + col] : 0;
      }
      bp[0] = 0;
      bool noisy = false;
      for (int i = 1; i <= test_k; i++)
        if (int(bp[i]) - int(bp[i - 1]) < sp.minseg / dw) noisy = true;
      int delta = ctrl[1];
      int tk = test_k;
      if (delta == 0 || tk + delta > k_max) {
        ctrl[3] = 1;
      } else if (tk != 1 && noisy) {
        ctrl[2] = tk;
        tk -= delta;
      } else {
        if (tk == 1 || ctrl[2] == tk + 1)
          ctrl[3] = 1;
        else
          tk += delta;
      }
      ctrl[1] = (delta + 1) / 2;
      if (!ctrl[3]) ctrl[0] = tk;
    }
    __syncthreads();
  }
  const int test_k = ctrl[0];

  // 5. medians of the raw samples (segmentation.hpp:287-333)
  // samples past the block read as 0 (the reference reads whatever its shared
  // memory holds there, which only an even-span last segment can reach)
  for (int i = t; i < spb + 2; i += blockDim.x)
    od[i] = (i < spb && (long)by * spb + i < orig_N) ? x[i] : T(0);
  __syncthreads();
  for (int seg = t + 1; seg <= k_max; seg += blockDim.x)
    if (seg > test_k) out[seg - 1] = SegLim<T>::hi();
  for (int seg = t + 1; seg <= test_k; seg += blockDim.x) {
    int rb = bp[seg] * dw;
    if (rb > N) rb = N;
    const int lb = bp[seg - 1] * dw;
    for (int i = lb; i < rb - 1; ++i)
      for (int j = i + 1; j < rb; ++j)
        if (od[i] > od[j]) {
          const T tmp = od[i];
          od[i] = od[j];
          od[j] = tmp;
        }
  }
  __syncthreads();
  for (int seg = t + 1; seg <= test_k; seg += blockDim.x) {
    int rb = bp[seg] * dw;
    if (rb > N) rb = N;
    const int lb = bp[seg - 1] * dw;
    const int mid = (lb + rb) / 2;
    out[seg - 1] = ((lb - rb) % 2) ? od[mid] : (od[mid] + od[mid + 1]) / 2;
  }
}

}  // namespace

void segment_params(int minseg, int *dw, int *spb, int *k_max) {
  *dw = (minseg + 2) / 3;
  *spb = 256 * *dw;
  const float per = float(minseg) / float(*dw);
  *k_max = int((256 + per - 1) / per);
}

template <typename T>
int segment_launch(const T *series, const uint64_t *offsets, const uint64_t *lens,
                   const unsigned long long *seg_base, int n, int max_blocks, int minseg,
                   T *medians, cudaStream_t stream) {
  SegParams sp;
  segment_params(minseg, &sp.dw, &sp.spb, &sp.k_max);
  sp.minseg = minseg;
  int dev = 0;
  cudaGetDevice(&dev);
  sp.smem_optin = 48 * 1024;
  cudaDeviceGetAttribute(&sp.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int W = 256 + 2;
  const size_t smem = size_t(sp.spb + 2) * sizeof(T) + 2 * 257 * 4 + 2 * W * 4 +
                      size_t(sp.k_max + 2) * 2 + size_t(sp.k_max + 1) * W * 2 + 64;
  if (smem > size_t(sp.smem_optin))
    return fail(ODBA_ERR_INVALID_ARGUMENT, "minimum segment length needs more shared memory than the device has");
  cudaFuncSetAttribute(segment_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (n < 1 || max_blocks < 1) return ODBA_OK;
  dim3 grid(n, max_blocks);
  segment_kernel<T><<<grid, 256, smem, stream>>>(series, offsets, lens, seg_base, sp, medians);
  return check_launch("segmentation kernel");
}

__global__ void seg_base_kernel(const uint64_t *lens, int n, int spb, int k_max,
                                unsigned long long *base) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long acc = 0;
  for (int i = 0; i < n; ++i) {
    base[i] = acc;
    acc += (unsigned long long)((lens[i] + spb - 1) / spb) * k_max;
  }
}

template <typename T>
int segment_blocks(const T *series, const uint64_t *offsets, const uint64_t *lens,
                   const uint64_t *h_lens, int n, int minseg, T *medians, void *ws,
                   size_t ws_bytes, cudaStream_t stream) {
  if (n < 1) return ODBA_OK;
  if (ws_bytes < size_t(n) * 8) return fail(ODBA_ERR_WORKSPACE_TOO_SMALL, "segmentation workspace too small");
  int dw, spb, k_max;
  segment_params(minseg, &dw, &spb, &k_max);
  int max_blocks = 0;
  for (int i = 0; i < n; ++i) {
    const long nb = long((h_lens[i] + spb - 1) / spb);
    if (nb > 65535) return fail(ODBA_ERR_INVALID_ARGUMENT, "series too long for one segmentation grid");
    if (nb > max_blocks) max_blocks = int(nb);
  }
  auto *base = static_cast<unsigned long long *>(ws);
  seg_base_kernel<<<1, 32, 0, stream>>>(lens, n, spb, k_max, base);
  return segment_launch<T>(series, offsets, lens, base, n, max_blocks, minseg, medians, stream);
}

template int segment_blocks<float>(const float *, const uint64_t *, const uint64_t *,
                                   const uint64_t *, int, int, float *, void *, size_t,
                                   cudaStream_t);
template int segment_blocks<double>(const double *, const uint64_t *, const uint64_t *,
                                    const uint64_t *, int, int, double *, void *, size_t,
                                    cudaStream_t);

template int segment_launch<float>(const float *, const uint64_t *, const uint64_t *,
                                   const unsigned long long *, int, int, int, float *, cudaStream_t);
template int segment_launch<double>(const double *, const uint64_t *, const uint64_t *,
                                    const unsigned long long *, int, int, int, double *,
                                    cudaStream_t);

}  // namespace odba
