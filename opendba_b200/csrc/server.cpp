// Serving loop with continuous batching (no reference counterpart; the
// reference runs one job per process).
//
// Requests:
//   * query: nreads series against resident centroids -> nreads x ncentroids
//     DTW distances (the reference's pair distance, dtw.hpp:116-125, 242-257;
//     the read is the first series, the centroid the second);
//   * job:   an averaging job, i.e. performDBA for one cluster (cdist 1, no
//     files): truncation, length sort, z-norm, medoid, rounds to convergence,
//     rescale -- the same result odba_dba_jobs_* gives.
// A worker thread repeats: admit pending requests in arrival order while the
// device-memory estimate of everything admitted stays under the budget; run
// one pair-list launch with every admitted query's pairs and every job still
// in its medoid stage; pick those jobs' medoids; run one batched DBA round
// for every job in its round stage; retire what finished.  Requests that
// arrive meanwhile join the next iteration.  Every pair and every job is
// computed independently of what else is in the batch, so a request's result
// is the same alone and in any mix.
//
// Series that live in separate device allocations share one pair-list launch
// through a null series base: the launch's offsets are element addresses
// (device address / sizeof(T)), which the kernels add to the null base.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "opendba_b200.h"

namespace {

template <typename T>
struct ServerOps;
template <>
struct ServerOps<float> {
  static int pairlist(const float *s, const uint64_t *o, const uint64_t *l, const odba_pair_task *t,
                      uint64_t n, uint64_t ml, float *d, void *w, size_t wb, void *st) {
    return odba_dtw_pairlist_f32(s, o, l, t, n, ml, d, w, wb, st);
  }
  static int znorm(float *s, const uint64_t *o, const uint64_t *l, int n, double *m, double *sg, void *st) {
    return odba_znorm_f32(s, o, l, n, m, sg, st);
  }
  static int medoid(const float *d, const uint64_t *l, int n, float *sos, int *med, void *st) {
    return odba_medoid_f32(d, l, n, sos, med, st);
  }
  template <typename... A>
  static int round(A... a) {
    return odba_dba_batch_round_f32(a...);
  }
};
template <>
struct ServerOps<double> {
  static int pairlist(const double *s, const uint64_t *o, const uint64_t *l, const odba_pair_task *t,
                      uint64_t n, uint64_t ml, double *d, void *w, size_t wb, void *st) {
    return odba_dtw_pairlist_f64(s, o, l, t, n, ml, d, w, wb, st);
  }
  static int znorm(double *s, const uint64_t *o, const uint64_t *l, int n, double *m, double *sg, void *st) {
    return odba_znorm_f64(s, o, l, n, m, sg, st);
  }
  static int medoid(const double *d, const uint64_t *l, int n, double *sos, int *med, void *st) {
    return odba_medoid_f64(d, l, n, sos, med, st);
  }
  template <typename... A>
  static int round(A... a) {
    return odba_dba_batch_round_f64(a...);
  }
};

enum Stage { kPending = 0, kMedoid = 1, kRounds = 2, kDone = 3, kFailed = 4 };

template <typename T>
struct Request {
  int64_t id = 0;
  bool is_query = false;
  int flags = 0;  // bit 0 open start, bit 1 open end
  int norm = 0;
  std::vector<T> host;           // input series, concatenated (jobs: sorted, truncated)
  std::vector<uint64_t> lens;    // per series
  std::vector<int> order;        // jobs: sorted position -> input position
  std::vector<int> centroid_ids; // queries
  size_t footprint = 0;
  int stage = kPending;
  // device
  T *d_series = nullptr;
  uint64_t *d_offs = nullptr, *d_lens = nullptr;
  std::vector<uint64_t> elem_addr;  // element address of every series (null-base offsets)
  T *d_dists = nullptr;
  int *d_med = nullptr;
  T *d_sos = nullptr;
  double *d_mean = nullptr, *d_sig = nullptr;
  std::vector<double> means, sigmas;
  // job state
  int medoid = -1;
  std::vector<T> centroid, prev, two_prev;
  int rounds = 0;
  double delta = 0;
  // results
  std::vector<T> result;
  int status = ODBA_OK;
  double t_submit = 0, t_done = 0;
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
class Server {
 public:
  Server(size_t budget, int device) : budget_(budget), device_(device) {
    cudaSetDevice(device_);
    cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
    // A private stream-ordered pool that keeps up to the HBM budget mapped:
    // the device's default pool unmaps freed memory at every synchronisation,
    // which would re-map the per-iteration workspaces on every iteration.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    if (cudaMemPoolCreate(&pool_, &props) == cudaSuccess) {
      uint64_t keep = budget_;
      cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
      cudaGetLastError();
      pool_ = nullptr;
    }
    worker_ = std::thread([this] { loop(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    worker_.join();
    for (auto &kv : reqs_) release(*kv.second);
    cudaStreamSynchronize(st_);
    for (auto &c : centroids_) cudaFree(c.d);
    if (pool_) cudaMemPoolDestroy(pool_);
    cudaStreamDestroy(st_);
  }

  int add_centroid(const T *h, uint64_t len) {
    std::lock_guard<std::mutex> g(cmu_);
    Centroid c;
    c.len = len;
    cudaSetDevice(device_);
    if (cudaMalloc(&c.d, len * sizeof(T)) != cudaSuccess) return -ODBA_ERR_OUT_OF_MEMORY;
    cudaMemcpy(c.d, h, len * sizeof(T), cudaMemcpyHostToDevice);
    centroids_.push_back(c);
    return int(centroids_.size()) - 1;
  }

  int64_t submit_query(const T *h_reads, const uint64_t *h_lens, int nreads, const int *ids, int nids,
                       int flags) {
    auto r = std::make_shared<Request<T>>();
    r->is_query = true;
    r->flags = flags & 3;
    uint64_t total = 0;
    for (int i = 0; i < nreads; ++i) total += h_lens[i];
    r->host.assign(h_reads, h_reads + total);
    r->lens.assign(h_lens, h_lens + nreads);
    r->centroid_ids.assign(ids, ids + nids);
    {
      std::lock_guard<std::mutex> g(cmu_);
      for (int id : r->centroid_ids)
        if (id < 0 || id >= int(centroids_.size())) return -ODBA_ERR_INVALID_ARGUMENT;
    }
    r->footprint = total * sizeof(T) + size_t(nreads) * nids * sizeof(T) + 4096;
    return enqueue(r);
  }

  int64_t submit_job(const T *h_series, const uint64_t *h_lens, int n, int flags, int norm) {
    auto r = std::make_shared<Request<T>>();
    r->is_query = false;
    r->flags = flags & 3;
    r->norm = norm;
    std::vector<uint64_t> offs(n), L(n);
    uint64_t acc = 0;
    for (int i = 0; i < n; ++i) {
      offs[i] = acc;
      acc += h_lens[i];
      L[i] = h_lens[i];
      if (L[i] && h_series[offs[i] + L[i] - 1] >= std::sqrt(std::numeric_limits<T>::max())) --L[i];
    }
    r->order.resize(n);
    std::iota(r->order.begin(), r->order.end(), 0);
    std::stable_sort(r->order.begin(), r->order.end(), [&](int a, int b) { return L[a] < L[b]; });
    uint64_t maxlen = 1;
    for (int k : r->order) {
      r->host.insert(r->host.end(), h_series + offs[k], h_series + offs[k] + L[k]);
      r->lens.push_back(L[k]);
      maxlen = std::max<uint64_t>(maxlen, L[k]);
    }
    // series, triangle, and the 2-bit paths of one round against the longest centroid
    uint64_t words = 0;
    for (uint64_t l : r->lens) words += (l + 64) * (maxlen + 1024) / 16;
    r->footprint = r->host.size() * sizeof(T) + size_t(n) * n * sizeof(T) / 2 + words + 8 * 1024 * 1024;
    return enqueue(r);
  }

  // 0 = running, 1 = done, negative = failed / unknown
  int poll(int64_t id) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -ODBA_ERR_INVALID_ARGUMENT;
    if (it->second->stage == kFailed) return -it->second->status;
    return it->second->stage == kDone ? 1 : 0;
  }

  int wait(int64_t id, double timeout_s) {
    std::unique_lock<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -ODBA_ERR_INVALID_ARGUMENT;
    auto r = it->second;
    const bool ok = done_cv_.wait_for(g, std::chrono::duration<double>(timeout_s),
                                      [&] { return r->stage == kDone || r->stage == kFailed; });
    if (!ok) return -ODBA_ERR_TIMEOUT;
    return r->stage == kDone ? 1 : -r->status;
  }

  // Copies a finished request's result out and forgets the request.
  int take(int64_t id, T *out, uint64_t cap, uint64_t *len, int *medoid, int *rounds,
           double *latency_s) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return ODBA_ERR_INVALID_ARGUMENT;
    auto r = it->second;
    if (r->stage != kDone) return r->stage == kFailed ? r->status : ODBA_ERR_INVALID_ARGUMENT;
    if (len) *len = r->result.size();
    if (out && cap >= r->result.size()) std::memcpy(out, r->result.data(), r->result.size() * sizeof(T));
    if (medoid) *medoid = r->medoid >= 0 ? r->order[r->medoid] : -1;
    if (rounds) *rounds = r->rounds;
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    reqs_.erase(it);
    return (out && cap < r->result.size()) ? ODBA_ERR_INVALID_ARGUMENT : ODBA_OK;
  }

  void stats(uint64_t *iterations, uint64_t *cells, double *busy_s) {
    *iterations = iters_.load();
    *cells = cells_.load();
    *busy_s = busy_.load();
  }

 private:
  struct Centroid {
    T *d = nullptr;
    uint64_t len = 0;
  };

  int64_t enqueue(std::shared_ptr<Request<T>> r) {
    std::lock_guard<std::mutex> g(mu_);
    r->id = next_id_++;
    r->t_submit = now_s();
    reqs_[r->id] = r;
    pending_.push_back(r);
    cv_.notify_all();
    return r->id;
  }

  // Stream-ordered frees: no device-wide synchronisation per request.
  void release(Request<T> &r) {
    for (void *p : {static_cast<void *>(r.d_series), static_cast<void *>(r.d_offs),
                    static_cast<void *>(r.d_lens), static_cast<void *>(r.d_dists),
                    static_cast<void *>(r.d_med), static_cast<void *>(r.d_sos),
                    static_cast<void *>(r.d_mean), static_cast<void *>(r.d_sig)})
      if (p) cudaFreeAsync(p, st_);
    r.d_series = nullptr;
    r.d_offs = r.d_lens = nullptr;
    r.d_dists = r.d_sos = nullptr;
    r.d_med = nullptr;
    r.d_mean = r.d_sig = nullptr;
  }

  void finish(std::shared_ptr<Request<T>> r, int stage, int status = ODBA_OK) {
    release(*r);
    std::lock_guard<std::mutex> g(mu_);
    r->stage = stage;
    r->status = status;
    r->t_done = now_s();
    used_ -= r->footprint;
    done_cv_.notify_all();
  }

  template <typename U>
  cudaError_t dmalloc(U **p, size_t bytes) {
    return pool_ ? cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool_, st_)
                 : cudaMallocAsync(reinterpret_cast<void **>(p), bytes, st_);
  }

  // device copies of an admitted request
  bool upload(Request<T> &r) {
    const int n = int(r.lens.size());
    std::vector<uint64_t> offs(n);
    uint64_t acc = 0;
    for (int i = 0; i < n; ++i) {
      offs[i] = acc;
      acc += r.lens[i];
    }
    if (dmalloc(&r.d_series, (acc + 16) * sizeof(T)) != cudaSuccess ||
        dmalloc(&r.d_offs, n * sizeof(uint64_t)) != cudaSuccess ||
        dmalloc(&r.d_lens, n * sizeof(uint64_t)) != cudaSuccess)
      return false;
    cudaMemcpyAsync(r.d_series, r.host.data(), acc * sizeof(T), cudaMemcpyHostToDevice, st_);
    cudaMemcpyAsync(r.d_offs, offs.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st_);
    cudaMemcpyAsync(r.d_lens, r.lens.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st_);
    r.elem_addr.resize(n);
    for (int i = 0; i < n; ++i)
      r.elem_addr[i] = reinterpret_cast<uint64_t>(r.d_series) / sizeof(T) + offs[i];
    if (!r.is_query) {
      if (dmalloc(&r.d_mean, n * sizeof(double)) != cudaSuccess ||
          dmalloc(&r.d_sig, n * sizeof(double)) != cudaSuccess)
        return false;
      if (r.norm &&
          ServerOps<T>::znorm(r.d_series, r.d_offs, r.d_lens, n, r.d_mean, r.d_sig, st_) != ODBA_OK)
        return false;
      const size_t np = size_t(n) * (n - 1) / 2;
      if (dmalloc(&r.d_dists, std::max<size_t>(np, 1) * sizeof(T)) != cudaSuccess ||
          dmalloc(&r.d_sos, n * sizeof(T)) != cudaSuccess ||
          dmalloc(&r.d_med, sizeof(int)) != cudaSuccess)
        return false;
      r.means.assign(n, 0.0);
      r.sigmas.assign(n, 1.0);
      if (r.norm) {
        cudaMemcpyAsync(r.means.data(), r.d_mean, n * sizeof(double), cudaMemcpyDeviceToHost, st_);
        cudaMemcpyAsync(r.sigmas.data(), r.d_sig, n * sizeof(double), cudaMemcpyDeviceToHost, st_);
      }
    } else {
      const size_t nd = r.lens.size() * r.centroid_ids.size();
      if (dmalloc(&r.d_dists, std::max<size_t>(nd, 1) * sizeof(T)) != cudaSuccess) return false;
    }
    return true;
  }

  void loop() {
    cudaSetDevice(device_);
    for (;;) {
      std::vector<std::shared_ptr<Request<T>>> admitted;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || !pending_.empty() || !active_.empty(); });
        if (stop_) return;
        while (!pending_.empty() && (active_.empty() || used_ + pending_.front()->footprint <= budget_)) {
          auto r = pending_.front();
          pending_.pop_front();
          used_ += r->footprint;
          admitted.push_back(r);
        }
      }
      const double t0 = now_s();
      for (auto &r : admitted) {
        if (!upload(*r)) {
          cudaGetLastError();
          finish(r, kFailed, ODBA_ERR_OUT_OF_MEMORY);
          continue;
        }
        r->stage = r->is_query ? kMedoid : (r->lens.size() > 1 ? kMedoid : kRounds);
        active_.push_back(r);
      }
      iterate();
      busy_ = busy_.load() + (now_s() - t0);
      iters_++;
      // retire
      std::vector<std::shared_ptr<Request<T>>> still;
      for (auto &r : active_)
        if (r->stage != kDone && r->stage != kFailed) still.push_back(r);
      active_.swap(still);
    }
  }

  void iterate() {
    // ---- one pair-list launch: queries + jobs in their medoid stage
    std::vector<odba_pair_task> tasks;
    std::vector<double> cost;
    std::vector<uint64_t> offs, lens;
    std::vector<std::pair<std::shared_ptr<Request<T>>, uint64_t>> outs;  // request, output base
    uint64_t out_total = 0, max_first = 1, cells = 0;
    auto add_series = [&](uint64_t addr, uint64_t len) {
      offs.push_back(addr);
      lens.push_back(len);
      return uint32_t(offs.size() - 1);
    };
    std::vector<std::shared_ptr<Request<T>>> medoid_jobs;
    for (auto &r : active_) {
      if (r->stage != kMedoid) continue;
      const uint64_t fl = (uint64_t(r->flags & 1) << 62) | (uint64_t((r->flags >> 1) & 1) << 63);
      if (r->is_query) {
        std::vector<uint32_t> cidx;
        {
          std::lock_guard<std::mutex> g(cmu_);
          for (int id : r->centroid_ids)
            cidx.push_back(add_series(reinterpret_cast<uint64_t>(centroids_[id].d) / sizeof(T),
                                      centroids_[id].len));
        }
        for (size_t i = 0; i < r->lens.size(); ++i) {
          const uint32_t ri = add_series(r->elem_addr[i], r->lens[i]);
          max_first = std::max<uint64_t>(max_first, r->lens[i]);
          for (size_t c = 0; c < cidx.size(); ++c) {
            tasks.push_back({ri, cidx[c], (out_total + i * cidx.size() + c) | fl});
            cost.push_back(double(r->lens[i]) * double(lens[cidx[c]]));
          }
        }
      } else {
        const int n = int(r->lens.size());
        std::vector<uint32_t> si(n);
        for (int i = 0; i < n; ++i) {
          si[i] = add_series(r->elem_addr[i], r->lens[i]);
          max_first = std::max<uint64_t>(max_first, r->lens[i]);
        }
        uint64_t p = 0;
        for (int s = 0; s + 1 < n; ++s)
          for (int t = s + 1; t < n; ++t, ++p) {
            tasks.push_back({si[s], si[t], (out_total + p) | fl});
            cost.push_back(double(r->lens[s]) * double(r->lens[t]));
          }
        medoid_jobs.push_back(r);
      }
      outs.push_back({r, out_total});
      out_total += r->is_query ? r->lens.size() * r->centroid_ids.size()
                               : r->lens.size() * (r->lens.size() - 1) / 2;
    }
    if (!tasks.empty()) {
      std::vector<size_t> perm(tasks.size());
      std::iota(perm.begin(), perm.end(), 0);
      std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
      std::vector<odba_pair_task> sorted(tasks.size());
      for (size_t i = 0; i < perm.size(); ++i) {
        sorted[i] = tasks[perm[i]];
        cells += uint64_t(cost[perm[i]]);
      }
      odba_pair_task *d_tasks = nullptr;
      uint64_t *d_offs = nullptr, *d_lens = nullptr;
      T *d_out = nullptr;
      void *ws = nullptr;
      const size_t wsb = odba_dtw_pairwise_workspace_bytes(sizeof(T), max_first);
      bool ok = dmalloc(&d_tasks, sorted.size() * sizeof(odba_pair_task)) == cudaSuccess &&
                dmalloc(&d_offs, offs.size() * 8) == cudaSuccess &&
                dmalloc(&d_lens, lens.size() * 8) == cudaSuccess &&
                dmalloc(&d_out, out_total * sizeof(T)) == cudaSuccess &&
                dmalloc(reinterpret_cast<char **>(&ws), wsb) == cudaSuccess;
      if (ok) {
        cudaMemcpyAsync(d_tasks, sorted.data(), sorted.size() * sizeof(odba_pair_task), cudaMemcpyHostToDevice, st_);
        cudaMemcpyAsync(d_offs, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, st_);
        cudaMemcpyAsync(d_lens, lens.data(), lens.size() * 8, cudaMemcpyHostToDevice, st_);
        ok = ServerOps<T>::pairlist(nullptr, d_offs, d_lens, d_tasks, sorted.size(), max_first, d_out,
                                    ws, wsb, st_) == ODBA_OK;
      }
      if (ok) {
        for (auto &o : outs) {
          auto &r = o.first;
          const uint64_t cnt = r->is_query ? r->lens.size() * r->centroid_ids.size()
                                           : r->lens.size() * (r->lens.size() - 1) / 2;
          cudaMemcpyAsync(r->d_dists, d_out + o.second, cnt * sizeof(T), cudaMemcpyDeviceToDevice, st_);
        }
        for (auto &r : medoid_jobs)
          ServerOps<T>::medoid(r->d_dists, r->d_lens, int(r->lens.size()), r->d_sos, r->d_med, st_);
      }
      // the pair kernels' hand-off wait error word (byte 8 of the workspace)
      unsigned wait_err = 0;
      if (ok) cudaMemcpyAsync(&wait_err, static_cast<char *>(ws) + 8, sizeof wait_err, cudaMemcpyDeviceToHost, st_);
      cudaFreeAsync(d_tasks, st_);
      cudaFreeAsync(d_offs, st_);
      cudaFreeAsync(d_lens, st_);
      cudaFreeAsync(d_out, st_);
      cudaFreeAsync(ws, st_);
      if (!ok || cudaStreamSynchronize(st_) != cudaSuccess) {
        cudaGetLastError();
        for (auto &o : outs) finish(o.first, kFailed, ODBA_ERR_CUDA);
        return;
      }
      if (wait_err) {
        for (auto &o : outs) finish(o.first, kFailed, ODBA_ERR_TIMEOUT);
        return;
      }
      cells_ += cells;
      for (auto &o : outs) {
        auto &r = o.first;
        if (r->is_query) {
          r->result.resize(r->lens.size() * r->centroid_ids.size());
          cudaMemcpy(r->result.data(), r->d_dists, r->result.size() * sizeof(T), cudaMemcpyDeviceToHost);
          finish(r, kDone);
        } else {
          cudaMemcpy(&r->medoid, r->d_med, sizeof(int), cudaMemcpyDeviceToHost);
          const int n = int(r->lens.size());
          uint64_t off = 0;
          for (int i = 0; i < r->medoid; ++i) off += r->lens[i];
          r->centroid.resize(r->lens[r->medoid]);
          cudaMemcpy(r->centroid.data(), r->d_series + off, r->centroid.size() * sizeof(T), cudaMemcpyDeviceToHost);
          r->prev.assign(r->centroid.size(), T(0));
          r->two_prev.assign(r->centroid.size(), T(0));
          r->stage = n > 1 ? kRounds : kDone;
        }
      }
    }
    for (auto &r : active_) {
      if (!r->is_query && r->stage == kRounds && r->lens.size() == 1) {
        // single series: the series is its own average
        cudaStreamSynchronize(st_);
        r->medoid = 0;
        r->centroid.resize(r->lens[0]);
        cudaMemcpy(r->centroid.data(), r->d_series, r->centroid.size() * sizeof(T), cudaMemcpyDeviceToHost);
        complete_job(r);
      }
    }
    // ---- one batched DBA round for every job in its round stage
    std::vector<std::shared_ptr<Request<T>>> rj;
    for (auto &r : active_)
      if (!r->is_query && r->stage == kRounds) rj.push_back(r);
    if (rj.empty()) return;
    const int nj = int(rj.size());
    std::vector<uint64_t> coff(nj), clenh(nj), s_offs, s_lens, h_mlens;
    std::vector<int> clen(nj), flags(nj), mbeg(nj), mend(nj), mseries, mjob;
    uint64_t ctot = 0;
    int max_clen = 1;
    uint64_t rcells = 0;
    for (int j = 0; j < nj; ++j) {
      auto &r = rj[j];
      coff[j] = ctot;
      clen[j] = int(r->centroid.size());
      clenh[j] = r->centroid.size();
      ctot += r->centroid.size();
      max_clen = std::max(max_clen, clen[j]);
      flags[j] = r->flags | 4;
      mbeg[j] = int(mseries.size());
      for (size_t i = 0; i < r->lens.size(); ++i) {
        mseries.push_back(int(s_offs.size()));
        mjob.push_back(j);
        s_offs.push_back(r->elem_addr[i]);
        s_lens.push_back(r->lens[i]);
        h_mlens.push_back(r->lens[i]);
        rcells += r->lens[i] * r->centroid.size();
      }
      mend[j] = int(mseries.size());
    }
    const int nm = int(mseries.size());
    std::vector<int> morder(nm);
    std::iota(morder.begin(), morder.end(), 0);
    std::stable_sort(morder.begin(), morder.end(), [&](int a, int b) {
      return double(h_mlens[a]) * clenh[mjob[a]] > double(h_mlens[b]) * clenh[mjob[b]];
    });
    std::vector<T> cent(ctot);
    for (int j = 0; j < nj; ++j) std::copy(rj[j]->centroid.begin(), rj[j]->centroid.end(), cent.begin() + coff[j]);
    const size_t wsb = odba_dba_batch_workspace_bytes(sizeof(T), h_mlens.data(), mjob.data(), nm,
                                                      clenh.data(), flags.data(), nj);
    char *blob = nullptr;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t sz[] = {up(ctot * sizeof(T)), up(ctot * sizeof(T)), up(ctot * 4), up(nj * 8),
                         up(nj * 8), up(nj * 4), up(nj * 4), up(nj * 4), up(nj * 4), up(s_offs.size() * 8),
                         up(s_lens.size() * 8), up(nm * 4), up(nm * 4), up(nm * 4), wsb};
    size_t total = 0, o[15];
    for (int i = 0; i < 15; ++i) {
      o[i] = total;
      total += sz[i];
    }
    if (dmalloc(&blob, total) != cudaSuccess) {
      cudaGetLastError();
      for (auto &r : rj) finish(r, kFailed, ODBA_ERR_OUT_OF_MEMORY);
      return;
    }
    auto put = [&](int i, const void *src, size_t bytes) {
      if (bytes) cudaMemcpyAsync(blob + o[i], src, bytes, cudaMemcpyHostToDevice, st_);
    };
    put(0, cent.data(), ctot * sizeof(T));
    put(4, coff.data(), nj * 8);
    put(5, clen.data(), nj * 4);
    put(6, flags.data(), nj * 4);
    put(7, mbeg.data(), nj * 4);
    put(8, mend.data(), nj * 4);
    put(9, s_offs.data(), s_offs.size() * 8);
    put(10, s_lens.data(), s_lens.size() * 8);
    put(11, mseries.data(), nm * 4);
    put(12, mjob.data(), nm * 4);
    put(13, morder.data(), nm * 4);
    const int rc = ServerOps<T>::round(
        reinterpret_cast<const T *>(blob + o[0]), reinterpret_cast<const uint64_t *>(blob + o[4]),
        reinterpret_cast<const int *>(blob + o[5]), reinterpret_cast<const int *>(blob + o[6]),
        reinterpret_cast<const int *>(blob + o[7]), reinterpret_cast<const int *>(blob + o[8]), nj,
        max_clen, static_cast<const T *>(nullptr), reinterpret_cast<const uint64_t *>(blob + o[9]),
        reinterpret_cast<const uint64_t *>(blob + o[10]), reinterpret_cast<const int *>(blob + o[11]),
        reinterpret_cast<const int *>(blob + o[12]), reinterpret_cast<const int *>(blob + o[13]), nm,
        h_mlens.data(), mjob.data(), clenh.data(), flags.data(), reinterpret_cast<T *>(blob + o[1]),
        reinterpret_cast<uint32_t *>(blob + o[2]), reinterpret_cast<double *>(blob + o[3]),
        static_cast<int32_t *>(nullptr), static_cast<int64_t *>(nullptr), blob + o[14], wsb, st_);
    std::vector<T> nb(ctot);
    std::vector<double> deltas(nj);
    unsigned wait_err = 0;
    if (rc == ODBA_OK) {
      cudaMemcpyAsync(nb.data(), blob + o[1], ctot * sizeof(T), cudaMemcpyDeviceToHost, st_);
      cudaMemcpyAsync(deltas.data(), blob + o[3], nj * 8, cudaMemcpyDeviceToHost, st_);
      // the round's hand-off wait error word (byte 8 of its workspace)
      cudaMemcpyAsync(&wait_err, blob + o[14] + 8, sizeof wait_err, cudaMemcpyDeviceToHost, st_);
    }
    cudaFreeAsync(blob, st_);
    if (rc != ODBA_OK || cudaStreamSynchronize(st_) != cudaSuccess) {
      cudaGetLastError();
      for (auto &r : rj) finish(r, kFailed, ODBA_ERR_CUDA);
      return;
    }
    if (wait_err) {
      for (auto &r : rj) finish(r, kFailed, ODBA_ERR_TIMEOUT);
      return;
    }
    cells_ += rcells;
    for (int j = 0; j < nj; ++j) {
      auto &r = rj[j];
      std::vector<T> v(nb.begin() + coff[j], nb.begin() + coff[j] + clen[j]);
      const int round = r->rounds;
      r->rounds++;
      r->delta = deltas[j];
      bool done = deltas[j] == 0;
      if (!done && (r->flags & 3)) {
        if (round >= 1 && !std::memcmp(v.data(), r->two_prev.data(), sizeof(T) * v.size())) done = true;
        if (!done) {
          if (round > 1) r->two_prev = r->prev;
          if (round > 0) r->prev = v;
        }
      }
      r->centroid = v;
      if (done || r->rounds >= 250) complete_job(r);
    }
  }

  void complete_job(std::shared_ptr<Request<T>> r) {
    r->result = r->centroid;
    if (r->norm)
      for (auto &x : r->result) x = (T)(r->means[r->medoid] + x * r->sigmas[r->medoid]);
    finish(r, kDone);
  }

  size_t budget_;
  int device_;
  cudaStream_t st_ = nullptr;
  cudaMemPool_t pool_ = nullptr;
  std::mutex mu_, cmu_;
  std::condition_variable cv_, done_cv_;
  bool stop_ = false;
  int64_t next_id_ = 1;
  size_t used_ = 0;
  std::map<int64_t, std::shared_ptr<Request<T>>> reqs_;
  std::deque<std::shared_ptr<Request<T>>> pending_;
  std::vector<std::shared_ptr<Request<T>>> active_;
  std::vector<Centroid> centroids_;
  std::thread worker_;
  std::atomic<uint64_t> iters_{0}, cells_{0};
  std::atomic<double> busy_{0.0};
};

struct ServerHandle {
  int elem_size;
  void *impl;
};

}  // namespace

extern "C" {

void *odba_server_create(int elem_size, size_t hbm_budget_bytes, int device) {
  auto *h = new ServerHandle{elem_size == 8 ? 8 : 4, nullptr};
  if (h->elem_size == 8)
    h->impl = new Server<double>(hbm_budget_bytes, device);
  else
    h->impl = new Server<float>(hbm_budget_bytes, device);
  return h;
}

void odba_server_destroy(void *handle) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h) return;
  if (h->elem_size == 8)
    delete static_cast<Server<double> *>(h->impl);
  else
    delete static_cast<Server<float> *>(h->impl);
  delete h;
}

#define ODBA_SRV(h, call) \
  ((h)->elem_size == 8 ? static_cast<Server<double> *>((h)->impl)->call : static_cast<Server<float> *>((h)->impl)->call)

int odba_server_add_centroid(void *handle, const void *h_centroid, uint64_t len) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h || !h_centroid || len == 0) return -ODBA_ERR_INVALID_ARGUMENT;
  if (h->elem_size == 8)
    return static_cast<Server<double> *>(h->impl)->add_centroid(static_cast<const double *>(h_centroid), len);
  return static_cast<Server<float> *>(h->impl)->add_centroid(static_cast<const float *>(h_centroid), len);
}

int64_t odba_server_submit_query(void *handle, const void *h_reads, const uint64_t *h_read_lens,
                                 int nreads, const int *centroid_ids, int ncentroids, int flags) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h || !h_reads || !h_read_lens || nreads < 1 || !centroid_ids || ncentroids < 1)
    return -ODBA_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < nreads; ++i)
    if (h_read_lens[i] == 0) return -ODBA_ERR_INVALID_ARGUMENT;
  if (h->elem_size == 8)
    return static_cast<Server<double> *>(h->impl)->submit_query(static_cast<const double *>(h_reads),
                                                                h_read_lens, nreads, centroid_ids, ncentroids, flags);
  return static_cast<Server<float> *>(h->impl)->submit_query(static_cast<const float *>(h_reads),
                                                             h_read_lens, nreads, centroid_ids, ncentroids, flags);
}

int64_t odba_server_submit_job(void *handle, const void *h_series, const uint64_t *h_lens, int n,
                               int flags, int norm) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h || !h_series || !h_lens || n < 1) return -ODBA_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (h_lens[i] == 0) return -ODBA_ERR_INVALID_ARGUMENT;
  if (h->elem_size == 8)
    return static_cast<Server<double> *>(h->impl)->submit_job(static_cast<const double *>(h_series), h_lens, n, flags, norm);
  return static_cast<Server<float> *>(h->impl)->submit_job(static_cast<const float *>(h_series), h_lens, n, flags, norm);
}

int odba_server_poll(void *handle, int64_t request) {
  auto *h = static_cast<ServerHandle *>(handle);
  return h ? ODBA_SRV(h, poll(request)) : -ODBA_ERR_INVALID_ARGUMENT;
}

int odba_server_wait(void *handle, int64_t request, double timeout_s) {
  auto *h = static_cast<ServerHandle *>(handle);
  return h ? ODBA_SRV(h, wait(request, timeout_s)) : -ODBA_ERR_INVALID_ARGUMENT;
}

int odba_server_take(void *handle, int64_t request, void *h_out, uint64_t capacity,
                     uint64_t *out_len, int *medoid, int *rounds, double *latency_s) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h) return ODBA_ERR_INVALID_ARGUMENT;
  if (h->elem_size == 8)
    return static_cast<Server<double> *>(h->impl)->take(request, static_cast<double *>(h_out), capacity,
                                                        out_len, medoid, rounds, latency_s);
  return static_cast<Server<float> *>(h->impl)->take(request, static_cast<float *>(h_out), capacity, out_len,
                                                     medoid, rounds, latency_s);
}

int odba_server_stats(void *handle, uint64_t *iterations, uint64_t *cells, double *busy_s) {
  auto *h = static_cast<ServerHandle *>(handle);
  if (!h || !iterations || !cells || !busy_s) return ODBA_ERR_INVALID_ARGUMENT;
  ODBA_SRV(h, stats(iterations, cells, busy_s));
  return ODBA_OK;
}

}  // extern "C"
