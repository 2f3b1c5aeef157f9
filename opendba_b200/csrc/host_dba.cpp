// C++ host side of the drop-in: the reference's templated entry points
// (include/opendba.hpp) implemented over the C ABI, with the reference's
// input readers (cpu_utils.hpp), output writers (dba.hpp, io_utils.hpp) and
// control flow (performDBA, dba.hpp:863-1189; setupAndRun, openDBA.cuh:13-200).
//
// Files written, byte-identical to the reference for identical values
// (std::ostream default formatting, 6 significant digits):
//   <prefix>.pair_dists.txt             dba.hpp:186-216
//   <prefix>.avg.txt (append)           dba.hpp:1004-1031, 1126-1131
//   <prefix>.<c>.path<k>.txt            io_utils.hpp:285-323 (last round of each cluster)
//   <prefix>.<c>.evolving_centroid.txt  io_utils.hpp:57-76 (every round, removed on convergence)
//   <prefix>.segmented_seqs.txt         io_utils.hpp:242-261
// The reference rewrites every path file in every round; only the last
// round's version survives, so only that one is written here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <numeric>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "opendba.hpp"
#include "opendba_b200.h"
#include "text_parse.h"

namespace {

[[noreturn]] void die(int code) { std::exit(code); }

void check(int status, const char *what) {
  if (status != ODBA_OK) {
    std::cerr << "Device library error in " << what << ": " << odba_status_string(status) << ": "
              << odba_last_error() << std::endl;
    die(odba_exit::DEVICE_LIBRARY_ERROR);
  }
}

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::cerr << "CUDA error: " << cudaGetErrorString(e) << " (" << what << ")" << std::endl;
    die(int(e));
  }
}

bool file_exists(const std::string &f) {
  std::ifstream in(f);
  return in.good();
}

template <typename T>
struct Ops;
template <>
struct Ops<float> {
  static int pairwise(const float *s, const uint64_t *o, const uint64_t *l, int n, uint64_t ml,
                      int os, int oe, float *d, void *w, size_t wb, void *st) {
    return odba_dtw_pairwise_f32(s, o, l, n, ml, os, oe, d, w, wb, st);
  }
  static int znorm(float *s, const uint64_t *o, const uint64_t *l, int n, double *m, double *sg,
                   void *st) {
    return odba_znorm_f32(s, o, l, n, m, sg, st);
  }
  static int segment(const float *s, const uint64_t *o, const uint64_t *l, const uint64_t *hl,
                     int n, int minseg, float *med, void *w, size_t wb, void *st) {
    return odba_segment_blocks_f32(s, o, l, hl, n, minseg, med, w, wb, st);
  }
  // stripe_rows < 0: full-path round; otherwise stripe mode with that tile height
  static int round(const float *c, uint64_t Lc, const float *s, const uint64_t *o,
                   const uint64_t *l, const uint64_t *hl, int n, int os, int oe, float *mean,
                   uint32_t *cnt, double *delta, int32_t *tri, int64_t *tc, void *w, size_t wb,
                   void *st, int stripe_rows = -1) {
    if (stripe_rows >= 0)
      return odba_dba_round_stripe_f32(c, Lc, s, o, l, hl, n, os, oe, stripe_rows, mean, cnt, delta,
                                       tri, tc, w, wb, st);
    return odba_dba_round_f32(c, Lc, s, o, l, hl, n, os, oe, mean, cnt, delta, tri, tc, w, wb, st);
  }
};
template <>
struct Ops<double> {
  static int pairwise(const double *s, const uint64_t *o, const uint64_t *l, int n, uint64_t ml,
                      int os, int oe, double *d, void *w, size_t wb, void *st) {
    return odba_dtw_pairwise_f64(s, o, l, n, ml, os, oe, d, w, wb, st);
  }
  static int znorm(double *s, const uint64_t *o, const uint64_t *l, int n, double *m, double *sg,
                   void *st) {
    return odba_znorm_f64(s, o, l, n, m, sg, st);
  }
  static int segment(const double *s, const uint64_t *o, const uint64_t *l, const uint64_t *hl,
                     int n, int minseg, double *med, void *w, size_t wb, void *st) {
    return odba_segment_blocks_f64(s, o, l, hl, n, minseg, med, w, wb, st);
  }
  // stripe_rows < 0: full-path round; otherwise stripe mode with that tile height
  static int round(const double *c, uint64_t Lc, const double *s, const uint64_t *o,
                   const uint64_t *l, const uint64_t *hl, int n, int os, int oe, double *mean,
                   uint32_t *cnt, double *delta, int32_t *tri, int64_t *tc, void *w, size_t wb,
                   void *st, int stripe_rows = -1) {
    if (stripe_rows >= 0)
      return odba_dba_round_stripe_f64(c, Lc, s, o, l, hl, n, os, oe, stripe_rows, mean, cnt, delta,
                                       tri, tc, w, wb, st);
    return odba_dba_round_f64(c, Lc, s, o, l, hl, n, os, oe, mean, cnt, delta, tri, tc, w, wb, st);
  }
};

// Full path or stripe mode for a DBA round.  Like the reference
// (dba.hpp:515-527), stripe mode is chosen when the full-path workspace does
// not fit in free device memory; ODBA_FORCE_STRIPE=1 forces it.  Returns the
// workspace bytes; *stripe_rows is -1 (full path) or the stripe tile height
// (0 = the library default).
template <typename T>
size_t round_workspace(const uint64_t *lens, int n, uint64_t Lc, int os, int oe, int *stripe_rows) {
  const size_t full = odba_dba_round_workspace_bytes(sizeof(T), lens, n, Lc, os, oe);
  *stripe_rows = -1;
  bool stripe = false;
  if (const char *f = std::getenv("ODBA_FORCE_STRIPE")) stripe = *f && *f != '0';
  if (!stripe) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && full > fr / 20 * 19) stripe = true;
    cudaGetLastError();
  }
  if (!stripe) return full;
  // tile height: ODBA_STRIPE_ROWS, else the smallest of 1024, 2048, ... whose
  // workspace fits in free memory (shorter tiles recompute with more warps
  // at once: 16 x 1M-4M members, 4096 rows 97 s, 1024 rows 75 s per round)
  int rows = 0;
  if (const char *r = std::getenv("ODBA_STRIPE_ROWS")) rows = std::atoi(r);
  if (rows <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
    cudaGetLastError();
    rows = 1024;
    while (rows < (1 << 20) &&
           odba_dba_round_stripe_workspace_bytes(sizeof(T), lens, n, Lc, os, oe, rows) > fr / 20 * 19)
      rows *= 2;
  }
  *stripe_rows = rows;
  return odba_dba_round_stripe_workspace_bytes(sizeof(T), lens, n, Lc, os, oe, rows);
}

// True if the launch that used workspace ws (pairwise or round) reported a
// swath hand-off wait that ran out: the error word at byte 8, which every
// launch clears.  Call after the launch's stream has synchronized.
bool wait_ran_out(const void *ws) {
  unsigned err = 0;
  check_cuda(cudaMemcpy(&err, static_cast<const char *>(ws) + 8, sizeof err, cudaMemcpyDeviceToHost),
             "wait error word");
  return err != 0;
}

// The pipeline's form: ends the process like the other device errors.
void check_wait(const void *ws, const char *what) {
  if (wait_ran_out(ws)) {
    std::cerr << what << ": a swath hand-off wait ran out on the device" << std::endl;
    die(odba_exit::DEVICE_LIBRARY_ERROR);
  }
}

// RAII device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  explicit DevBuf(size_t b = 0) { resize(b); }
  void resize(size_t b) {
    if (b <= bytes && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (b) {
      check_cuda(cudaMalloc(&p, b), "device allocation in the host façade");
      bytes = b;
    }
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

template <typename U>
U *ptr(const DevBuf &b) {
  return static_cast<U *>(b.p);
}

// A ragged set of series resident on the device, concatenated.
template <typename T>
struct DeviceSet {
  DevBuf data, offs, lens;
  std::vector<uint64_t> h_offs, h_lens;
  int n = 0;
  uint64_t max_len = 0, total = 0;

  // Copies sequences[i][0..lens[i]) from any memory space.
  void upload(T *const *sequences, const size_t *lengths, int count, cudaStream_t st) {
    n = count;
    h_offs.assign(n, 0);
    h_lens.assign(n, 0);
    total = 0;
    max_len = 0;
    for (int i = 0; i < n; ++i) {
      h_offs[i] = total;
      h_lens[i] = lengths[i];
      total += lengths[i];
      max_len = std::max<uint64_t>(max_len, lengths[i]);
    }
    data.resize((total + 16) * sizeof(T));
    offs.resize(std::max(1, n) * sizeof(uint64_t));
    lens.resize(std::max(1, n) * sizeof(uint64_t));
    for (int i = 0; i < n; ++i)
      check_cuda(cudaMemcpyAsync(ptr<T>(data) + h_offs[i], sequences[i], lengths[i] * sizeof(T),
                                 cudaMemcpyDefault, st),
                 "series upload");
    check_cuda(cudaMemcpyAsync(offs.p, h_offs.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st),
               "offsets upload");
    check_cuda(cudaMemcpyAsync(lens.p, h_lens.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st),
               "lengths upload");
  }
};

template <typename T>
std::vector<T> fetch_series(const T *p, size_t len) {
  std::vector<T> v(len);
  if (len) check_cuda(cudaMemcpy(v.data(), p, len * sizeof(T), cudaMemcpyDefault), "series read-back");
  return v;
}

// ---- path file (io_utils.hpp:285-323) ----
const char *move_name(int mv) {
  switch (mv) {
    case 1: return "DIAG";
    case 2: return "RIGHT";
    case 3: return "UP";
    case 4: return "OPEN_RIGHT";
    case 255: return "NIL";
    case 5: return "NIL_OPEN_RIGHT";
    default: return "?";
  }
}

template <typename T>
bool write_path_file(const std::string &fname, const char *name, const std::vector<T> &seq,
                     const std::vector<T> &centroid, bool flip, const int32_t *tri, int64_t count) {
  std::ofstream path(fname);
  if (!path.is_open()) {
    std::cerr << "Cannot write to " << fname << std::endl;
    return false;
  }
  // the reference's bytes (io_utils.hpp:287-323 ends lines with std::endl);
  // '\n' without the per-line flush keeps them in the stream's buffer
  path << name << '\n';
  for (int64_t k = 0; k + 1 < count; ++k) {
    const int i = tri[3 * k], j = tri[3 * k + 1], mv = tri[3 * k + 2];
    if (flip)
      path << j << '\t' << seq[j] << '\t' << i << '\t' << centroid[i] << '\t' << move_name(mv) << '\n';
    else
      path << i << '\t' << seq[i] << '\t' << j << '\t' << centroid[j] << '\t' << move_name(mv) << '\n';
  }
  if (count > 0) {
    const int64_t k = count - 1;
    const int i = tri[3 * k], j = tri[3 * k + 1], mv = tri[3 * k + 2];
    path << i << '\t' << seq[i] << '\t' << j << '\t' << centroid[j] << '\t'
         << (mv == 255 ? "NIL" : (mv == 5 ? "NIL_OPEN_RIGHT" : "?")) << '\n';
  }
  return true;
}

// ---- checkpoint (io_utils.hpp:57-115) ----
bool g_warned_checkpoint = false;

template <typename T>
void write_checkpoint(const std::string &fname, const T *c, size_t len) {
  std::ofstream f(fname);
  if (!f.is_open()) {
    if (!g_warned_checkpoint) {
      g_warned_checkpoint = true;
      std::cerr << "Cannot open centroid convergence checkpoint file " << fname
                << " for writing, no checkpointing for this cluster will be done (i.e. computation "
                   "cannot be resumed if the program dies unexpectedly)"
                << std::endl;
    }
    return;
  }
  // the stream's default output of each value (append_stream_value), one
  // write per round instead of one formatted insertion per value
  std::string line;
  line.reserve(len * 12 + 1);
  odba::append_stream_value(line, c[0]);
  for (size_t i = 1; i < len; ++i) {
    line += ' ';
    odba::append_stream_value(line, c[i]);
  }
  line += '\n';
  f.write(line.data(), std::streamsize(line.size()));
  f.flush();
}

template <typename T>
bool read_checkpoint(const std::string &fname, T *c, size_t len) {
  if (!file_exists(fname)) return false;
  std::ifstream f(fname);
  if (!f.is_open()) {
    std::cerr << "Cannot open existing centroid convergence checkpoint file " << fname
              << " for reading, will have to restart convergence for this cluster from the start (medoid)"
              << std::endl;
    return false;
  }
  std::string line;
  if (!std::getline(f, line)) {
    std::cerr << "Existing centroid convergence checkpoint file " << fname
              << "is blank, will have to restart convergence for this cluster from the start (centroid = medoid)"
              << std::endl;
    return false;
  }
  std::vector<std::string> values;
  {
    std::stringstream ss(line);
    std::string tok;
    while (std::getline(ss, tok, ' ')) values.push_back(tok);
  }
  if (values.size() != len) {
    std::cerr << "Existing centroid convergence checkpoint file " << fname
              << " contents does not have the same sequence length as the cluster medoid ("
              << values.size() << " != " << len
              << "), assuming corrupt checkpoint file and will have to restart convergence for this "
                 "cluster from the start (centroid = medoid)"
              << std::endl;
    return false;
  }
  std::cerr << "Resuming convergence from partially converged centroid in file " << fname << std::endl;
  std::stringstream ss(line);
  for (size_t i = 0; i < len; ++i) ss >> c[i];
  return true;
}

// ---- membership file (io_utils.hpp:160-240) ----
int *read_medoid_indices(const std::string &fname, int n, char **names, int *membership) {
  std::ifstream f(fname);
  if (!f.is_open()) {
    std::cerr << "Cannot open sequence cluster membership file " << fname << " for reading" << std::endl;
    die(odba_exit::CANNOT_READ_MEMBERSHIP);
  }
  std::string line;
  std::getline(f, line);
  if (line.compare(0, 1, "#")) {
    std::cerr << "The existing sequence cluster membership file " << fname
              << " has a first line without the expected '#' comment start" << std::endl;
    die(odba_exit::MEMBERSHIP_FILE_FORMAT_VIOLATION);
  }
  auto split = [](const std::string &s) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, '\t')) out.push_back(tok);
    return out;
  };
  auto find = [&](const std::string &nm) {
    for (int i = 0; i < n; ++i)
      if (nm.compare(names[i]) == 0) return i;
    return -1;
  };
  int max_cluster = 0, line_number = 1;
  std::vector<std::vector<std::string>> rows;
  while (std::getline(f, line)) {
    ++line_number;
    auto v = split(line);
    if (v.size() != 3) {
      std::cerr << "The existing sequence cluster membership file " << fname << " has a line (#"
                << line_number << ") without the expected three columns (found " << v.size() << ")"
                << std::endl;
      die(odba_exit::MEMBERSHIP_FILE_FORMAT_VIOLATION);
    }
    int cl = 0;
    try {
      cl = std::stoi(v[1]);
    } catch (const std::exception &ex) {
      std::cerr << "The existing sequence cluster membership file " << fname << " has a line (#"
                << line_number << ") where the second tab-delimited column value (" << v[1]
                << ") is not an integer as expected: " << ex.what() << std::endl;
      die(odba_exit::MEMBERSHIP_FILE_FORMAT_VIOLATION);
    }
    max_cluster = std::max(max_cluster, cl);
    const int si = find(v[0]);
    if (si == -1) {
      std::cerr << "The existing sequence cluster membership file " << fname << " has a line (#"
                << line_number << ") with a sequence name not found in the input (" << v[0]
                << " not in existing list of " << n << " names)" << std::endl;
      die(odba_exit::MEMBERSHIP_FILE_FORMAT_VIOLATION);
    }
    membership[si] = cl;
    rows.push_back(v);
  }
  // The reference sizes the medoid array by the largest cluster index it saw
  // (io_utils.hpp:220); one more slot keeps the last cluster addressable.
  int *medoids = new int[max_cluster + 1];
  for (int c = 0; c <= max_cluster; ++c) medoids[c] = -1;
  for (const auto &v : rows)
    if (v[0] == v[2]) medoids[std::stoi(v[1])] = find(v[0]);
  return medoids;
}

// pair_dists.txt (dba.hpp:186-216): row s holds the name of series s, s tabs,
// "\t0" and its distances to the later series, each after a tab; the last
// line is the last name, n tabs and "0".  Numbers print as the stream's
// default format prints them (append_stream_value).  Up to 16 threads
// format the rows (2 M numbers for 2000 series), which are then written in
// order.
template <typename T>
void write_pair_dists(const std::string &path, char **names, int n, const std::vector<T> &dists) {
  if (n < 1) return;
  std::vector<std::string> rows(size_t(n) - 1);
  std::vector<size_t> off(size_t(n), 0);
  for (int s = 1; s < n; ++s) off[s] = off[s - 1] + size_t(n - s);
  const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < nthreads; ++w) {
    pool.emplace_back([&, w]() {
      for (int s = int(w); s + 1 < n; s += int(nthreads)) {
        std::string &r = rows[s];
        r.reserve(size_t(s) + 16 + size_t(n - s) * 10);
        r += names[s];
        r.append(size_t(s), '\t');
        r += "\t0";
        const T *d = dists.data() + off[s];
        for (int j = s + 1; j < n; ++j) {
          r += '\t';
          odba::append_stream_value(r, d[j - s - 1]);
        }
        r += '\n';
      }
    });
  }
  for (auto &t : pool) t.join();
  std::ofstream mats(path.c_str(), std::ios::binary);
  for (const std::string &r : rows) mats.write(r.data(), std::streamsize(r.size()));
  mats << names[n - 1];
  for (int pad = 0; pad < n; ++pad) mats << "\t";
  mats << "0\n";
}

// Medoid pass on device-resident series: distances, pair_dists.txt, medoid
// (dba.hpp:170-351 for one cluster).
template <typename T>
int *medoid_pass(const T *d_data, const uint64_t *d_offs, const uint64_t *d_lens,
                 const std::vector<uint64_t> &h_lens, int n, uint64_t max_len, char **names, int os,
                 int oe, const char *output_prefix, double *cdist, int *memberships,
                 cudaStream_t st) {
  const size_t npairs = size_t(n) * (n - 1) / 2;
  std::vector<T> dists(npairs);
  if (n >= 2) {
    DevBuf d_dists(npairs * sizeof(T));
    DevBuf ws(odba_dtw_pairwise_workspace_bytes(sizeof(T), max_len));
    check(Ops<T>::pairwise(d_data, d_offs, d_lens, n, max_len, os, oe, ptr<T>(d_dists), ws.p,
                           ws.bytes, st),
          "all-pairs DTW");
    check_cuda(cudaMemcpyAsync(dists.data(), d_dists.p, npairs * sizeof(T), cudaMemcpyDeviceToHost, st),
               "distance download");
    check_cuda(cudaStreamSynchronize(st), "all-pairs DTW");
    check_wait(ws.p, "all-pairs DTW");
  }
  write_pair_dists<T>(std::string(output_prefix) + ".pair_dists.txt", names, n, dists);
  // complete linkage, the cut and the per-cluster medoids (dba.hpp:219-343)
  std::vector<int> med(std::max(n, 1), -1);
  int num_clusters = 1;
  check(sizeof(T) == 4
            ? odba_cluster_medoids_f32(n, reinterpret_cast<const float *>(dists.data()), h_lens.data(),
                                       *cdist, memberships, med.data(), &num_clusters)
            : odba_cluster_medoids_f64(n, reinterpret_cast<const double *>(dists.data()), h_lens.data(),
                                       *cdist, memberships, med.data(), &num_clusters),
        "clustering");
  std::cerr << "There are " << num_clusters << " clusters" << std::endl;
  int *medoids = new int[num_clusters];
  for (int c = 0; c < num_clusters; ++c) {
    if (med[c] == -1) {
      std::cerr << "Logic error in medoid finding routine" << std::endl;
      die(odba_exit::MEDOID_FINDING_ERROR);
    }
    medoids[c] = med[c];
    std::cerr << "Processing cluster " << c << " medoid is " << med[c] << std::endl;
  }
  return medoids;
}

// Runs DBA rounds for one cluster on device-resident members; returns the
// converged centroid (unscaled) and writes the checkpoint and path files.
template <typename T>
std::vector<T> converge_cluster(const DeviceSet<T> &all, const std::vector<int> &member_idx,
                                char **names, const std::vector<T> &seed, int os, int oe,
                                const std::string &cluster_prefix, cudaStream_t st) {
  const int n = int(member_idx.size());
  const size_t Lc = seed.size();
  std::vector<uint64_t> m_offs(n), m_lens(n);
  for (int k = 0; k < n; ++k) {
    m_offs[k] = all.h_offs[member_idx[k]];
    m_lens[k] = all.h_lens[member_idx[k]];
  }
  DevBuf d_moffs(n * sizeof(uint64_t)), d_mlens(n * sizeof(uint64_t));
  check_cuda(cudaMemcpyAsync(d_moffs.p, m_offs.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "member offsets");
  check_cuda(cudaMemcpyAsync(d_mlens.p, m_lens.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "member lengths");
  int stripe_rows = -1;
  DevBuf ws(round_workspace<T>(m_lens.data(), n, Lc, os, oe, &stripe_rows));
  DevBuf d_c(Lc * sizeof(T)), d_mean(Lc * sizeof(T)), d_counts(Lc * sizeof(uint32_t)),
      d_delta(sizeof(double));
  size_t cap = 0;
  for (int k = 0; k < n; ++k) cap += m_lens[k] + Lc + 1;
  DevBuf d_tri(3 * cap * sizeof(int32_t)), d_tc(n * sizeof(int64_t));
  std::vector<T> centroid = seed, input_centroid = seed, nb(Lc), prev(Lc, T(0)), two_prev(Lc, T(0));
  check_cuda(cudaMemcpyAsync(d_c.p, centroid.data(), Lc * sizeof(T), cudaMemcpyHostToDevice, st), "centroid upload");
  const int max_rounds = 250;
  const std::string ckpt = cluster_prefix + ".evolving_centroid.txt";
  for (int i = 0; i < max_rounds; ++i) {
    input_centroid = centroid;
    check(Ops<T>::round(ptr<T>(d_c), Lc, ptr<T>(all.data), ptr<uint64_t>(d_moffs),
                        ptr<uint64_t>(d_mlens), m_lens.data(), n, os, oe, ptr<T>(d_mean),
                        ptr<uint32_t>(d_counts), ptr<double>(d_delta), ptr<int32_t>(d_tri),
                        ptr<int64_t>(d_tc), ws.p, ws.bytes, st, stripe_rows),
          "DBA round");
    double delta = 0;
    check_cuda(cudaMemcpyAsync(nb.data(), d_mean.p, Lc * sizeof(T), cudaMemcpyDeviceToHost, st), "centroid download");
    check_cuda(cudaMemcpyAsync(&delta, d_delta.p, sizeof(double), cudaMemcpyDeviceToHost, st), "delta download");
    check_cuda(cudaStreamSynchronize(st), "DBA round");
    check_wait(ws.p, "DBA round");
    std::cerr << "New delta is " << delta << std::endl;
    if (delta == 0) break;
    if (os || oe) {
      // two_prev starts zeroed (fresh page-locked memory in the reference, dba.hpp:1053-1056)
      if (i >= 1 && !std::memcmp(nb.data(), two_prev.data(), sizeof(T) * Lc)) {
        std::cerr << "Detected a flip-flop between two alternative converged centroids (should "
                     "happen only in open end mode), keeping the first one calculated"
                  << std::endl;
        break;
      }
      if (i > 1) two_prev = prev;
      if (i > 0) prev = nb;
    }
    write_checkpoint(ckpt, nb.data(), Lc);
    centroid = nb;
    check_cuda(cudaMemcpyAsync(d_c.p, centroid.data(), Lc * sizeof(T), cudaMemcpyHostToDevice, st), "centroid upload");
  }
  // path files of the last round (each member against that round's input centroid)
  std::vector<int64_t> tc(n);
  std::vector<int32_t> tri(3 * cap);
  check_cuda(cudaMemcpy(tc.data(), d_tc.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost), "path counts");
  check_cuda(cudaMemcpy(tri.data(), d_tri.p, 3 * cap * sizeof(int32_t), cudaMemcpyDeviceToHost), "paths");
  std::vector<size_t> tri_off(n);
  size_t acc = 0;
  for (int k = 0; k < n; ++k) {
    tri_off[k] = acc;
    acc += m_lens[k] + Lc + 1;
  }
  const unsigned nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < nthreads; ++w) {
    pool.emplace_back([&, w]() {
      for (int k = int(w); k < n; k += int(nthreads)) {
        std::vector<T> seq(m_lens[k]);
        cudaMemcpy(seq.data(), ptr<T>(all.data) + m_offs[k], m_lens[k] * sizeof(T), cudaMemcpyDeviceToHost);
        const bool flip = oe && Lc < m_lens[k];
        write_path_file<T>(cluster_prefix + ".path" + std::to_string(k) + ".txt",
                           names[member_idx[k]], seq, input_centroid, flip,
                           tri.data() + 3 * tri_off[k], tc[k]);
      }
    });
  }
  for (auto &t : pool) t.join();
  return nb;
}

}  // namespace

// ---------------------------------------------------------------------------

template <typename T>
void normalizeSequences(T **sequences, size_t num_sequences, size_t *sequence_lengths,
                        int refSequenceIndex, double *sequence_means, double *sequence_sigmas,
                        cudaStream_t stream) {
  if (refSequenceIndex >= 0 && size_t(refSequenceIndex) < num_sequences) {
    std::cerr << "Rescaling to a reference sequence's mean and deviation is not available; "
                 "only z-normalisation (refSequenceIndex < 0)"
              << std::endl;
    die(odba_exit::DEVICE_LIBRARY_ERROR);
  }
  DeviceSet<T> ds;
  ds.upload(sequences, sequence_lengths, int(num_sequences), stream);
  DevBuf m(num_sequences * sizeof(double) + 8), s(num_sequences * sizeof(double) + 8);
  check(Ops<T>::znorm(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens),
                      int(num_sequences), ptr<double>(m), ptr<double>(s), stream),
        "z-normalisation");
  for (size_t i = 0; i < num_sequences; ++i)
    check_cuda(cudaMemcpyAsync(sequences[i], ptr<T>(ds.data) + ds.h_offs[i],
                               sequence_lengths[i] * sizeof(T), cudaMemcpyDefault, stream),
               "normalised series write-back");
  if (sequence_means)
    check_cuda(cudaMemcpyAsync(sequence_means, m.p, num_sequences * sizeof(double), cudaMemcpyDefault, stream), "means");
  if (sequence_sigmas)
    check_cuda(cudaMemcpyAsync(sequence_sigmas, s.p, num_sequences * sizeof(double), cudaMemcpyDefault, stream), "sigmas");
  check_cuda(cudaStreamSynchronize(stream), "z-normalisation");
}

template <typename T>
int *approximateMedoidIndices(T *gpu_sequences, size_t maxSeqLength, size_t num_sequences,
                              size_t *sequence_lengths, char **sequence_names, int use_open_start,
                              int use_open_end, char *output_prefix, double *cdist,
                              int *memberships, cudaStream_t stream) {
  const int n = int(num_sequences);
  std::vector<T *> ptrs(n);
  for (int i = 0; i < n; ++i) ptrs[i] = gpu_sequences + size_t(i) * maxSeqLength;
  DeviceSet<T> ds;
  ds.upload(ptrs.data(), sequence_lengths, n, stream);
  return medoid_pass<T>(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens), ds.h_lens,
                        n, ds.max_len, sequence_names, use_open_start, use_open_end, output_prefix,
                        cdist, memberships, stream);
}

template <typename T>
double DBAUpdate(T *C, size_t centerLength, T **sequences, char **sequence_names,
                 size_t num_sequences, size_t *sequence_lengths, int use_open_start,
                 int use_open_end, T *updatedMean, std::string output_prefix, cudaStream_t stream) {
  const int n = int(num_sequences);
  DeviceSet<T> ds;
  ds.upload(sequences, sequence_lengths, n, stream);
  std::vector<T> centroid = fetch_series(C, centerLength);
  int stripe_rows = -1;
  DevBuf ws(round_workspace<T>(ds.h_lens.data(), n, centerLength, use_open_start, use_open_end,
                               &stripe_rows));
  DevBuf d_c(centerLength * sizeof(T)), d_mean(centerLength * sizeof(T)),
      d_counts(centerLength * sizeof(uint32_t)), d_delta(sizeof(double));
  size_t cap = 0;
  for (int k = 0; k < n; ++k) cap += ds.h_lens[k] + centerLength + 1;
  DevBuf d_tri(3 * cap * sizeof(int32_t)), d_tc(n * sizeof(int64_t));
  check_cuda(cudaMemcpyAsync(d_c.p, centroid.data(), centerLength * sizeof(T), cudaMemcpyHostToDevice, stream), "centroid upload");
  check(Ops<T>::round(ptr<T>(d_c), centerLength, ptr<T>(ds.data), ptr<uint64_t>(ds.offs),
                      ptr<uint64_t>(ds.lens), ds.h_lens.data(), n, use_open_start, use_open_end,
                      ptr<T>(d_mean), ptr<uint32_t>(d_counts), ptr<double>(d_delta),
                      ptr<int32_t>(d_tri), ptr<int64_t>(d_tc), ws.p, ws.bytes, stream,
                      stripe_rows),
        "DBA round");
  double delta = 0;
  check_cuda(cudaMemcpyAsync(updatedMean, d_mean.p, centerLength * sizeof(T), cudaMemcpyDefault, stream), "centroid download");
  check_cuda(cudaMemcpyAsync(&delta, d_delta.p, sizeof(double), cudaMemcpyDeviceToHost, stream), "delta download");
  check_cuda(cudaStreamSynchronize(stream), "DBA round");
  check_wait(ws.p, "DBA round");
  if (!output_prefix.empty()) {
    std::vector<int64_t> tc(n);
    std::vector<int32_t> tri(3 * cap);
    check_cuda(cudaMemcpy(tc.data(), d_tc.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost), "path counts");
    check_cuda(cudaMemcpy(tri.data(), d_tri.p, 3 * cap * sizeof(int32_t), cudaMemcpyDeviceToHost), "paths");
    size_t off = 0;
    for (int k = 0; k < n; ++k) {
      std::vector<T> seq = fetch_series(ptr<T>(ds.data) + ds.h_offs[k], ds.h_lens[k]);
      const bool flip = use_open_end && centerLength < ds.h_lens[k];
      if (!write_path_file<T>(output_prefix + ".path" + std::to_string(k) + ".txt",
                              sequence_names[k], seq, centroid, flip, tri.data() + 3 * off, tc[k]))
        return odba_exit::CANNOT_WRITE_DTW_PATH_MATRIX;
      off += ds.h_lens[k] + centerLength + 1;
    }
  }
  return delta;
}

template <typename T>
void performDBA(T **sequences, int num_sequences, size_t *sequence_lengths, char **sequence_names,
                int use_open_start, int use_open_end, char *output_prefix, int norm_sequences,
                double cdist, char **series_file_names, int num_series, int read_mode,
                bool is_segmented, int algo_mode, cudaStream_t stream) {
  (void)series_file_names;
  (void)num_series;
  (void)read_mode;
  (void)is_segmented;
  const int n = num_sequences;
  // sanitise the last sample (dba.hpp:868-872)
  for (int i = 0; i < n; ++i) {
    if (sequence_lengths[i] == 0) continue;
    T last;
    check_cuda(cudaMemcpy(&last, sequences[i] + sequence_lengths[i] - 1, sizeof(T), cudaMemcpyDefault),
               "reading a last sample");
    if (last >= std::sqrt(std::numeric_limits<T>::max())) sequence_lengths[i]--;
  }
  // stable sort by length; pointers, names and lengths permuted in place (dba.hpp:876-885)
  {
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return sequence_lengths[a] < sequence_lengths[b]; });
    std::vector<T *> s2(n);
    std::vector<char *> n2(n);
    std::vector<size_t> l2(n);
    for (int i = 0; i < n; ++i) {
      s2[i] = sequences[order[i]];
      n2[i] = sequence_names[order[i]];
      l2[i] = sequence_lengths[order[i]];
    }
    for (int i = 0; i < n; ++i) {
      sequences[i] = s2[i];
      sequence_names[i] = n2[i];
      sequence_lengths[i] = l2[i];
    }
  }
  DeviceSet<T> ds;
  ds.upload(sequences, sequence_lengths, n, stream);
  std::vector<double> means(n, 0.0), sigmas(n, 1.0);
  if (norm_sequences) {
    DevBuf m(n * sizeof(double) + 8), s(n * sizeof(double) + 8);
    check(Ops<T>::znorm(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens), n,
                        ptr<double>(m), ptr<double>(s), stream),
          "z-normalisation");
    check_cuda(cudaMemcpyAsync(means.data(), m.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream), "means");
    check_cuda(cudaMemcpyAsync(sigmas.data(), s.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream), "sigmas");
    // the reference normalises the caller's series in place
    for (int i = 0; i < n; ++i)
      check_cuda(cudaMemcpyAsync(sequences[i], ptr<T>(ds.data) + ds.h_offs[i],
                                 sequence_lengths[i] * sizeof(T), cudaMemcpyDefault, stream),
                 "normalised series write-back");
    check_cuda(cudaStreamSynchronize(stream), "z-normalisation");
  }
  std::vector<int> membership(n, 0);
  int *medoids = nullptr;
  if (algo_mode == CLUSTER_AND_CONSENSUS || algo_mode == CLUSTER_ONLY) {
    medoids = medoid_pass<T>(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens),
                             ds.h_lens, n, ds.max_len, sequence_names, use_open_start,
                             use_open_end, output_prefix, &cdist, membership.data(), stream);
  } else if (algo_mode == CONSENSUS_ONLY) {
    std::cerr << "Reading previous clustering data" << std::endl;
    medoids = read_medoid_indices(std::string(output_prefix) + ".cluster_membership.txt", n,
                                  sequence_names, membership.data());
  } else {
    std::cerr << "Call to performDBA included an unrecognized algorithm mode " << algo_mode
              << " (programming error, please contact the developer)" << std::endl;
    die(odba_exit::UNKNOWN_ALGO);
  }
  int num_clusters = 1;
  for (int i = 0; i < n; ++i) num_clusters = std::max(num_clusters, membership[i] + 1);
  if (cdist != 1 && algo_mode != CONSENSUS_ONLY) {
    const std::string mf = std::string(output_prefix) + ".cluster_membership.txt";
    std::ofstream membership_file(mf.c_str());
    if (!membership_file.is_open()) {
      std::cerr << "Cannot open sequence cluster membership file " << mf << " for writing" << std::endl;
      die(odba_exit::CANNOT_WRITE_MEMBERSHIP);
    }
    membership_file << "## cluster distance threshold was " << cdist << std::endl;
    for (int i = 0; i < n; ++i)
      membership_file << sequence_names[i] << "\t" << membership[i] << "\t"
                      << sequence_names[medoids[membership[i]]] << std::endl;
  }
  if (algo_mode == CLUSTER_ONLY) {
    delete[] medoids;
    return;
  }
  const std::string avg_name = std::string(output_prefix) + ".avg.txt";
  int curr = 0;
  if (file_exists(avg_name)) {
    // text-mode builds of the reference count no finished averages and always
    // resume at cluster index 1 (io_utils.hpp:119-123, dba.hpp:982-986)
    curr = 1;
    std::cerr << "Restarting convergence with cluster " << (curr + 1) << "/" << num_clusters
              << " based on checkpoint in " << avg_name << std::endl;
  }
  std::ofstream avgs(avg_name.c_str(), std::ios::app);
  if (!avgs.is_open()) {
    std::cerr << "Cannot open sequence averages file " << output_prefix << ".avg.txt for writing" << std::endl;
    die(odba_exit::CANNOT_WRITE_DBA_AVG);
  }
  for (; curr < num_clusters; ++curr) {
    std::vector<int> members;
    for (int i = 0; i < n; ++i)
      if (membership[i] == curr) members.push_back(i);
    const int med = medoids[curr];
    const size_t medoid_len = sequence_lengths[med];
    std::vector<T> medoid_seq = fetch_series(ptr<T>(ds.data) + ds.h_offs[med], medoid_len);
    if (members.size() == 1) {
      std::cerr << "Outputting singleton sequence " << sequence_names[med] << " as-is (a.k.a. cluster "
                << (curr + 1) << "/" << num_clusters << ")." << std::endl;
      avgs << sequence_names[med];
      for (size_t i = 0; i < medoid_len; ++i) {
        if (norm_sequences)
          avgs << "\t" << ((T)(means[med] + medoid_seq[i] * sigmas[med]));
        else
          avgs << "\t" << medoid_seq[i];
      }
      avgs << std::endl;
      avgs.flush();
      continue;
    }
    const std::string cprefix = std::string(output_prefix) + "." + std::to_string(curr);
    std::vector<T> seed = medoid_seq;
    read_checkpoint(cprefix + ".evolving_centroid.txt", seed.data(), medoid_len);
    std::cerr << "Processing cluster " << (curr + 1) << " of " << num_clusters << ", "
              << members.size() << " members, medoid " << sequence_names[med] << " has length "
              << medoid_len << std::endl;
    std::vector<T> nb = converge_cluster<T>(ds, members, sequence_names, seed, use_open_start,
                                            use_open_end, cprefix, stream);
    if (norm_sequences)
      for (size_t i = 0; i < medoid_len; ++i) nb[i] = (T)(means[med] + nb[i] * sigmas[med]);
    avgs << sequence_names[med];
    for (size_t i = 0; i < medoid_len; ++i) avgs << "\t" << nb[i];
    avgs << std::endl;
    avgs.flush();
    const std::string ck = cprefix + ".evolving_centroid.txt";
    if (std::remove(ck.c_str()) != 0)
      std::cerr << "Warning: could not remove temporary checkpoint file " << ck << std::endl;
  }
  delete[] medoids;
}

// Block-edge merge and sentinel removal after the segmentation kernel
// (segmentation.hpp:486-578).  segmented_sequences / segmented_seq_lengths are
// allocated with cudaMallocManaged, as the reference does, for the caller to free.
template <typename T>
void adaptive_segmentation(T **sequences, size_t *seq_lengths, int num_seqs, int min_segment_length,
                           T ***segmented_sequences, size_t **segmented_seq_lengths,
                           int prefix_length_to_skip, cudaStream_t stream) {
  const int n = num_seqs;
  DeviceSet<T> ds;
  ds.upload(sequences, seq_lengths, n, stream);
  const size_t cap = odba_segment_capacity(ds.h_lens.data(), n, min_segment_length);
  DevBuf d_med(std::max<size_t>(cap, 1) * sizeof(T));
  DevBuf ws(odba_segment_workspace_bytes(n));
  check(Ops<T>::segment(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens),
                        ds.h_lens.data(), n, min_segment_length, ptr<T>(d_med), ws.p, ws.bytes,
                        stream),
        "segmentation");
  std::vector<T> med(cap);
  check_cuda(cudaMemcpyAsync(med.data(), d_med.p, cap * sizeof(T), cudaMemcpyDeviceToHost, stream), "segment download");
  check_cuda(cudaStreamSynchronize(stream), "segmentation");
  check_cuda(cudaMallocManaged(segmented_sequences, sizeof(T *) * std::max(1, n)), "segmented sequence pointers");
  check_cuda(cudaMallocManaged(segmented_seq_lengths, sizeof(size_t) * std::max(1, n)), "segmented lengths");
  int dw = (min_segment_length + 2) / 3;
  const int spb = 256 * dw;
  const float per = float(min_segment_length) / float(dw);
  const int k_max = int((256 + per - 1) / per);
  const T TMAX = std::numeric_limits<T>::max();
  size_t base = 0;
  for (int i = 0; i < n; ++i) {
    T *seg = med.data() + base;
    const size_t slen = size_t(k_max) * size_t((ds.h_lens[i] + spb - 1) / spb);
    base += slen;
    T epsilon = TMAX;
    T previous = seg[0];
    for (size_t j = 1; j < slen; ++j) {
      const T current = seg[j];
      if (current != TMAX && previous != TMAX &&
          ((current <= previous && previous - current < epsilon) ||
           (current > previous && current - previous < epsilon))) {
        if (current - previous == 0) {
          for (size_t k = j; k < slen; k++) {
            seg[k - 1] = seg[k];
            if (seg[k] == TMAX) break;
          }
        } else {
          epsilon = current < previous ? (previous - current) : (current - previous);
        }
      }
      previous = current;
    }
    bool prev_undef = false;
    long cursor = 0;
    for (size_t j = 0; j < slen; ++j) {
      if (seg[j] == TMAX) {
        prev_undef = true;
        continue;
      }
      if (prev_undef) {
        prev_undef = false;
        if (cursor >= 1 && seg[cursor - 1] < seg[j] + epsilon && seg[cursor - 1] > seg[j] - epsilon)
          seg[cursor - 1] = (seg[cursor - 1] + seg[j]) / 2;
      }
      if (size_t(cursor) != j) seg[cursor] = seg[j];
      cursor++;
    }
    if (cursor >= 1 && seg[cursor - 1] >= TMAX / 2) cursor--;
    long skipped = 0;
    if (prefix_length_to_skip) {
      if (cursor <= prefix_length_to_skip) {
        skipped = cursor - 1;
        cursor = 1;
      } else {
        skipped = prefix_length_to_skip;
        cursor -= prefix_length_to_skip;
      }
    }
    (*segmented_seq_lengths)[i] = size_t(cursor);
    check_cuda(cudaMallocManaged(&(*segmented_sequences)[i], sizeof(T) * std::max<long>(cursor, 1)),
               "a segmented sequence");
    std::memcpy((*segmented_sequences)[i], seg + skipped, sizeof(T) * size_t(cursor));
  }
}

// ---------------------------------------------------------------------------
// Readers (cpu_utils.hpp:60-134, 381-456, 553-624).

namespace {

// One value per line for every newline in the file (a last line without one
// is not read), each the first token of its line (parse_line_value).
template <typename T>
int read_text_data(const char *fname, std::vector<T> &out) {
  std::ifstream ifs(fname, std::ios::binary);
  if (!ifs) {
    std::cerr << "Error reading in file " << fname << ", skipping" << std::endl;
    return 1;
  }
  std::string text;
  {
    std::vector<char> buf(1 << 20);
    while (true) {
      ifs.read(buf.data(), buf.size());
      const std::streamsize got = ifs.gcount();
      if (got <= 0) break;
      text.append(buf.data(), size_t(got));
    }
  }
  const size_t lines = size_t(std::count(text.begin(), text.end(), '\n'));
  if (lines == 0) {
    std::cerr << "File " << fname << " is empty or not properly formatted. Skipping." << std::endl;
    return 1;
  }
  out.assign(lines, T(0));
  const char *p = text.data();
  for (size_t i = 0; i < lines; ++i) {
    const char *nl = static_cast<const char *>(std::memchr(p, '\n', text.data() + text.size() - p));
    out[i] = odba::parse_line_value<T>(p, nl);
    p = nl + 1;
  }
  return 0;
}

template <typename T>
int read_binary_data(const char *fname, std::vector<T> &out, bool is_short) {
  std::ifstream ifs(fname, std::ios::binary);
  if (!ifs) return 1;
  ifs.seekg(0, ifs.end);
  const std::streamoff bytes = ifs.tellg();
  ifs.seekg(0, std::ios::beg);
  if (is_short) {
    std::vector<short> raw(size_t(bytes) / 2);
    ifs.read(reinterpret_cast<char *>(raw.data()), raw.size() * 2);
    out.resize(raw.size());
    for (size_t i = 0; i < raw.size(); ++i) out[i] = T(float(raw[i]));
  } else {
    out.resize(size_t(bytes) / sizeof(T));
    ifs.read(reinterpret_cast<char *>(out.data()), out.size() * sizeof(T));
  }
  return 0;
}

template <typename T>
int read_tsv_data(const char *fname, std::vector<std::vector<T>> &seqs,
                  std::vector<std::string> &names) {
  std::ifstream ifs(fname);
  if (!ifs) return 0;
  int count = 0;
  for (std::string line; std::getline(ifs, line);) {
    const size_t cols = size_t(std::count(line.begin(), line.end(), '\t'));
    std::vector<T> s(cols, T(0));
    std::istringstream iss(line);
    std::string name;
    iss >> name;
    size_t k = 0;
    while (iss.good()) {
      T v = T(0);
      iss >> v;
      if (k < cols) s[k] = v;
      ++k;
    }
    seqs.push_back(std::move(s));
    names.push_back(name);
    ++count;
  }
  return count;
}

char *dup_cstr(const std::string &s) {
  char *p = new char[s.size() + 1];
  std::memcpy(p, s.c_str(), s.size() + 1);
  return p;
}

template <typename T>
int write_sequences(T **seqs, size_t *lens, char **names, int n, const std::string &fname) {
  std::ofstream out(fname);
  if (!out.is_open()) {
    std::cerr << "Cannot write to " << fname << std::endl;
    return odba_exit::CANNOT_WRITE_DTW_PATH_MATRIX;
  }
  for (int i = 0; i < n; ++i) {
    std::vector<T> s = fetch_series(seqs[i], lens[i]);
    out << names[i] << "\t" << s[0];
    for (size_t j = 1; j < lens[i]; ++j) out << "\t" << s[j];
    out << std::endl;
  }
  return 0;
}

// The alignment half of chopPrefixFromSequences (dba.hpp:1191-1336): with
// norm, the leader and the series are z-normalised (the series in place, as
// the reference does to its managed copies); then every series' chop position
// and leader-row histogram.
template <typename T>
void prefix_chop_core(const T *prefix, size_t P, T **seqs, const size_t *lens, int n, int norm,
                      std::vector<long long> &chop, std::vector<int> &hist, cudaStream_t st) {
  DeviceSet<T> ds;
  ds.upload(seqs, lens, n, st);
  DevBuf d_pre((P + 16) * sizeof(T));
  check_cuda(cudaMemcpyAsync(d_pre.p, prefix, P * sizeof(T), cudaMemcpyDefault, st), "prefix upload");
  if (norm) {
    const uint64_t zero = 0, plen = P;
    DevBuf po(sizeof(uint64_t)), pl(sizeof(uint64_t));
    check_cuda(cudaMemcpyAsync(po.p, &zero, 8, cudaMemcpyHostToDevice, st), "prefix offset");
    check_cuda(cudaMemcpyAsync(pl.p, &plen, 8, cudaMemcpyHostToDevice, st), "prefix length");
    check(Ops<T>::znorm(ptr<T>(d_pre), ptr<uint64_t>(po), ptr<uint64_t>(pl), 1, nullptr, nullptr, st),
          "prefix z-normalisation");
    check(Ops<T>::znorm(ptr<T>(ds.data), ptr<uint64_t>(ds.offs), ptr<uint64_t>(ds.lens), n, nullptr,
                        nullptr, st),
          "z-normalisation for prefix chopping");
    for (int i = 0; i < n; ++i)
      check_cuda(cudaMemcpyAsync(seqs[i], ptr<T>(ds.data) + ds.h_offs[i], lens[i] * sizeof(T),
                                 cudaMemcpyDefault, st),
                 "normalised series write-back");
    check_cuda(cudaStreamSynchronize(st), "z-normalisation for prefix chopping");
  }
  DevBuf ws(odba_prefix_chop_workspace_bytes(sizeof(T), ds.h_lens.data(), n, P));
  DevBuf d_chop(n * sizeof(long long)), d_hist(size_t(n) * P * sizeof(int));
  check(sizeof(T) == 4
            ? odba_prefix_chop_f32(reinterpret_cast<const float *>(d_pre.p), P,
                                   reinterpret_cast<const float *>(ds.data.p), ptr<uint64_t>(ds.offs),
                                   ptr<uint64_t>(ds.lens), ds.h_lens.data(), n,
                                   reinterpret_cast<int64_t *>(d_chop.p), ptr<int32_t>(d_hist), ws.p,
                                   ws.bytes, st)
            : odba_prefix_chop_f64(reinterpret_cast<const double *>(d_pre.p), P,
                                   reinterpret_cast<const double *>(ds.data.p), ptr<uint64_t>(ds.offs),
                                   ptr<uint64_t>(ds.lens), ds.h_lens.data(), n,
                                   reinterpret_cast<int64_t *>(d_chop.p), ptr<int32_t>(d_hist), ws.p,
                                   ws.bytes, st),
        "prefix chop");
  chop.assign(n, 0);
  hist.assign(size_t(n) * P, 0);
  check_cuda(cudaMemcpyAsync(chop.data(), d_chop.p, n * sizeof(long long), cudaMemcpyDeviceToHost, st),
             "chop positions");
  check_cuda(cudaMemcpyAsync(hist.data(), d_hist.p, size_t(n) * P * sizeof(int), cudaMemcpyDeviceToHost, st),
             "leader histograms");
  check_cuda(cudaStreamSynchronize(st), "prefix chop");
  for (int i = 0; i < n; ++i)
    if (chop[i] < 0) {
      std::cerr << "Prefix chop: the path walk of series " << i << " failed" << std::endl;
      die(odba_exit::DEVICE_LIBRARY_ERROR);
    }
}

// One line of <prefix>.prefix_chop.txt (dba.hpp:1346-1351).
void write_chop_line(std::ofstream &f, const char *name, long long chop, size_t len, const int *hist,
                     size_t P) {
  f << name << "\t" << chop << "\t" << len;
  for (size_t j = 0; j < P; ++j) f << "\t" << hist[j];
  f << std::endl;
}

}  // namespace

template <typename T>
void setupAndRun(char *seqprefix_file_name, char **series_file_names, int num_series,
                 char *output_prefix, int read_mode, int use_open_start, int use_open_end,
                 char *min_segment_length_string, int norm_sequences, double cdist,
                 const int prefix_start, const int prefix_length, bool is_short) {
  int min_segment_length_2 = -1;
  char *pos = std::strchr(min_segment_length_string, ',');
  if (pos) {
    min_segment_length_2 = std::atoi(pos + 1);
    *pos = '\0';
  }
  const int min_segment_length = std::atoi(min_segment_length_string);

  std::vector<std::vector<T>> data;
  std::vector<std::string> names;
  if (read_mode == TSV_READ_MODE) {
    std::cerr << "Step 1 of 3: Loading " << num_series << (num_series == 1 ? " TSV data file" : " TSV data files") << std::endl;
    for (int i = 0; i < num_series; ++i)
      if (read_tsv_data<T>(series_file_names[i], data, names) < 1)
        std::cerr << "Error reading in TSV file " << series_file_names[i] << ", skipping" << std::endl;
  } else {
    const bool binary = read_mode == BINARY_READ_MODE;
    std::cerr << "Step 1 of 3: Loading " << num_series
              << (binary ? (num_series == 1 ? " binary data file" : " binary data files")
                         : (num_series == 1 ? " text data file" : " text data files"))
              << ", total sequence count " << num_series << std::endl;
    for (int i = 0; i < num_series; ++i) {
      std::vector<T> s;
      const int rc = binary ? read_binary_data<T>(series_file_names[i], s, is_short)
                            : read_text_data<T>(series_file_names[i], s);
      if (rc) {
        std::cerr << "Error reading in " << (binary ? "binary" : "text") << " file "
                  << series_file_names[i] << ", skipping" << std::endl;
        continue;
      }
      data.push_back(std::move(s));
      names.push_back(series_file_names[i]);
    }
  }
  int n = int(data.size());
  if (n < 2) {
    std::cerr << "At least two sequences must be provided to calculate an average, but found " << n
              << ", aborting" << std::endl;
    die(odba_exit::NOT_ENOUGH_SEQUENCES);
  }
  // shorten names to everything before the first "." (openDBA.cuh:58-59)
  for (auto &nm : names) {
    const size_t dot = nm.find('.');
    if (dot != std::string::npos) nm.resize(dot);
  }
  // Step 1: chop a leading sequence off all inputs (openDBA.cuh:61-83, dba.hpp:1191-1395)
  if (seqprefix_file_name != nullptr) {
    std::vector<T> leader;
    const bool binary = read_mode == BINARY_READ_MODE;
    const int rc = binary ? read_binary_data<T>(seqprefix_file_name, leader, false)
                          : read_text_data<T>(seqprefix_file_name, leader);
    if (rc || leader.empty()) {
      std::cerr << "Cannot read prefix " << (binary ? "binary" : "text") << " data from "
                << seqprefix_file_name << ", aborting" << std::endl;
      die(odba_exit::CANNOT_READ_SEQUENCE_PREFIX_FILE);
    }
    std::vector<T *> ptrs(n);
    std::vector<size_t> lns(n);
    for (int i = 0; i < n; ++i) {
      ptrs[i] = data[i].data();
      lns[i] = data[i].size();
    }
    std::vector<long long> chop;
    std::vector<int> hist;
    prefix_chop_core<T>(leader.data(), leader.size(), ptrs.data(), lns.data(), n, norm_sequences,
                        chop, hist, 0);
    std::ofstream cf((std::string(output_prefix) + ".prefix_chop.txt").c_str());
    std::vector<std::vector<T>> kept;
    std::vector<std::string> kept_names;
    for (int i = 0; i < n; ++i) {
      write_chop_line(cf, names[i].c_str(), chop[i], lns[i], hist.data() + size_t(i) * leader.size(),
                      leader.size());
      if (lns[i] - size_t(chop[i]) == 0) {
        std::cerr << "Skipping " << names[i] << " due to zero-length after prefix chopping" << std::endl;
        continue;
      }
      kept.emplace_back(data[i].begin() + chop[i], data[i].end());
      kept_names.push_back(names[i]);
    }
    data.swap(kept);
    names.swap(kept_names);
    n = int(data.size());
  }
  std::vector<T *> seq_ptrs(n);
  std::vector<size_t> lens(n);
  std::vector<char *> name_ptrs(n);
  for (int i = 0; i < n; ++i) {
    seq_ptrs[i] = data[i].data();
    lens[i] = data[i].size();
    name_ptrs[i] = dup_cstr(names[i]);
  }
  T **segs = nullptr;
  size_t *seglens = nullptr;
  if (min_segment_length > 0) {
    adaptive_segmentation<T>(seq_ptrs.data(), lens.data(), n, min_segment_length, &segs, &seglens,
                             prefix_start);
    int removed = 0;
    for (int i = 0; i < n; ++i) {
      const int j = i - removed;
      if (seglens[j] < 2 || (prefix_length > 0 && seglens[j] < size_t(prefix_length))) {
        cudaFree(segs[j]);
        for (int k = j + 1; k < n - removed; ++k) {
          segs[k - 1] = segs[k];
          seglens[k - 1] = seglens[k];
          name_ptrs[k - 1] = name_ptrs[k];
        }
        ++removed;
      }
    }
    if (removed) {
      std::cerr << "Removing " << removed << " segmented sequences that are too short, as they may "
                << "unduly skew the convergence process. To retain more sequences, consider setting "
                << "a smaller minimum segment size (currently " << min_segment_length << ")" << std::endl;
      n -= removed;
      if (n < 2) {
        std::cerr << "At least two sequences must survive segmentation filters to calculate an "
                     "average, but found " << n << ", aborting" << std::endl;
        die(odba_exit::NOT_ENOUGH_SEQUENCES);
      }
    }
    if (prefix_length > 0)
      for (int i = 0; i < n; ++i) seglens[i] = size_t(prefix_length);
    write_sequences<T>(segs, seglens, name_ptrs.data(), n,
                       std::string(output_prefix) + ".segmented_seqs.txt");
    if (min_segment_length_2 != -1) {
      std::cerr << "Performing cluster generation with segment size of " << min_segment_length << std::endl;
      performDBA<T>(segs, n, seglens, name_ptrs.data(), use_open_start, use_open_end, output_prefix,
                    norm_sequences, cdist, series_file_names, num_series, read_mode,
                    min_segment_length > 1, CLUSTER_ONLY);
    } else {
      for (int i = 0; i < n; ++i) {
        seq_ptrs[i] = segs[i];
        lens[i] = seglens[i];
      }
    }
  }
  if (min_segment_length_2 != -1) {
    std::cerr << "Performing consensus generation with segment size of " << min_segment_length_2 << std::endl;
    performDBA<T>(seq_ptrs.data(), n, lens.data(), name_ptrs.data(), use_open_start, use_open_end,
                  output_prefix, norm_sequences, cdist, series_file_names, num_series, read_mode,
                  min_segment_length > 1, CONSENSUS_ONLY);
  } else {
    std::cerr << "Performing both clustering and consensus generation with segment size of "
              << min_segment_length << std::endl;
    performDBA<T>(seq_ptrs.data(), n, lens.data(), name_ptrs.data(), use_open_start, use_open_end,
                  output_prefix, norm_sequences, cdist, series_file_names, num_series, read_mode,
                  min_segment_length > 1, CLUSTER_AND_CONSENSUS);
  }
  if (segs) {
    for (int i = 0; i < n; ++i) cudaFree(segs[i]);
    cudaFree(segs);
    cudaFree(seglens);
  }
  for (auto p : name_ptrs) delete[] p;
}

// chopPrefixFromSequences<T> (dba.hpp:1191-1395) with the reference's
// signature and side effects: with norm_sequences the caller's series are
// z-normalised in place; <output_prefix>.prefix_chop.txt is written; every
// series is replaced by a new cudaMallocManaged copy of its chopped tail (the
// old array is released with cudaFree when it is CUDA memory, as the
// reference's managed inputs are); series left empty are dropped and
// *num_sequences shrinks.
template <typename T>
void chopPrefixFromSequences(T *sequence_prefix, size_t sequence_prefix_length, T **sequences,
                             int *num_sequences, size_t *sequence_lengths, char **sequence_names,
                             char *output_prefix, int norm_sequences, cudaStream_t stream) {
  const int n = *num_sequences;
  const size_t P = sequence_prefix_length;
  std::vector<long long> chop;
  std::vector<int> hist;
  prefix_chop_core<T>(sequence_prefix, P, sequences, sequence_lengths, n, norm_sequences, chop, hist,
                      stream);
  std::ofstream cf((std::string(output_prefix) + ".prefix_chop.txt").c_str());
  int out = 0;
  for (int i = 0; i < n; ++i) {
    write_chop_line(cf, sequence_names[i], chop[i], sequence_lengths[i], hist.data() + size_t(i) * P, P);
    const size_t kept = sequence_lengths[i] - size_t(chop[i]);
    cudaPointerAttributes attr;
    const bool cuda_mem = cudaPointerGetAttributes(&attr, sequences[i]) == cudaSuccess &&
                          (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    if (kept == 0) {
      std::cerr << "Skipping " << sequence_names[i] << " due to zero-length after prefix chopping" << std::endl;
      if (cuda_mem) cudaFree(sequences[i]);
      continue;
    }
    T *ns = nullptr;
    check_cuda(cudaMallocManaged(&ns, sizeof(T) * kept), "chopped sequence");
    check_cuda(cudaMemcpy(ns, sequences[i] + chop[i], sizeof(T) * kept, cudaMemcpyDefault),
               "chopped sequence copy");
    if (cuda_mem) cudaFree(sequences[i]);
    sequences[out] = ns;
    sequence_lengths[out] = kept;
    sequence_names[out] = sequence_names[i];
    ++out;
  }
  *num_sequences = out;
}

#define ODBA_INSTANTIATE(T)                                                                     \
  template void chopPrefixFromSequences<T>(T *, size_t, T **, int *, size_t *, char **, char *,  \
                                           int, cudaStream_t);                                   \
  template void setupAndRun<T>(char *, char **, int, char *, int, int, int, char *, int, double, \
                               const int, const int, bool);                                     \
  template void performDBA<T>(T **, int, size_t *, char **, int, int, char *, int, double,       \
                              char **, int, int, bool, int, cudaStream_t);                       \
  template int *approximateMedoidIndices<T>(T *, size_t, size_t, size_t *, char **, int, int,    \
                                            char *, double *, int *, cudaStream_t);              \
  template double DBAUpdate<T>(T *, size_t, T **, char **, size_t, size_t *, int, int, T *,      \
                               std::string, cudaStream_t);                                       \
  template void normalizeSequences<T>(T **, size_t, size_t *, int, double *, double *,           \
                                      cudaStream_t);                                            \
  template void adaptive_segmentation<T>(T **, size_t *, int, int, T ***, size_t **, int,        \
                                         cudaStream_t);
ODBA_INSTANTIATE(float)
ODBA_INSTANTIATE(double)

// ---------------------------------------------------------------------------
// C entry points over the façade (declared in opendba_b200.h).  Like the
// reference's host code they end the process with its exit codes on fatal
// errors (missing files, unwritable outputs, too few sequences).

extern "C" int odba_perform_dba_f32(float **sequences, int num_sequences, size_t *lengths,
                                    char **names, int use_open_start, int use_open_end,
                                    const char *output_prefix, int norm, double cdist,
                                    int algo_mode) {
  std::string pfx(output_prefix ? output_prefix : "");
  std::vector<char> buf(pfx.begin(), pfx.end());
  buf.push_back('\0');
  performDBA<float>(sequences, num_sequences, lengths, names, use_open_start, use_open_end,
                    buf.data(), norm, cdist, nullptr, 0, BINARY_READ_MODE, false, algo_mode);
  return ODBA_OK;
}

extern "C" int odba_perform_dba_f64(double **sequences, int num_sequences, size_t *lengths,
                                    char **names, int use_open_start, int use_open_end,
                                    const char *output_prefix, int norm, double cdist,
                                    int algo_mode) {
  std::string pfx(output_prefix ? output_prefix : "");
  std::vector<char> buf(pfx.begin(), pfx.end());
  buf.push_back('\0');
  performDBA<double>(sequences, num_sequences, lengths, names, use_open_start, use_open_end,
                     buf.data(), norm, cdist, nullptr, 0, BINARY_READ_MODE, false, algo_mode);
  return ODBA_OK;
}

extern "C" int odba_setup_and_run(int elem_size, const char *seqprefix_file, char **files,
                                  int num_files, const char *output_prefix, int read_mode,
                                  int use_open_start, int use_open_end,
                                  const char *min_segment_length, int norm, double cdist,
                                  int prefix_start, int prefix_length, int is_short) {
  std::vector<char> pfx(output_prefix, output_prefix + std::strlen(output_prefix) + 1);
  std::vector<char> ms(min_segment_length, min_segment_length + std::strlen(min_segment_length) + 1);
  std::vector<char> leader;
  if (seqprefix_file) leader.assign(seqprefix_file, seqprefix_file + std::strlen(seqprefix_file) + 1);
  char *lp = seqprefix_file ? leader.data() : nullptr;
  if (elem_size == 8)
    setupAndRun<double>(lp, files, num_files, pfx.data(), read_mode, use_open_start, use_open_end,
                        ms.data(), norm, cdist, prefix_start, prefix_length, is_short != 0);
  else
    setupAndRun<float>(lp, files, num_files, pfx.data(), read_mode, use_open_start, use_open_end,
                       ms.data(), norm, cdist, prefix_start, prefix_length, is_short != 0);
  return ODBA_OK;
}

namespace {
template <typename T>
int segment_host(const T *h_series, const uint64_t *h_lens, int n, int minseg, int prefix_skip,
                 T *h_out, uint64_t *h_out_lens) {
  std::vector<T *> ptrs(n);
  std::vector<size_t> lens(n);
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    ptrs[i] = const_cast<T *>(h_series + off);
    lens[i] = h_lens[i];
    off += h_lens[i];
  }
  T **segs = nullptr;
  size_t *seglens = nullptr;
  adaptive_segmentation<T>(ptrs.data(), lens.data(), n, minseg, &segs, &seglens, prefix_skip);
  size_t pos = 0;
  for (int i = 0; i < n; ++i) {
    std::memcpy(h_out + pos, segs[i], seglens[i] * sizeof(T));
    pos += seglens[i];
    h_out_lens[i] = seglens[i];
    cudaFree(segs[i]);
  }
  cudaFree(segs);
  cudaFree(seglens);
  return ODBA_OK;
}
}  // namespace

extern "C" int odba_segment_host_f32(const float *h_series, const uint64_t *h_lens, int n,
                                     int min_segment_length, int prefix_skip, float *h_out,
                                     uint64_t *h_out_lens) {
  if (n < 1 || !h_series || !h_lens || !h_out || !h_out_lens || min_segment_length < 1)
    return ODBA_ERR_INVALID_ARGUMENT;
  return segment_host<float>(h_series, h_lens, n, min_segment_length, prefix_skip, h_out, h_out_lens);
}

extern "C" int odba_segment_host_f64(const double *h_series, const uint64_t *h_lens, int n,
                                     int min_segment_length, int prefix_skip, double *h_out,
                                     uint64_t *h_out_lens) {
  if (n < 1 || !h_series || !h_lens || !h_out || !h_out_lens || min_segment_length < 1)
    return ODBA_ERR_INVALID_ARGUMENT;
  return segment_host<double>(h_series, h_lens, n, min_segment_length, prefix_skip, h_out, h_out_lens);
}

// ---------------------------------------------------------------------------
// Many independent DBA jobs (one cluster each, cdist 1, no files): every job is
// what performDBA computes for its series -- truncation, stable length sort,
// z-norm, medoid, rounds to delta 0 / flip-flop / 250 rounds, rescale -- but
// run either batched (all pairs of all jobs in one length-sorted launch; one
// DBA round for all unconverged jobs per CUDA graph replay) or plain (job by
// job through the single-job entry points, the drop-in path).

namespace {

template <typename T>
struct JobSet {
  int njobs = 0;
  std::vector<int> jbeg, jend, flags;         // series range per job in the sorted table
  std::vector<std::vector<int>> order;        // per job: sorted position -> input position
  DeviceSet<T> ds;                            // all jobs' series, sorted within each job
};

// Truncation and stable sort per job (dba.hpp:868-885), then upload.
template <typename T>
void build_jobs(const T *h_series, const uint64_t *h_lens, const int *job_begin, const int *job_end,
                const int *job_flags, int njobs, JobSet<T> &js, cudaStream_t st) {
  js.njobs = njobs;
  js.jbeg.assign(njobs, 0);
  js.jend.assign(njobs, 0);
  js.flags.assign(job_flags, job_flags + njobs);
  js.order.assign(njobs, {});
  std::vector<uint64_t> offs;
  uint64_t acc = 0;
  for (int j = 0; j < njobs; ++j) {
    (void)0;
  }
  // input offsets of every series
  int total = 0;
  for (int j = 0; j < njobs; ++j) total = std::max(total, job_end[j]);
  offs.assign(total, 0);
  for (int i = 0; i < total; ++i) {
    offs[i] = acc;
    acc += h_lens[i];
  }
  std::vector<T *> ptrs;
  std::vector<size_t> lens;
  for (int j = 0; j < njobs; ++j) {
    const int b = job_begin[j], e = job_end[j];
    std::vector<int> idx(e - b);
    std::vector<size_t> L(e - b);
    for (int i = b; i < e; ++i) {
      idx[i - b] = i - b;
      size_t len = h_lens[i];
      if (len && h_series[offs[i] + len - 1] >= std::sqrt(std::numeric_limits<T>::max())) --len;
      L[i - b] = len;
    }
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return L[a] < L[c]; });
    js.jbeg[j] = int(ptrs.size());
    for (int k : idx) {
      ptrs.push_back(const_cast<T *>(h_series + offs[b + k]));
      lens.push_back(L[k]);
    }
    js.jend[j] = int(ptrs.size());
    js.order[j] = idx;
  }
  js.ds.upload(ptrs.data(), lens.data(), int(ptrs.size()), st);
}

template <typename T>
bool flip_flop_or_done(double delta, int round, bool open, std::vector<T> &nb, std::vector<T> &prev,
                       std::vector<T> &two_prev) {
  if (delta == 0) return true;
  if (open) {
    if (round >= 1 && !std::memcmp(nb.data(), two_prev.data(), sizeof(T) * nb.size())) return true;
    if (round > 1) two_prev = prev;
    if (round > 0) prev = nb;
  }
  return false;
}

template <typename T>
int run_jobs(const T *h_series, const uint64_t *h_lens, const int *job_begin, const int *job_end,
             const int *job_flags, int njobs, int norm, int max_rounds, bool batched,
             int *h_medoids, uint64_t *h_centroid_offsets, T *h_centroids, int *h_rounds,
             double *h_deltas, cudaStream_t st) {
  JobSet<T> js;
  build_jobs<T>(h_series, h_lens, job_begin, job_end, job_flags, njobs, js, st);
  const int n = js.ds.n;
  DevBuf d_means(std::max(1, n) * sizeof(double)), d_sig(std::max(1, n) * sizeof(double));
  std::vector<double> means(n, 0.0), sigmas(n, 1.0);
  if (norm) {
    check(Ops<T>::znorm(ptr<T>(js.ds.data), ptr<uint64_t>(js.ds.offs), ptr<uint64_t>(js.ds.lens), n,
                        ptr<double>(d_means), ptr<double>(d_sig), st),
          "z-normalisation");
    check_cuda(cudaMemcpyAsync(means.data(), d_means.p, n * sizeof(double), cudaMemcpyDeviceToHost, st), "means");
    check_cuda(cudaMemcpyAsync(sigmas.data(), d_sig.p, n * sizeof(double), cudaMemcpyDeviceToHost, st), "sigmas");
  }
  // ---- medoids
  std::vector<unsigned long long> tri_off(njobs + 1, 0);
  for (int j = 0; j < njobs; ++j) {
    const unsigned long long m = (unsigned long long)(js.jend[j] - js.jbeg[j]);
    tri_off[j + 1] = tri_off[j] + m * (m - 1) / 2;
  }
  DevBuf d_dists(std::max<unsigned long long>(tri_off[njobs], 1) * sizeof(T));
  DevBuf d_sos(std::max(1, n) * sizeof(T)), d_med(std::max(1, njobs) * sizeof(int));
  DevBuf ws(odba_dtw_pairwise_workspace_bytes(sizeof(T), std::max<uint64_t>(js.ds.max_len, 1)));
  if (batched) {
    // one launch for every pair of every job, largest m*n first
    std::vector<odba_pair_task> tasks;
    tasks.reserve(tri_off[njobs]);
    std::vector<double> cost;
    cost.reserve(tri_off[njobs]);
    for (int j = 0; j < njobs; ++j) {
      const int b = js.jbeg[j], m = js.jend[j] - js.jbeg[j];
      const uint64_t fl = (uint64_t(js.flags[j] & 1) << 62) | (uint64_t((js.flags[j] >> 1) & 1) << 63);
      unsigned long long p = tri_off[j];
      for (int s = 0; s + 1 < m; ++s)
        for (int t = s + 1; t < m; ++t) {
          tasks.push_back(odba_pair_task{uint32_t(b + s), uint32_t(b + t), p | fl});
          cost.push_back(double(js.ds.h_lens[b + s]) * double(js.ds.h_lens[b + t]));
          ++p;
        }
    }
    std::vector<size_t> perm(tasks.size());
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<odba_pair_task> sorted(tasks.size());
    for (size_t i = 0; i < perm.size(); ++i) sorted[i] = tasks[perm[i]];
    DevBuf d_tasks(std::max<size_t>(sorted.size(), 1) * sizeof(odba_pair_task));
    check_cuda(cudaMemcpyAsync(d_tasks.p, sorted.data(), sorted.size() * sizeof(odba_pair_task),
                               cudaMemcpyHostToDevice, st), "task upload");
    if (!sorted.empty())
      check(sizeof(T) == 4
                ? odba_dtw_pairlist_f32((const float *)js.ds.data.p, ptr<uint64_t>(js.ds.offs),
                                        ptr<uint64_t>(js.ds.lens), ptr<odba_pair_task>(d_tasks),
                                        sorted.size(), js.ds.max_len, (float *)d_dists.p, ws.p,
                                        ws.bytes, st)
                : odba_dtw_pairlist_f64((const double *)js.ds.data.p, ptr<uint64_t>(js.ds.offs),
                                        ptr<uint64_t>(js.ds.lens), ptr<odba_pair_task>(d_tasks),
                                        sorted.size(), js.ds.max_len, (double *)d_dists.p, ws.p,
                                        ws.bytes, st),
            "pair-list DTW");
    check_cuda(cudaStreamSynchronize(st), "pair-list DTW");
    if (wait_ran_out(ws.p)) return ODBA_ERR_TIMEOUT;
  }
  for (int j = 0; j < njobs; ++j) {
    const int b = js.jbeg[j], m = js.jend[j] - js.jbeg[j];
    if (m < 1) continue;
    if (!batched && m >= 2)
      check(Ops<T>::pairwise(ptr<T>(js.ds.data), ptr<uint64_t>(js.ds.offs) + b,
                             ptr<uint64_t>(js.ds.lens) + b, m, js.ds.max_len, js.flags[j] & 1,
                             (js.flags[j] >> 1) & 1, ptr<T>(d_dists) + tri_off[j], ws.p, ws.bytes, st),
            "all-pairs DTW");
    check(sizeof(T) == 4
              ? odba_medoid_f32((const float *)d_dists.p + tri_off[j], ptr<uint64_t>(js.ds.lens) + b,
                                m, (float *)d_sos.p + b, ptr<int>(d_med) + j, st)
              : odba_medoid_f64((const double *)d_dists.p + tri_off[j], ptr<uint64_t>(js.ds.lens) + b,
                                m, (double *)d_sos.p + b, ptr<int>(d_med) + j, st),
          "medoid");
    if (!batched) {
      check_cuda(cudaStreamSynchronize(st), "medoid");
      if (m >= 2 && wait_ran_out(ws.p)) return ODBA_ERR_TIMEOUT;
    }
  }
  std::vector<int> med(njobs, 0);
  check_cuda(cudaMemcpyAsync(med.data(), d_med.p, njobs * sizeof(int), cudaMemcpyDeviceToHost, st), "medoid download");
  check_cuda(cudaStreamSynchronize(st), "medoids");
  // ---- rounds
  std::vector<uint64_t> coff(njobs, 0);
  std::vector<int> clen(njobs, 0);
  uint64_t ctot = 0;
  int max_clen = 1;
  for (int j = 0; j < njobs; ++j) {
    const int mi = js.jbeg[j] + med[j];
    coff[j] = ctot;
    clen[j] = int(js.ds.h_lens[mi]);
    ctot += clen[j];
    max_clen = std::max(max_clen, clen[j]);
    h_medoids[j] = js.order[j][med[j]];
    h_centroid_offsets[j] = coff[j];
  }
  DevBuf cbuf[2] = {DevBuf(std::max<uint64_t>(ctot, 1) * sizeof(T)), DevBuf(std::max<uint64_t>(ctot, 1) * sizeof(T))};
  DevBuf d_counts(std::max<uint64_t>(ctot, 1) * sizeof(uint32_t)), d_deltas(njobs * sizeof(double));
  for (int j = 0; j < njobs; ++j)
    check_cuda(cudaMemcpyAsync(ptr<T>(cbuf[0]) + coff[j], ptr<T>(js.ds.data) + js.ds.h_offs[js.jbeg[j] + med[j]],
                               clen[j] * sizeof(T), cudaMemcpyDeviceToDevice, st), "seed centroids");
  std::vector<T> host_c(ctot);
  check_cuda(cudaMemcpyAsync(host_c.data(), cbuf[0].p, ctot * sizeof(T), cudaMemcpyDeviceToHost, st), "seed download");
  check_cuda(cudaStreamSynchronize(st), "seeds");
  std::vector<int> active(njobs, 0), rounds(njobs, 0);
  std::vector<double> deltas(njobs, 0.0);
  std::vector<std::vector<T>> prev(njobs), two_prev(njobs);
  int live = 0;
  for (int j = 0; j < njobs; ++j) {
    if (js.jend[j] - js.jbeg[j] > 1) {
      active[j] = 1;
      ++live;
      prev[j].assign(clen[j], T(0));
      two_prev[j].assign(clen[j], T(0));
    }
  }
  // member tables: member k of job j is series jbeg[j] + k, in sorted order
  std::vector<int> mseries(n), mjob(n), mbeg(njobs), mend(njobs), h_flags(njobs);
  std::vector<uint64_t> h_mlens(n), h_clen(njobs);
  for (int j = 0; j < njobs; ++j) {
    mbeg[j] = js.jbeg[j];
    mend[j] = js.jend[j];
    h_clen[j] = uint64_t(clen[j]);
    for (int k = js.jbeg[j]; k < js.jend[j]; ++k) {
      mseries[k] = k;
      mjob[k] = j;
      h_mlens[k] = js.ds.h_lens[k];
    }
  }
  std::vector<int> morder(n);
  std::iota(morder.begin(), morder.end(), 0);
  std::stable_sort(morder.begin(), morder.end(), [&](int a, int b) {
    return double(h_mlens[a]) * h_clen[mjob[a]] > double(h_mlens[b]) * h_clen[mjob[b]];
  });
  auto flags_now = [&]() {
    for (int j = 0; j < njobs; ++j) h_flags[j] = (js.flags[j] & 3) | (active[j] ? 4 : 0);
  };
  flags_now();
  DevBuf d_mseries(n * sizeof(int)), d_mjob(n * sizeof(int)), d_mbeg(njobs * sizeof(int)),
      d_mend(njobs * sizeof(int)), d_flags(njobs * sizeof(int)), d_clen(njobs * sizeof(int)),
      d_coff(njobs * sizeof(uint64_t)), d_order(n * sizeof(int));
  check_cuda(cudaMemcpyAsync(d_mseries.p, mseries.data(), n * sizeof(int), cudaMemcpyHostToDevice, st), "members");
  check_cuda(cudaMemcpyAsync(d_mjob.p, mjob.data(), n * sizeof(int), cudaMemcpyHostToDevice, st), "members");
  check_cuda(cudaMemcpyAsync(d_mbeg.p, mbeg.data(), njobs * sizeof(int), cudaMemcpyHostToDevice, st), "jobs");
  check_cuda(cudaMemcpyAsync(d_mend.p, mend.data(), njobs * sizeof(int), cudaMemcpyHostToDevice, st), "jobs");
  check_cuda(cudaMemcpyAsync(d_clen.p, clen.data(), njobs * sizeof(int), cudaMemcpyHostToDevice, st), "jobs");
  check_cuda(cudaMemcpyAsync(d_coff.p, coff.data(), njobs * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "jobs");
  check_cuda(cudaMemcpyAsync(d_order.p, morder.data(), n * sizeof(int), cudaMemcpyHostToDevice, st), "members");
  check_cuda(cudaMemcpyAsync(d_flags.p, h_flags.data(), njobs * sizeof(int), cudaMemcpyHostToDevice, st), "flags");
  std::vector<T> nb(ctot);
  if (batched && live) {
    // Waves: jobs in order, as many per wave as the round workspace budget
    // allows (only a wave's jobs are active and take path space); each wave
    // runs its rounds to convergence from two captured graphs.
    auto ws_for = [&](const std::vector<int> &fl) {
      return odba_dba_batch_workspace_bytes(sizeof(T), h_mlens.data(), mjob.data(), n, h_clen.data(),
                                            fl.data(), njobs);
    };
    size_t budget = 0;
    if (const char *e = std::getenv("ODBA_ROUND_BUDGET_BYTES")) budget = std::strtoull(e, nullptr, 10);
    if (!budget) {
      size_t fr = 0, tot = 0;
      check_cuda(cudaMemGetInfo(&fr, &tot), "device memory query");
      budget = fr / 10 * 7;
    }
    std::vector<int> none(njobs);
    for (int j = 0; j < njobs; ++j) none[j] = js.flags[j] & 3;
    const size_t fixed = ws_for(none);
    std::vector<std::vector<int>> waves;
    {
      std::vector<int> cur_wave, fl = none;
      size_t used = fixed;
      for (int j = 0; j < njobs; ++j) {
        if (!active[j]) continue;
        fl[j] = none[j] | 4;
        const size_t cost = ws_for(fl) - fixed;
        fl[j] = none[j];
        if (!cur_wave.empty() && used + cost > budget) {
          waves.push_back(cur_wave);
          cur_wave.clear();
          used = fixed;
        }
        cur_wave.push_back(j);
        used += cost;
      }
      if (!cur_wave.empty()) waves.push_back(cur_wave);
    }
    size_t ws_max = fixed;
    for (auto &w : waves) {
      std::vector<int> fl = none;
      for (int j : w) fl[j] |= 4;
      ws_max = std::max(ws_max, ws_for(fl));
    }
    DevBuf rws(ws_max);
    const std::vector<int> was_active = active;
    for (auto &wave : waves) {
      std::vector<int> size_flags = none;
      for (int j = 0; j < njobs; ++j) active[j] = 0;
      live = 0;
      for (int j : wave) {
        size_flags[j] |= 4;
        active[j] = was_active[j];
        live += active[j];
      }
      flags_now();
      cudaGraphExec_t exec[2] = {nullptr, nullptr};
      for (int g = 0; g < 2; ++g) {
        cudaGraph_t graph;
        check_cuda(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
        const T *cin = ptr<T>(cbuf[g]);
        T *cout = ptr<T>(cbuf[1 - g]);
        const int rc = sizeof(T) == 4
            ? odba_dba_batch_round_f32((const float *)cin, ptr<uint64_t>(d_coff), ptr<int>(d_clen), ptr<int>(d_flags),
                                       ptr<int>(d_mbeg), ptr<int>(d_mend), njobs, max_clen,
                                       (const float *)js.ds.data.p, ptr<uint64_t>(js.ds.offs), ptr<uint64_t>(js.ds.lens),
                                       ptr<int>(d_mseries), ptr<int>(d_mjob), ptr<int>(d_order), n, h_mlens.data(),
                                       mjob.data(), h_clen.data(), size_flags.data(), (float *)cout,
                                       ptr<uint32_t>(d_counts), ptr<double>(d_deltas), nullptr, nullptr, rws.p,
                                       rws.bytes, st)
            : odba_dba_batch_round_f64((const double *)cin, ptr<uint64_t>(d_coff), ptr<int>(d_clen), ptr<int>(d_flags),
                                       ptr<int>(d_mbeg), ptr<int>(d_mend), njobs, max_clen,
                                       (const double *)js.ds.data.p, ptr<uint64_t>(js.ds.offs), ptr<uint64_t>(js.ds.lens),
                                       ptr<int>(d_mseries), ptr<int>(d_mjob), ptr<int>(d_order), n, h_mlens.data(),
                                       mjob.data(), h_clen.data(), size_flags.data(), (double *)cout,
                                       ptr<uint32_t>(d_counts), ptr<double>(d_deltas), nullptr, nullptr, rws.p,
                                       rws.bytes, st);
        check_cuda(cudaStreamEndCapture(st, &graph), "graph capture");
        check(rc, "batched DBA round (capture)");
        check_cuda(cudaGraphInstantiate(&exec[g], graph, 0), "graph instantiate");
        cudaGraphDestroy(graph);
      }
      int cur = 0;
      for (int round = 0; round < max_rounds && live; ++round) {
        check_cuda(cudaMemcpyAsync(d_flags.p, h_flags.data(), njobs * sizeof(int), cudaMemcpyHostToDevice, st), "flags");
        check_cuda(cudaGraphLaunch(exec[cur], st), "graph launch");
        check_cuda(cudaMemcpyAsync(nb.data(), cbuf[1 - cur].p, ctot * sizeof(T), cudaMemcpyDeviceToHost, st), "means");
        check_cuda(cudaMemcpyAsync(deltas.data(), d_deltas.p, njobs * sizeof(double), cudaMemcpyDeviceToHost, st), "deltas");
        check_cuda(cudaStreamSynchronize(st), "batched round");
        if (wait_ran_out(rws.p)) {
          for (int g = 0; g < 2; ++g) cudaGraphExecDestroy(exec[g]);
          return ODBA_ERR_TIMEOUT;
        }
        for (int j = 0; j < njobs; ++j) {
          if (!active[j]) continue;
          rounds[j] = round + 1;
          std::vector<T> v(nb.begin() + coff[j], nb.begin() + coff[j] + clen[j]);
          const bool open = (js.flags[j] & 3) != 0;
          std::copy(v.begin(), v.end(), host_c.begin() + coff[j]);
          h_deltas[j] = deltas[j];
          if (flip_flop_or_done<T>(deltas[j], round, open, v, prev[j], two_prev[j])) {
            active[j] = 0;
            --live;
          }
        }
        flags_now();
        // the next round reads the means just written (the other buffer)
        cur = 1 - cur;
      }
      for (int g = 0; g < 2; ++g) cudaGraphExecDestroy(exec[g]);
    }
  } else if (live) {
    // plain: job by job, one round per call, synchronizing every round (performDBA's loop)
    for (int j = 0; j < njobs; ++j) {
      if (!active[j]) continue;
      const int b = js.jbeg[j], m = js.jend[j] - js.jbeg[j];
      const int os = js.flags[j] & 1, oe = (js.flags[j] >> 1) & 1;
      DevBuf rws(odba_dba_round_workspace_bytes(sizeof(T), js.ds.h_lens.data() + b, m, clen[j], os, oe));
      T *cin = ptr<T>(cbuf[0]) + coff[j];
      T *cout = ptr<T>(cbuf[1]) + coff[j];
      std::vector<T> v(clen[j]);
      for (int round = 0; round < max_rounds; ++round) {
        check(Ops<T>::round(cin, clen[j], ptr<T>(js.ds.data), ptr<uint64_t>(js.ds.offs) + b,
                            ptr<uint64_t>(js.ds.lens) + b, js.ds.h_lens.data() + b, m, os, oe, cout,
                            ptr<uint32_t>(d_counts) + coff[j], ptr<double>(d_deltas) + j, nullptr, nullptr,
                            rws.p, rws.bytes, st),
              "DBA round");
        double delta = 0;
        check_cuda(cudaMemcpyAsync(v.data(), cout, clen[j] * sizeof(T), cudaMemcpyDeviceToHost, st), "means");
        check_cuda(cudaMemcpyAsync(&delta, ptr<double>(d_deltas) + j, sizeof(double), cudaMemcpyDeviceToHost, st), "delta");
        check_cuda(cudaStreamSynchronize(st), "DBA round");
        if (wait_ran_out(rws.p)) return ODBA_ERR_TIMEOUT;
        rounds[j] = round + 1;
        h_deltas[j] = delta;
        std::copy(v.begin(), v.end(), host_c.begin() + coff[j]);
        if (flip_flop_or_done<T>(delta, round, (js.flags[j] & 3) != 0, v, prev[j], two_prev[j])) break;
        check_cuda(cudaMemcpyAsync(cin, cout, clen[j] * sizeof(T), cudaMemcpyDeviceToDevice, st), "centroid update");
      }
    }
  }
  // rescale by the medoid's mean and sigma (dba.hpp:1117-1125) and return
  for (int j = 0; j < njobs; ++j) {
    const int mi = js.jbeg[j] + med[j];
    h_rounds[j] = rounds[j];
    for (int i = 0; i < clen[j]; ++i) {
      T v = host_c[coff[j] + i];
      if (norm) v = (T)(means[mi] + v * sigmas[mi]);
      h_centroids[coff[j] + i] = v;
    }
  }
  return ODBA_OK;
}

}  // namespace

#define ODBA_JOBS_ENTRY(SFX, T)                                                                  \
  extern "C" int odba_dba_jobs_##SFX(const T *h_series, const uint64_t *h_lens,                 \
                                     const int *job_begin, const int *job_end,                  \
                                     const int *job_flags, int njobs, int norm, int max_rounds,   \
                                     int batched, int *h_medoids, uint64_t *h_centroid_offsets,   \
                                     T *h_centroids, int *h_rounds, double *h_deltas,            \
                                     void *stream) {                                              \
    if (njobs < 1 || !h_series || !h_lens || !job_begin || !job_end || !job_flags ||             \
        !h_medoids || !h_centroid_offsets || !h_centroids || !h_rounds || !h_deltas)             \
      return ODBA_ERR_INVALID_ARGUMENT;                                                          \
    for (int j = 0; j < njobs; ++j)                                                              \
      if (job_end[j] <= job_begin[j] || (j && job_begin[j] != job_end[j - 1]) ||                 \
          (j == 0 && job_begin[0] != 0))                                                         \
        return ODBA_ERR_INVALID_ARGUMENT;                                                        \
    /* graphs cannot be captured on the legacy default stream: run on a private      */    \
    /* stream ordered after the caller's                                              */    \
    cudaStream_t caller = static_cast<cudaStream_t>(stream), own = nullptr;                      \
    cudaEvent_t ready = nullptr;                                                                 \
    check_cuda(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking), "job stream");            \
    check_cuda(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "job event");           \
    check_cuda(cudaEventRecord(ready, caller), "job event");                                     \
    check_cuda(cudaStreamWaitEvent(own, ready, 0), "job event");                                 \
    const int rc = run_jobs<T>(h_series, h_lens, job_begin, job_end, job_flags, njobs, norm,     \
                               max_rounds > 0 ? max_rounds : 250, batched != 0, h_medoids,       \
                               h_centroid_offsets, h_centroids, h_rounds, h_deltas, own);        \
    check_cuda(cudaStreamSynchronize(own), "job stream");                                        \
    cudaEventDestroy(ready);                                                                     \
    cudaStreamDestroy(own);                                                                      \
    return rc;                                                                                   \
  }
ODBA_JOBS_ENTRY(f32, float)
ODBA_JOBS_ENTRY(f64, double)
#undef ODBA_JOBS_ENTRY
