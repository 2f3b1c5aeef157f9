// Test-infrastructure harness, NOT product code.
//
// Compiles the reference's own header-only CUDA implementation (from the
// reference tree, via -I, never copied) for sm_100a and runs its entry points
// on seeded inputs so that its GPU results can be captured as golden fixtures.
// Build recipe: oracle/Makefile (outputs only under oracle/_ref/).  Driver:
// tests/golden/make_reference_golden.py.
//
// Modes (inputs and outputs are series bundles, see oracle/series_bundle.h):
//   pairwise   <in.odbs> <out.odbs> <open_start> <open_end> [max_rows]
//       The all-vs-all distance launches of approximateMedoidIndices
//       (dba.hpp:67-161): one DTWDistance launch per 1024-column swath per
//       row, each followed by the boundary copy, on one device.  Writes the
//       upper-triangle distances (dtw.hpp:242-257) as one series and prints
//       the cells and the device time.
//   medoid     <in.odbs> <out_prefix> <open_start> <open_end>
//       approximateMedoidIndices itself (cdist = 1): writes
//       <out_prefix>.pair_dists.txt and <out_prefix>.medoid.txt.
//   dbaupdate  <members.odbs> <centroid.odbs> <out_prefix> <open_start> <open_end>
//       One DBAUpdate round (dba.hpp:432-848): writes <out_prefix>.mean.odbs
//       (the updated centroid), <out_prefix>.delta.txt and the per-member
//       path files <out_prefix>.path<k>.txt.  With the environment variable
//       ODBA_HARNESS_FORCE_STRIPE set, the round runs in the reference's stripe
//       mode (dba.hpp:515-763).
//   znorm      <in.odbs> <out_prefix>
//       normalizeSequences (gpu_utils.hpp:132-170): writes the normalised
//       series, and the per-series means and sigmas (float64).
//   performdba <in.odbs> <out_prefix> <open_start> <open_end> <norm> [cdist]
//       performDBA (dba.hpp:863-1189), CLUSTER_AND_CONSENSUS, cdist default 1.
//   setupandrun <out_prefix> <open_start> <open_end> <norm> <file>...
//       setupAndRun<float> on text files, as tests/openDBA_test.cu does; with
//       ODBA_HARNESS_SEQPREFIX=<leader text file> it chops that prefix first.
//   segment    <in.odbs> <out.odbs> <min_segment_length> <prefix_skip>
//       adaptive_segmentation (segmentation.hpp:340-583).
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

// Forced stripe mode (dbaupdate with ODBA_HARNESS_FORCE_STRIPE set): DBAUpdate
// takes its stripe path when the free device memory it reads is below the full
// path matrix's size (dba.hpp:523-525), so the harness reports no free memory
// to the reference's code while the flag is on.
static bool g_force_stripe = false;
static cudaError_t harness_mem_get_info(size_t *free_bytes, size_t *total_bytes) {
  const cudaError_t e = cudaMemGetInfo(free_bytes, total_bytes);
  if (g_force_stripe && free_bytes) *free_bytes = 0;
  return e;
}
#define cudaMemGetInfo harness_mem_get_info

#include "openDBA.cuh"
#include "series_bundle.h"

static void die(const char *msg) {
  std::fprintf(stderr, "ref_harness: %s\n", msg);
  std::exit(2);
}

template <typename T>
static T **managed_series(const SeriesBundle &b, size_t **lens_out) {
  T **seqs = nullptr;
  cudaMallocManaged(&seqs, sizeof(T *) * b.n());
  CUERR("harness: managed series pointers");
  size_t *lens = nullptr;
  cudaMallocManaged(&lens, sizeof(size_t) * b.n());
  CUERR("harness: managed lengths");
  for (size_t i = 0; i < b.n(); ++i) {
    lens[i] = b.lens[i];
    cudaMallocManaged(&seqs[i], sizeof(T) * (b.lens[i] ? b.lens[i] : 1));
    CUERR("harness: managed series");
    std::memcpy(seqs[i], b.series<T>(i), sizeof(T) * b.lens[i]);
  }
  *lens_out = lens;
  return seqs;
}

static char **make_names(size_t n) {
  char **names = nullptr;
  cudaMallocHost(&names, sizeof(char *) * n);
  for (size_t i = 0; i < n; ++i) {
    std::string s = "s" + std::to_string(i);
    cudaMallocHost(&names[i], s.size() + 1);
    std::memcpy(names[i], s.c_str(), s.size() + 1);
  }
  return names;
}

// The launch loop of approximateMedoidIndices on one device, capturing the
// distance triangle in binary instead of the 6-significant-digit text file.
template <typename T>
static int run_pairwise(const SeriesBundle &b, const std::string &out, int os, int oe, size_t max_rows) {
  size_t n = b.n();
  size_t maxLen = 0;
  for (auto l : b.lens) maxLen = l > maxLen ? l : maxLen;
  T *gpu_sequences = nullptr;
  cudaMallocManaged(&gpu_sequences, sizeof(T) * n * maxLen);
  CUERR("harness: padded sequences");
  std::memset(gpu_sequences, 0, sizeof(T) * n * maxLen);
  size_t *lens = nullptr;
  cudaMallocManaged(&lens, sizeof(size_t) * n);
  for (size_t i = 0; i < n; ++i) {
    lens[i] = b.lens[i];
    std::memcpy(gpu_sequences + i * maxLen, b.series<T>(i), sizeof(T) * b.lens[i]);
  }
  size_t npairs = n * (n - 1) / 2;
  T *dists = nullptr;
  cudaMalloc(&dists, sizeof(T) * npairs);
  cudaMemset(dists, 0, sizeof(T) * npairs);
  CUERR("harness: distance buffer");
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, 0);
  dim3 block(prop.maxThreadsPerBlock, 1, 1);
  size_t rows = n - 1;
  if (max_rows && max_rows < rows) rows = max_rows;
  double cells = 0;
  for (size_t s = 0; s < rows; ++s)
    for (size_t j = s + 1; j < n; ++j) cells += double(b.lens[s]) * double(b.lens[j]);
  // Timed by the host clock between two device synchronisations: the launches
  // go to non-blocking streams, which an event on the legacy stream does not
  // wait for.  Boundary buffers are released every kDrainRows rows (the
  // reference frees them in stream callbacks, dba.hpp:157-160) so the whole
  // triangle of a large set never holds them all at once.
  constexpr size_t kDrainRows = 256;
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<T *> bufs;
  std::vector<cudaStream_t> streams;
  auto drain = [&]() {
    cudaDeviceSynchronize();
    CUERR("harness: pairwise sync");
    for (auto p : bufs) cudaFree(p);
    for (auto st : streams) cudaStreamDestroy(st);
    bufs.clear();
    streams.clear();
  };
  for (size_t s = 0; s < rows; ++s) {
    dim3 grid(n - s - 1, 1, 1);
    size_t bytes = sizeof(T) * lens[s] * grid.x;
    T *cost = nullptr, *newcost = nullptr;
    cudaMallocManaged(&cost, bytes);
    cudaMallocManaged(&newcost, bytes);
    CUERR("harness: boundary buffers");
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (size_t off = 0; off < maxLen; off += block.x) {
      DTWDistance<T><<<grid, block, block.x * 3 * sizeof(T), st>>>(
          (T *)0, (size_t)0, (T *)0, (size_t)0, s, off, gpu_sequences, maxLen, n, lens, cost,
          newcost, (unsigned char *)0, (size_t)0, dists, os, oe);
      CUERR("harness: DTWDistance launch");
      cudaMemcpyAsync(cost, newcost, bytes, cudaMemcpyDeviceToDevice, st);
    }
    bufs.push_back(cost);
    bufs.push_back(newcost);
    streams.push_back(st);
    if ((s + 1) % kDrainRows == 0) drain();
  }
  drain();
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::vector<T> host(npairs);
  cudaMemcpy(host.data(), dists, sizeof(T) * npairs, cudaMemcpyDeviceToHost);
  CUERR("harness: distance copy");
  std::vector<uint64_t> lensv{npairs};
  write_bundle(out, sizeof(T), lensv, host.data());
  std::printf("{\"cells\": %.0f, \"ms\": %.3f, \"gcups\": %.3f, \"rows\": %zu}\n", cells, ms,
              cells / (ms * 1e-3) / 1e9, rows);
  return 0;
}

template <typename T>
static int run_medoid(const SeriesBundle &b, const std::string &prefix, int os, int oe) {
  size_t n = b.n();
  size_t maxLen = 0;
  for (auto l : b.lens) maxLen = l > maxLen ? l : maxLen;
  T *gpu_sequences = nullptr;
  cudaMallocManaged(&gpu_sequences, sizeof(T) * n * maxLen);
  std::memset(gpu_sequences, 0, sizeof(T) * n * maxLen);
  size_t *lens = nullptr;
  cudaMallocManaged(&lens, sizeof(size_t) * n);
  for (size_t i = 0; i < n; ++i) {
    lens[i] = b.lens[i];
    std::memcpy(gpu_sequences + i * maxLen, b.series<T>(i), sizeof(T) * b.lens[i]);
  }
  char **names = make_names(n);
  std::vector<int> memberships(n, 0);
  double cdist = 1.0;
  std::vector<char> pfx(prefix.begin(), prefix.end());
  pfx.push_back('\0');
  int *medoids = approximateMedoidIndices<T>(gpu_sequences, maxLen, n, lens, names, os, oe, pfx.data(),
                                             &cdist, memberships.data(), 0);
  std::ofstream(prefix + ".medoid.txt") << medoids[0] << "\n";
  return 0;
}

template <typename T>
static int run_dbaupdate(const SeriesBundle &members, const SeriesBundle &centroid,
                         const std::string &prefix, int os, int oe) {
  size_t *lens = nullptr;
  T **seqs = managed_series<T>(members, &lens);
  char **names = make_names(members.n());
  size_t Lc = centroid.lens[0];
  T *C = nullptr;
  cudaMallocManaged(&C, sizeof(T) * Lc);
  std::memcpy(C, centroid.series<T>(0), sizeof(T) * Lc);
  T *mean = nullptr;
  cudaMallocHost(&mean, sizeof(T) * Lc);
  double delta = DBAUpdate<T>(C, Lc, seqs, names, members.n(), lens, os, oe, mean, prefix, 0);
  std::vector<uint64_t> l1{Lc};
  write_bundle(prefix + ".mean.odbs", sizeof(T), l1, mean);
  FILE *f = std::fopen((prefix + ".delta.txt").c_str(), "w");
  std::fprintf(f, "%.17g\n", delta);
  std::fclose(f);
  return 0;
}

template <typename T>
static int run_znorm(const SeriesBundle &b, const std::string &prefix) {
  size_t *lens = nullptr;
  T **seqs = managed_series<T>(b, &lens);
  double *means = nullptr, *sigmas = nullptr;
  cudaMallocManaged(&means, sizeof(double) * b.n());
  cudaMallocManaged(&sigmas, sizeof(double) * b.n());
  normalizeSequences<T>(seqs, b.n(), lens, -1, means, sigmas, 0);
  cudaDeviceSynchronize();
  CUERR("harness: znorm sync");
  std::vector<unsigned char> flat;
  for (size_t i = 0; i < b.n(); ++i) {
    const unsigned char *p = reinterpret_cast<const unsigned char *>(seqs[i]);
    flat.insert(flat.end(), p, p + sizeof(T) * b.lens[i]);
  }
  write_bundle(prefix + ".norm.odbs", sizeof(T), b.lens, flat.data());
  std::vector<uint64_t> ln{b.n()};
  write_bundle(prefix + ".means.odbs", 8, ln, means);
  write_bundle(prefix + ".sigmas.odbs", 8, ln, sigmas);
  return 0;
}

template <typename T>
static int run_performdba(const SeriesBundle &b, const std::string &prefix, int os, int oe, int norm,
                          double cdist) {
  size_t *lens = nullptr;
  T **seqs = managed_series<T>(b, &lens);
  char **names = make_names(b.n());
  std::vector<char> pfx(prefix.begin(), prefix.end());
  pfx.push_back('\0');
  char *files[1] = {pfx.data()};
  performDBA<T>(seqs, (int)b.n(), lens, names, os, oe, pfx.data(), norm, cdist, files, 1,
                BINARY_READ_MODE, false, CLUSTER_AND_CONSENSUS);
  cudaDeviceSynchronize();
  CUERR("harness: performDBA sync");
  return 0;
}

template <typename T>
static int run_segment(const SeriesBundle &b, const std::string &out, int minseg, int skip) {
  size_t *lens = nullptr;
  T **seqs = managed_series<T>(b, &lens);
  T **segs = nullptr;
  size_t *seglens = nullptr;
  adaptive_segmentation<T>(seqs, lens, (int)b.n(), minseg, &segs, &seglens, skip);
  cudaDeviceSynchronize();
  CUERR("harness: segmentation sync");
  std::vector<uint64_t> l;
  std::vector<unsigned char> flat;
  for (size_t i = 0; i < b.n(); ++i) {
    l.push_back(seglens[i]);
    const unsigned char *p = reinterpret_cast<const unsigned char *>(segs[i]);
    flat.insert(flat.end(), p, p + sizeof(T) * seglens[i]);
  }
  write_bundle(out, sizeof(T), l, flat.data());
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 3) die("usage: ref_harness <mode> args...");
  std::string mode = argv[1];
  g_force_stripe = mode == "dbaupdate" && std::getenv("ODBA_HARNESS_FORCE_STRIPE") != nullptr;
  int rc = 0;
  if (mode == "setupandrun") {
    if (argc < 7) die("setupandrun <prefix> <os> <oe> <norm> <files...>");
    std::vector<char> pfx(argv[2], argv[2] + std::strlen(argv[2]) + 1);
    int nfiles = argc - 6;
    char **files = nullptr;
    cudaMallocHost(&files, sizeof(char *) * nfiles);
    for (int i = 0; i < nfiles; ++i) {
      size_t len = std::strlen(argv[6 + i]) + 1;
      cudaMallocHost(&files[i], len);
      std::memcpy(files[i], argv[6 + i], len);
    }
    char minseg[8] = "0";
    // a leader (prefix) file for the prefix chop, if given in the environment
    std::vector<char> leader;
    if (const char *lp = std::getenv("ODBA_HARNESS_SEQPREFIX"))
      leader.assign(lp, lp + std::strlen(lp) + 1);
    setupAndRun<float>(leader.empty() ? nullptr : leader.data(), files, nfiles, pfx.data(),
                       TEXT_READ_MODE, std::atoi(argv[3]), std::atoi(argv[4]), minseg,
                       std::atoi(argv[5]), 1.0);
  } else {
    SeriesBundle b = read_bundle(argv[2]);
    bool dbl = b.elem_size == 8;
    if (mode == "pairwise") {
      if (argc < 6) die("pairwise <in> <out> <os> <oe> [max_rows]");
      size_t max_rows = argc > 6 ? std::strtoull(argv[6], nullptr, 10) : 0;
      rc = dbl ? run_pairwise<double>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]), max_rows)
               : run_pairwise<float>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]), max_rows);
    } else if (mode == "medoid") {
      if (argc < 6) die("medoid <in> <prefix> <os> <oe>");
      rc = dbl ? run_medoid<double>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]))
               : run_medoid<float>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]));
    } else if (mode == "dbaupdate") {
      if (argc < 7) die("dbaupdate <members> <centroid> <prefix> <os> <oe>");
      SeriesBundle c = read_bundle(argv[3]);
      rc = dbl ? run_dbaupdate<double>(b, c, argv[4], std::atoi(argv[5]), std::atoi(argv[6]))
               : run_dbaupdate<float>(b, c, argv[4], std::atoi(argv[5]), std::atoi(argv[6]));
    } else if (mode == "znorm") {
      rc = dbl ? run_znorm<double>(b, argv[3]) : run_znorm<float>(b, argv[3]);
    } else if (mode == "performdba") {
      if (argc < 7) die("performdba <in> <prefix> <os> <oe> <norm> [cdist]");
      const double cdist = argc > 7 ? std::atof(argv[7]) : 1.0;
      rc = dbl ? run_performdba<double>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]), std::atoi(argv[6]), cdist)
               : run_performdba<float>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]), std::atoi(argv[6]), cdist);
    } else if (mode == "segment") {
      if (argc < 6) die("segment <in> <out> <minseg> <skip>");
      rc = dbl ? run_segment<double>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]))
               : run_segment<float>(b, argv[3], std::atoi(argv[4]), std::atoi(argv[5]));
    } else {
      die("unknown mode");
    }
  }
  cudaDeviceSynchronize();
  CUERR("harness: final sync");
  return rc;
}
