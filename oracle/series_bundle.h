// Test-infrastructure helper, NOT product code.
//
// A "series bundle" is the on-disk container the test fixtures use to carry a
// ragged set of numeric series (and the outputs computed from them) between
// the generator, the reference harness, the CPU oracle and the tests:
//
//   bytes 0..3   magic "ODBS"
//   u32          element size in bytes (4 = float32, 8 = float64)
//   u64          number of series n
//   u64[n]       series lengths
//   T[sum(len)]  the series, concatenated, little endian
//
// The Python side (opendba_b200/bundle.py) reads and writes the same layout.
#ifndef ODBA_SERIES_BUNDLE_H
#define ODBA_SERIES_BUNDLE_H

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

struct SeriesBundle {
  uint32_t elem_size = 4;
  std::vector<uint64_t> lens;
  std::vector<unsigned char> data;  // concatenated raw values

  size_t n() const { return lens.size(); }
  size_t total() const {
    size_t t = 0;
    for (uint64_t l : lens) t += l;
    return t;
  }
  template <typename T>
  const T *series(size_t i) const {
    size_t off = 0;
    for (size_t k = 0; k < i; ++k) off += lens[k];
    return reinterpret_cast<const T *>(data.data()) + off;
  }
};

inline SeriesBundle read_bundle(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open bundle " + path);
  char magic[4];
  SeriesBundle b;
  uint64_t n = 0;
  if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "ODBS", 4) != 0 ||
      std::fread(&b.elem_size, 4, 1, f) != 1 || std::fread(&n, 8, 1, f) != 1) {
    std::fclose(f);
    throw std::runtime_error("bad bundle header " + path);
  }
  b.lens.resize(n);
  if (n && std::fread(b.lens.data(), 8, n, f) != n) {
    std::fclose(f);
    throw std::runtime_error("truncated bundle lengths " + path);
  }
  b.data.resize(b.total() * b.elem_size);
  if (!b.data.empty() && std::fread(b.data.data(), 1, b.data.size(), f) != b.data.size()) {
    std::fclose(f);
    throw std::runtime_error("truncated bundle data " + path);
  }
  std::fclose(f);
  return b;
}

inline void write_bundle(const std::string &path, uint32_t elem_size,
                         const std::vector<uint64_t> &lens, const void *data) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write bundle " + path);
  uint64_t n = lens.size(), total = 0;
  for (uint64_t l : lens) total += l;
  std::fwrite("ODBS", 1, 4, f);
  std::fwrite(&elem_size, 4, 1, f);
  std::fwrite(&n, 8, 1, f);
  if (n) std::fwrite(lens.data(), 8, n, f);
  if (total) std::fwrite(data, elem_size, total, f);
  std::fclose(f);
}

#endif
