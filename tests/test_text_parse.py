"""The text reader's fast line parser (opendba_b200/csrc/text_parse.h) against
the extraction it stands in for, std::stringstream(line) >> value, which is
how the reference reads text inputs (cpu_utils.hpp:92-134): every value bit
for bit, float and double, on edge cases and on random values printed in
many formats.  CPU only: a small C++ driver is compiled with g++."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DRIVER = r'''
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include "text_parse.h"

template <typename T> static bool same(T a, T b) { return std::memcmp(&a, &b, sizeof(T)) == 0; }

int main(int argc, char **argv) {
  std::ifstream f(argv[1], std::ios::binary);
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  size_t bad = 0, n = 0, pos = 0;
  while (true) {
    const size_t nl = text.find('\n', pos);
    if (nl == std::string::npos) break;
    const std::string line = text.substr(pos, nl - pos);
    {
      std::stringstream in(line);
      float want = 0.0f;
      in >> want;
      const float got = odba::parse_line_value<float>(line.data(), line.data() + line.size());
      if (!same(got, want)) { ++bad; std::printf("float [%s] %.9g %.9g\n", line.c_str(), got, want); }
    }
    {
      std::stringstream in(line);
      double want = 0.0;
      in >> want;
      const double got = odba::parse_line_value<double>(line.data(), line.data() + line.size());
      if (!same(got, want)) { ++bad; std::printf("double [%s] %.17g %.17g\n", line.c_str(), got, want); }
    }
    ++n;
    pos = nl + 1;
  }
  std::printf("%zu lines, %zu mismatches\n", n, bad);
  return bad ? 1 : 0;
}
'''

EDGE = ["", " ", "\t", "0", "-0", "+0", "1", "-1", "+1.5", "1.", ".5", "-.5", "+.5e-3", ".", "-",
        "+", "e5", "1e", "1e+", "1e-", "1E5", "1e5x", "1.5.3", "1,5", "12abc", "0x10", "0x1p3",
        "inf", "-inf", "Infinity", "nan", "NaN", "nan(1)", "1e40", "-1e40", "1e-40", "1e-50",
        "1e309", "1e-320", "3.4028235e38", "3.4028236e38", "1.17549435e-38", "  42  ", "42\r",
        " \t-7.25e2 trailing", "1e5e3", "00012.500", "9" * 40, "0." + "0" * 60 + "1",
        "1" + "0" * 130, "-" + "1" * 200 + ".5", "1 2", "7\t8", "--1", "+-1", ".e1", "1.e2",
        "4.9406564584124654e-324", "2.2250738585072014e-308", "1.7976931348623157e308"]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("textparse")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "opendba_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    return str(exe)


def _check(driver, tmp_path, lines):
    f = tmp_path / "lines.txt"
    f.write_bytes(("\n".join(lines) + "\n").encode("latin-1"))
    p = subprocess.run([driver, str(f)], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout[-3000:]


def test_edge_cases_match_stream_extraction(driver, tmp_path):
    _check(driver, tmp_path, EDGE)


def test_random_values_match_stream_extraction(driver, tmp_path):
    rng = np.random.default_rng(11)
    v = np.concatenate([rng.standard_normal(4000) * 10.0 ** rng.integers(-40, 40, 4000),
                        rng.standard_normal(2000), rng.uniform(-1e-300, 1e-300, 500),
                        rng.uniform(60, 140, 2000)])
    fmts = ["%g", "%.9g", "%.17g", "%e", "%.3f", "%.12E", " %g", "%+g", "%g\r", "%g x"]
    lines = [f % x for x in v for f in fmts[:1]] + [fmts[i % len(fmts)] % x for i, x in enumerate(v)]
    _check(driver, tmp_path, lines)


# The writers' number formatter (append_stream_value) against the stream's
# default output (`out << value`, precision 6), which the reference's
# pair_dists.txt writer uses (dba.hpp:186-216): the same characters for every
# value, float and double, finite or not.
FORMAT_DRIVER = r'''
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <sstream>
#include <string>
#include "text_parse.h"

template <typename T> static long check(T v) {
  std::string got;
  odba::append_stream_value(got, v);
  std::ostringstream want;
  want << v;
  if (got == want.str()) return 0;
  std::printf("mismatch [%s] [%s]\n", got.c_str(), want.str().c_str());
  return 1;
}

int main() {
  long bad = 0, n = 0;
  const double edge[] = {0.0, -0.0, 1.0, -1.0, 0.1, 1e-5, 1e-4, 123456.0, 1234567.0, 999999.5,
                         9999995.0, 0.000123456, 1e15, 1e16, 1e-300, 5e-324, 2.2250738585072014e-308,
                         1.7976931348623157e308, 3.4028234663852886e38, 1.1754943508222875e-38,
                         1.401298464324817e-45, 100000.0, 1e6, 0.5, 2.5e-7,
                         std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
                         std::numeric_limits<double>::quiet_NaN(), -std::numeric_limits<double>::quiet_NaN()};
  for (double e : edge) {
    bad += check(e) + check(float(e));
    n += 2;
  }
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> u(0.0, 400.0);
  for (int i = 0; i < 400000; ++i) {
    const uint64_t b = g();
    double d;
    std::memcpy(&d, &b, 8);
    const uint32_t c = uint32_t(b >> 17);
    float f;
    std::memcpy(&f, &c, 4);
    const double r = u(g);
    bad += check(d) + check(f) + check(r) + check(float(r)) + check(std::sqrt(r));
    n += 5;
  }
  std::printf("%ld values, %ld mismatches\n", n, bad);
  return bad ? 1 : 0;
}
'''


def test_number_formatter_matches_stream_output(tmp_path):
    src = tmp_path / "fmt.cpp"
    src.write_text(FORMAT_DRIVER)
    exe = tmp_path / "fmt"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "opendba_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout[-3000:]
