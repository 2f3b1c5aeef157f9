"""Pins the CPU oracle against the reference's own answers (CPU only).

Two sources of truth:
* the reference's known-answer tests (tests/openDBA_test.cu in the reference:
  centroids to three decimals on its test2 fixtures), and
* the reference's own GPU build run on a B200 (tests/golden/ref/, produced by
  tests/golden/make_reference_golden.py through oracle/_ref/ref_harness).
"""
import json
import os

import numpy as np
import pytest

from conftest import FIXTURES, GOLDEN
from oracle import oracle as O

MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}


def _bits(a):
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def _fx(name):
    return np.loadtxt(os.path.join(FIXTURES, name), dtype=np.float64).astype(np.float32)


def r3(v):
    # the reference test's round_to_three: "%.3f" then parsed back (tests/test_utils.cuh:20-36)
    return float(np.float32(float("%.3f" % v)))


# Known answers of tests/openDBA_test.cu (sections at :66-107, :109-150, :152-194,
# :196-245, :247-299), global mode unless noted, no z-norm, cdist 1.
KNOWN = {
    "same": (["random_short1.txt", "random_short1.txt"], 0,
             [1, 0.895, 0.8, 0.644, 0.586, 0.488, 0.357, 0.287, 0.139, 0.017]),
    "different": (["random_short1.txt", "random_short2.txt"], 0,
                  [1, 0.895, 0.796, 0.665, 0.59, 0.456, 0.347, 0.265, 0.137, 0.05]),
    "three": (["random_short1.txt", "random_short2.txt", "random_short3.txt"], 0,
              [0.972, 0.901, 0.814, 0.681, 0.56, 0.455, 0.362, 0.244, 0.128, 0.056]),
    "truncated_open_end": (["random_short1.txt", "random_trun_short2.txt"], 1,
                           [1, 0.895, 0.796, 0.665, 0.59, 0.488, 0.357, 0.287, 0.139, 0.017]),
}


@pytest.mark.parametrize("name", list(KNOWN))
def test_reference_known_answers(name):
    files, oe, expected = KNOWN[name]
    r = O.perform_dba([_fx(f) for f in files], open_end=oe, norm=0, fma_mode=1)
    got = [r3(v) for v in r["centroid"]]
    assert got == [float(np.float32(e)) for e in expected]


def test_reference_known_answer_large():
    r = O.perform_dba([_fx("random_large0.txt"), _fx("random_large1.txt")], norm=0, fma_mode=1)
    c = r["centroid"]
    assert len(c) == 2048
    assert c[0] == 1
    assert [r3(c[1]), r3(c[2]), r3(c[3]), r3(c[2047])] == [
        float(np.float32(v)) for v in (0.997, 1, 0.959, -0.457)]


def test_harness_runs_all_succeeded():
    with open(os.path.join(GOLDEN, "harness_log.jsonl")) as f:
        runs = [json.loads(line) for line in f]
    assert runs and all(r["rc"] == 0 for r in runs)


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_pairwise_bit_exact_vs_reference_gpu(sfx, mode):
    series = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}_{mode}.dist.odbs"))[0]
    got = O.pairwise(series, *MODES[mode], fma_mode=1)
    assert np.array_equal(_bits(got), _bits(ref))


@pytest.mark.parametrize("mode", ["global", "open_end"])
def test_pairwise_plain_dba_workload_bit_exact(mode):
    series = O.read_bundle(os.path.join(GOLDEN, "pw_c1_f32.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"pw_c1_f32_{mode}.dist.odbs"))[0]
    got = O.pairwise(series, *MODES[mode], fma_mode=1)
    assert np.array_equal(_bits(got), _bits(ref))
    # the unfused rounding is distinguishable on the same data, so the pin is meaningful
    unfused = O.pairwise(series, *MODES[mode], fma_mode=0)
    assert not np.array_equal(_bits(unfused), _bits(ref))


def test_medoid_and_pair_dists_text_match_reference():
    series = O.read_bundle(os.path.join(GOLDEN, "pw_c1_f32.odbs"))
    d = O.pairwise(series, 0, 0, fma_mode=1)
    lens = np.array([len(s) for s in series], dtype=np.uint64)
    m, _ = O.medoid(d, lens)
    with open(os.path.join(GOLDEN, "medoid_c1_f32_global.medoid.txt")) as f:
        assert int(f.read()) == m
    n = len(series)
    lines, off = [], 0
    for s in range(n - 1):
        row = [f"s{s}" + "\t" * s + "\t0"]
        row += ["\t" + "%g" % float(v) for v in d[off:off + n - s - 1]]
        off += n - s - 1
        lines.append("".join(row))
    lines.append(f"s{n - 1}" + "\t" * n + "0")
    with open(os.path.join(GOLDEN, "medoid_c1_f32_global.pair_dists.txt")) as f:
        assert f.read() == "\n".join(lines) + "\n"


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_dba_round_bit_exact_vs_reference_gpu(sfx, mode):
    members = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_members.odbs"))
    centroid = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_centroid.odbs"))[0]
    ref = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.mean.odbs"))[0]
    with open(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.delta.txt")) as f:
        ref_delta = float(f.read())
    os_, oe = MODES[mode]
    mean, _, _, delta = O.dba_update(centroid, members, os_, oe, fma_mode=1)
    assert np.array_equal(_bits(mean), _bits(ref))  # NaN columns (no pile-up) included
    assert delta == ref_delta
    paths = np.load(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.paths.npz"))
    for k, seq in enumerate(members):
        t = O.path_triples(centroid, seq, os_, oe, fma_mode=1)
        ij = paths[f"ij{k}"].copy()
        if oe and len(centroid) < len(seq):
            ij[:-1] = ij[:-1, ::-1]  # flipped members print "column, row" (io_utils.hpp:305-307)
        assert np.array_equal(t[:, :2], ij)
        assert np.array_equal(t[:, 2].astype(np.uint8), paths[f"mv{k}"])


@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_znorm_bit_exact_vs_reference_gpu(sfx):
    series = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.norm.odbs"))
    means = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.means.odbs"))[0]
    sigmas = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.sigmas.odbs"))[0]
    out, m, s = O.znorm(series)
    for a, b in zip(out, ref):
        assert np.array_equal(_bits(a), _bits(b))
    assert np.array_equal(m, means) and np.array_equal(s, sigmas)


def test_znorm_known_answer_population_sigma():
    for name in ("seq1_test", "seq2_test"):
        x = np.loadtxt(os.path.join(FIXTURES, name + ".txt"))
        want = np.loadtxt(os.path.join(FIXTURES, name + "_znorm.txt"))
        out, _, _ = O.znorm([x.astype(np.float64)])
        n = min(len(want), len(out[0]))
        assert np.allclose(out[0][:n], want[:n], atol=1e-12)


@pytest.mark.parametrize("tag,mode", [("f32_global", "global"), ("f32_open_end", "open_end"),
                                      ("f64_global", "global")])
def test_perform_dba_avg_text_matches_reference(tag, mode):
    series = O.read_bundle(os.path.join(GOLDEN, f"perform_{tag}.odbs"))
    r = O.perform_dba(series, *MODES[mode], norm=1, fma_mode=1)
    name = f"s{r['order'][r['medoid']]}"
    want = name + "".join("\t" + "%g" % float(v) for v in r["centroid"]) + "\n"
    with open(os.path.join(GOLDEN, f"perform_{tag}.avg.txt")) as f:
        assert f.read() == want
