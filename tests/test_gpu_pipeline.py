"""The drop-in pipeline on a B200: setupAndRun / performDBA / segmentation and
the openDBA CLI, checked against the reference's own outputs (tests/golden/ref/)
file for file.

The pipeline entry points end the process on fatal errors like the
reference, so each run happens in a child process.
"""
import gzip
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def built():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import build
    build.build_library()
    return True


def _child(code: str, cwd=ROOT):
    p = subprocess.run([sys.executable, "-c", "import sys; sys.path.insert(0, %r)\n" % ROOT + code],
                       cwd=cwd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    return p


def _read(path):
    with open(path) as f:
        return f.read()


SECTIONS = {
    "gsd": (0, ["random_short1.txt", "random_short1.txt"]),
    "gdd": (0, ["random_short1.txt", "random_short2.txt"]),
    "gtd": (0, ["random_short1.txt", "random_short2.txt", "random_short3.txt"]),
    "gdtd": (1, ["random_short1.txt", "random_trun_short2.txt"]),
    "gld": (0, ["random_large0.txt", "random_large1.txt"]),
}


@pytest.mark.parametrize("name", list(SECTIONS))
def test_reference_test_sections_byte_identical(built, tmp_path, name):
    oe, files = SECTIONS[name]
    rel = [f"tests/golden/ref_fixtures/{f}" for f in files]  # names are cut at the first '.'
    prefix = str(tmp_path / f"sar_{name}")
    _child(f"from opendba_b200 import api\napi.setup_and_run({rel!r}, {prefix!r}, read_mode=0, "
           f"open_end={oe}, norm=0)")
    assert _read(prefix + ".avg.txt") == _read(os.path.join(GOLDEN, f"sar_{name}.avg.txt"))
    assert _read(prefix + ".pair_dists.txt") == _read(os.path.join(GOLDEN, f"sar_{name}.pair_dists.txt"))


@pytest.mark.parametrize("tag,mode", [("f32_global", (0, 0)), ("f32_open_end", (0, 1)),
                                      ("f64_global", (0, 0))])
def test_perform_dba_files_byte_identical(built, tmp_path, tag, mode):
    src = os.path.join(GOLDEN, f"perform_{tag}.odbs")
    prefix = str(tmp_path / f"perform_{tag}")
    _child("from oracle import oracle as O\nfrom opendba_b200 import api\n"
           f"s = O.read_bundle({src!r})\n"
           f"api.perform_dba(s, ['s%d' % i for i in range(len(s))], {prefix!r}, {mode[0]}, {mode[1]}, norm=1)")
    assert _read(prefix + ".avg.txt") == _read(os.path.join(GOLDEN, f"perform_{tag}.avg.txt"))
    assert _read(prefix + ".pair_dists.txt") == _read(os.path.join(GOLDEN, f"perform_{tag}.pair_dists.txt"))
    assert not os.path.exists(prefix + ".0.evolving_centroid.txt")
    gold = np.load(os.path.join(GOLDEN, f"perform_{tag}.paths.npz"))
    k = 0
    while f"ij{k}" in gold:
        rows = [ln.split("\t") for ln in _read(f"{prefix}.0.path{k}.txt").splitlines()[1:]]
        ij = np.array([(int(r[0]), int(r[2])) for r in rows], dtype=np.int32)
        assert np.array_equal(ij, gold[f"ij{k}"]), f"path {k}"
        k += 1
    assert k == 10


def test_path_file_text_byte_identical(built, tmp_path):
    # one DBA round through DBAUpdate's file writer, against the reference's own path files
    members = O.read_bundle(os.path.join(GOLDEN, "dba_f32_members.odbs"))
    centroid = O.read_bundle(os.path.join(GOLDEN, "dba_f32_centroid.odbs"))[0]
    import torch
    from opendba_b200 import api
    for mode, oe in (("global", 0), ("open_end", 1)):
        ds = api.DeviceSeries.from_host(members)
        _, _, _, paths = api.dba_round(torch.from_numpy(centroid).cuda(), ds, 0, oe, with_paths=True)
        for k in (0, 5):
            with gzip.open(os.path.join(GOLDEN, f"dba_f32_{mode}.path{k}.txt.gz"), "rt") as f:
                want = f.read()
            seq, flip = members[k], oe and len(centroid) < len(members[k])
            lines = [f"s{k}"]
            for (i, j, mv) in paths[k][:-1]:
                a, b = (j, i) if flip else (i, j)
                va, vb = (seq[j], centroid[i]) if flip else (seq[i], centroid[j])
                lines.append(f"{a}\t{'%g' % va}\t{b}\t{'%g' % vb}\t{O.MOVE_NAMES[int(mv)]}")
            i, j, mv = paths[k][-1]
            lines.append(f"{i}\t{'%g' % seq[i]}\t{j}\t{'%g' % centroid[j]}\t{O.MOVE_NAMES[int(mv)]}")
            assert "\n".join(lines) + "\n" == want, f"{mode} member {k}"


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("minseg", [4, 6])
def test_segmentation_bit_exact_vs_reference_gpu(built, sfx, minseg):
    from opendba_b200 import api
    series = O.read_bundle(os.path.join(GOLDEN, f"seg_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"seg_{sfx}_m{minseg}.odbs"))
    got = api.segment_host(series, minseg)
    for a, b in zip(got, ref):
        assert len(a) == len(b)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_segmentation_random_vs_oracle(built):
    from opendba_b200 import api
    rng = np.random.default_rng(31)
    from opendba_b200 import synth
    for minseg in (1, 3, 5, 9):
        series = [synth.step_signal(rng, int(L), 90, 12, 8, 1.5).astype(np.float32)
                  for L in (1, 2, 130, 511, 512, 513, 1500, 4097)]
        got = api.segment_host(series, minseg)
        want = O.segment(series, minseg)
        for a, b in zip(got, want):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), minseg


def test_cli_text_inputs(built, tmp_path):
    rng = np.random.default_rng(8)
    files = []
    series = []
    for k in range(4):
        # float32 values printed with 9 significant digits parse back exactly
        x = (np.cumsum(rng.standard_normal(int(rng.integers(50, 400)))) + 20).astype(np.float32)
        fn = tmp_path / f"in{k}.txt"
        fn.write_text("".join("%.9g\n" % v for v in x))
        files.append(str(fn))
        series.append(x)
    prefix = str(tmp_path / "cli")
    cli = os.path.join(ROOT, "opendba_b200", "bin", "openDBA")
    p = subprocess.run([cli, "text", "float", "global", prefix, "0", "/dev/null", "1"] + files,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    r = O.perform_dba(series, 0, 0, norm=1, fma_mode=1)
    name = files[r["order"][r["medoid"]]].split(".")[0]
    want = name + "".join("\t" + "%g" % float(v) for v in r["centroid"]) + "\n"
    assert _read(prefix + ".avg.txt") == want


@pytest.mark.parametrize("kind", ["tsv", "binary"])
@pytest.mark.parametrize("ty", ["float", "double"])
def test_cli_tsv_and_binary_inputs(built, tmp_path, kind, ty):
    # the other two read modes of the CLI (cpu_utils.hpp:60-91, 381-456): one
    # TSV file with a named series per line, or one raw binary file per series
    dt = np.float32 if ty == "float" else np.float64
    fmt = "%.9g" if ty == "float" else "%.17g"  # both parse back exactly
    rng = np.random.default_rng(9 if kind == "tsv" else 10)
    series = [(np.cumsum(rng.standard_normal(int(rng.integers(50, 400)))) + 20).astype(dt)
              for _ in range(5)]
    if kind == "tsv":
        fn = tmp_path / "in.tsv"
        fn.write_text("".join(f"s{k}" + "".join("\t" + fmt % v for v in x) + "\n"
                              for k, x in enumerate(series)))
        files, names = [str(fn)], [f"s{k}" for k in range(len(series))]
    else:
        files = []
        for k, x in enumerate(series):
            fn = tmp_path / f"in{k}.bin"
            x.tofile(fn)
            files.append(str(fn))
        names = [f.split(".")[0] for f in files]
    prefix = str(tmp_path / f"cli_{kind}_{ty}")
    cli = os.path.join(ROOT, "opendba_b200", "bin", "openDBA")
    p = subprocess.run([cli, kind, ty, "global", prefix, "0", "/dev/null", "1"] + files,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    r = O.perform_dba(series, 0, 0, norm=1, fma_mode=1)
    want = names[r["order"][r["medoid"]]] + "".join("\t" + "%g" % float(v) for v in r["centroid"]) + "\n"
    assert _read(prefix + ".avg.txt") == want


def test_cli_rejects_bad_arguments(built, tmp_path):
    cli = os.path.join(ROOT, "opendba_b200", "bin", "openDBA")
    p = subprocess.run([cli, "text", "float"], capture_output=True, text=True)
    assert p.returncode == 1 and "Usage" in p.stdout
    p = subprocess.run([cli, "csv", "float", "global", str(tmp_path / "x"), "0", "/dev/null", "1", "a"],
                       capture_output=True, text=True)
    assert p.returncode == 1
    p = subprocess.run([cli, "text", "float", "global", str(tmp_path / "x"), "0", "/dev/null", "1",
                        str(tmp_path / "missing.txt")], capture_output=True, text=True)
    assert p.returncode == 32  # NOT_ENOUGH_SEQUENCES


@pytest.mark.parametrize("tag", ["f32_global_c0.3", "f32_global_c3", "f32_global_c0", "f64_open_end_c0.45"])
def test_perform_dba_clusters_byte_identical(built, tmp_path, tag):
    # clustering thresholds other than 1: the reference's run (with this
    # project's complete linkage in place of hclust-cpp) gives the golden files
    sfx, rest = tag.split("_", 1)
    mode, c = rest.rsplit("_c", 1)
    gold = os.path.join(GOLDEN, f"cluster_{tag}")
    if not os.path.exists(gold + ".avg.txt"):
        pytest.skip("cluster golden files not generated")
    src = os.path.join(GOLDEN, f"cluster_{sfx}.odbs")
    prefix = str(tmp_path / f"cluster_{tag}")
    os_, oe = {"global": (0, 0), "open_end": (0, 1)}[mode]
    _child("from oracle import oracle as O\nfrom opendba_b200 import api\n"
           f"s = O.read_bundle({src!r})\n"
           f"api.perform_dba(s, ['s%d' % i for i in range(len(s))], {prefix!r}, {os_}, {oe}, norm=1, "
           f"cdist={float(c)})")
    for ext in (".cluster_membership.txt", ".avg.txt", ".pair_dists.txt"):
        assert _read(prefix + ext) == _read(gold + ext), ext


@pytest.mark.parametrize("norm", [1, 0])
def test_setup_and_run_prefix_chop_byte_identical(built, tmp_path, norm):
    # setupAndRun with a leader file: the reference's prefix_chop.txt (chop
    # positions, lengths, leader-row histograms) and the averages of the tails
    d = os.path.join(GOLDEN, "chop_inputs")
    gold = os.path.join(GOLDEN, f"chop_n{norm}")
    if not os.path.exists(gold + ".prefix_chop.txt"):
        pytest.skip("prefix chop golden files not generated")
    files = sorted(f for f in os.listdir(d) if f.startswith("read"))
    prefix = str(tmp_path / f"chop_n{norm}")
    _child("from opendba_b200 import api\n"
           f"api.setup_and_run({files!r}, {prefix!r}, 0, 0, 0, '0', {norm}, 1.0, "
           f"seqprefix_file={os.path.join(d, 'leader.txt')!r})", cwd=d)
    for ext in (".prefix_chop.txt", ".avg.txt", ".pair_dists.txt"):
        assert _read(prefix + ext) == _read(gold + ext), ext
