"""Stripe-mode DBA round (the reference's stripe mode, dba.hpp:515-763) on a
B200: the forward pass keeps swath edges and checkpoint rows, the backtrack
recomputes tiles stripe by stripe.  Without an open end, centroid, counts,
delta and every member's path must equal the full-path round bit for bit
(the full-path round is itself pinned to the reference's GPU outputs); with
an open end they must equal the reference's own stripe-mode runs
(tests/golden/ref/stripe_ref.json) and the oracle's restatement of them."""
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_reference_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api as A
    from opendba_b200 import build
    build.build_library()
    return A


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def _compare(api, centroid, members, os_, rows):
    import torch
    ds = api.DeviceSeries.from_host(members)
    c = torch.from_numpy(centroid).cuda()
    full = api.dba_round(c, ds, os_, 0, with_paths=True)
    strp = api.dba_round(c, ds, os_, 0, with_paths=True, stripe_rows=rows)
    assert np.array_equal(_bits(full[0].cpu().numpy()), _bits(strp[0].cpu().numpy()))
    assert np.array_equal(full[1].cpu().numpy(), strp[1].cpu().numpy())
    assert full[2] == strp[2]
    for k, (a, b) in enumerate(zip(full[3], strp[3])):
        assert np.array_equal(a, b), f"path of member {k}"


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", ["global", "open_start"])
def test_stripe_round_equals_reference_round(api, sfx, mode):
    # the reference's own DBA round fixture (members 200..2100, centroid 1100)
    members = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_members.odbs"))
    centroid = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_centroid.odbs"))[0]
    os_ = 1 if mode == "open_start" else 0
    import torch
    ds = api.DeviceSeries.from_host(members)
    mean, counts, delta, _ = api.dba_round(torch.from_numpy(centroid).cuda(), ds, os_, 0,
                                           stripe_rows=64)
    want = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.mean.odbs"))[0]
    assert np.array_equal(_bits(mean.cpu().numpy()), _bits(want))
    _compare(api, centroid, members, os_, 64)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("rows", [2, 32, 256, 0])
def test_stripe_round_many_swaths_and_tiles(api, dtype, rows):
    rng = np.random.default_rng(900 + rows)
    # centroid over several swaths (1024 float / 512 double columns), a partial
    # last swath; members shorter and longer than a tile, one of length 1
    centroid = (np.cumsum(rng.standard_normal(3333)) * 0.05).astype(dtype)
    lens = [1, 2, 63, 64, 65, 700, 2049, 5000, 9001]
    members = [(np.cumsum(rng.standard_normal(L)) * 0.05).astype(dtype) for L in lens]
    for os_ in (0, 1):
        _compare(api, centroid, members, os_, rows)


REF = json.load(open(os.path.join(GOLDEN, "stripe_ref.json")))
DT = {"f32": np.float32, "f64": np.float64}


def _file_order(paths, centroid, members, oe):
    """Path cells as the reference's path files list them (column first for
    members the open end flips), each as (ij int32, moves uint8)."""
    out = []
    for k, p in enumerate(paths):
        ij = np.asarray(p)[:, :2].astype(np.int32)
        if oe and len(centroid) < len(members[k]):
            ij = ij[:, ::-1]
        out.append((ij, np.asarray(p)[:, 2].astype(np.uint8)))
    return out


@pytest.mark.parametrize("case", sorted(REF["cases"]))
def test_stripe_round_matches_reference_stripe_mode(api, case):
    # every mode, float and double, against the reference's forced stripe-mode
    # runs; tile heights vary with the case
    import torch
    tag, sfx, mode = case.split("_", 2)
    os_, oe = G.MODES[mode]
    centroid, members = G.stripe_inputs(DT[sfx], tag)
    rows = {"a": 64, "b": 256, "c": 0, "d": 32, "e": 128, "f": 1024, "g": 16, "h": 512}[tag]
    ds = api.DeviceSeries.from_host(members)
    mean, counts, delta, paths = api.dba_round(torch.from_numpy(centroid).cuda(), ds, os_, oe,
                                               with_paths=True, stripe_rows=rows)
    want = REF["cases"][case]
    assert G._sha(mean.cpu().numpy().tobytes()) == want["mean"]
    assert delta == float(want["delta"])
    got = [G.path_digest(ij, mv) for ij, mv in _file_order(paths, centroid, members, oe)]
    assert got == want["paths"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", [(0, 1), (1, 1)])
def test_stripe_round_open_end_edge_cases_vs_oracle(api, dtype, mode):
    # one-row and one-column matrices, members on both sides of the flip,
    # lengths at stripe edges, a member that starts with the centroid (the
    # forward shortcut fires early), tile heights 2 and the default
    import torch
    rng = np.random.default_rng(77 + mode[0])
    centroid = (np.cumsum(rng.standard_normal(2100)) * 0.1).astype(dtype)
    lens = [1, 2, 511, 512, 513, 1023, 1024, 1025, 2099, 2100, 2101, 3072, 4097]
    members = [(np.cumsum(rng.standard_normal(L)) * 0.1).astype(dtype) for L in lens]
    members.append(np.concatenate([centroid, rng.standard_normal(2500).astype(dtype)]))
    ds = api.DeviceSeries.from_host(members)
    w_mean, w_counts, w_delta, w_paths, _ = O.dba_update_stripe(centroid, members, *mode)
    for rows in (2, 0):
        mean, counts, delta, paths = api.dba_round(torch.from_numpy(centroid).cuda(), ds, *mode,
                                                   with_paths=True, stripe_rows=rows)
        assert np.array_equal(_bits(mean.cpu().numpy()), _bits(w_mean)), rows
        assert np.array_equal(counts.cpu().numpy().astype(np.uint32), w_counts), rows
        assert delta == w_delta
        for k in range(len(members)):
            assert np.array_equal(paths[k], w_paths[k].astype(np.int32)), (rows, k)


def test_stripe_round_rejects_bad_rows(api):
    import torch
    from opendba_b200 import _native
    members = [np.ones(50, np.float32), np.arange(70, dtype=np.float32)]
    ds = api.DeviceSeries.from_host(members)
    c = torch.ones(40, dtype=torch.float32, device="cuda")
    with pytest.raises(_native.OdbaError):
        api.dba_round(c, ds, 0, 0, stripe_rows=48, workspace=torch.empty(1 << 20, dtype=torch.uint8,
                                                                          device="cuda"))


@pytest.mark.parametrize("tag,mode", [("f32_global", (0, 0)), ("f64_global", (0, 0))])
def test_perform_dba_forced_stripe_files_byte_identical(tmp_path, tag, mode):
    # performDBA end to end with every round in stripe mode (small tiles):
    # the same avg.txt and path files as the reference's run
    import subprocess
    import sys
    from conftest import ROOT
    src = os.path.join(GOLDEN, f"perform_{tag}.odbs")
    prefix = str(tmp_path / f"perform_{tag}")
    code = ("import sys; sys.path.insert(0, %r)\n" % ROOT +
            "from oracle import oracle as O\nfrom opendba_b200 import api\n"
            f"s = O.read_bundle({src!r})\n"
            f"api.perform_dba(s, ['s%d' % i for i in range(len(s))], {prefix!r}, {mode[0]}, {mode[1]}, norm=1)")
    env = dict(os.environ, ODBA_FORCE_STRIPE="1", ODBA_STRIPE_ROWS="64")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    with open(prefix + ".avg.txt") as f, open(os.path.join(GOLDEN, f"perform_{tag}.avg.txt")) as g:
        assert f.read() == g.read()
    gold = np.load(os.path.join(GOLDEN, f"perform_{tag}.paths.npz"))
    k = 0
    while f"ij{k}" in gold:
        with open(f"{prefix}.0.path{k}.txt") as f:
            rows = [ln.split("\t") for ln in f.read().splitlines()[1:]]
        ij = np.array([(int(r[0]), int(r[2])) for r in rows], dtype=np.int32)
        assert np.array_equal(ij, gold[f"ij{k}"]), f"path {k}"
        k += 1
    assert k == 10
