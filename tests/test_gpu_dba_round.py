"""Parity of the CUDA DBA round (path DTW, backtrack, ordered centroid update).

Bit-exact against the reference's own GPU round (tests/golden/ref/dba_*: the
updated centroid, the delta and every member's path) and against the CPU
oracle on seeded random cases, including the open-end shortcut and flipped
(centroid-on-rows) members, through the C ABI.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api, build
    build.build_library()
    return torch, api


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def _round(env, centroid, members, os_, oe, with_paths=True):
    torch, api = env
    ds = api.DeviceSeries.from_host(members)
    c = torch.from_numpy(np.ascontiguousarray(centroid)).cuda()
    mean, counts, delta, paths = api.dba_round(c, ds, os_, oe, with_paths=with_paths)
    return mean.cpu().numpy(), counts.cpu().numpy(), delta, paths


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_round_matches_reference_gpu(env, sfx, mode):
    members = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_members.odbs"))
    centroid = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_centroid.odbs"))[0]
    ref = O.read_bundle(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.mean.odbs"))[0]
    with open(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.delta.txt")) as f:
        ref_delta = float(f.read())
    os_, oe = MODES[mode]
    mean, counts, delta, paths = _round(env, centroid, members, os_, oe)
    assert np.array_equal(_bits(mean), _bits(ref))
    assert delta == ref_delta
    gold = np.load(os.path.join(GOLDEN, f"dba_{sfx}_{mode}.paths.npz"))
    for k, seq in enumerate(members):
        ij = gold[f"ij{k}"].copy()
        if oe and len(centroid) < len(seq):
            ij[:-1] = ij[:-1, ::-1]  # flipped members print "column, row"
        assert np.array_equal(paths[k][:, :2], ij), f"member {k} path cells"
        assert np.array_equal(paths[k][:, 2].astype(np.uint8), gold[f"mv{k}"]), f"member {k} moves"


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", list(MODES))
def test_round_random_vs_oracle(env, dtype, mode):
    rng = np.random.default_rng(99 + list(MODES).index(mode))
    os_, oe = MODES[mode]
    # centroid 1500 > 1024: two swaths; members shorter (shortcut candidates
    # in open_end) and longer (flipped in open_end), ragged
    lens = [3, 40, 700, 1023, 1024, 1025, 1499, 1500, 1501, 2100, 3300, 500]
    members = [np.cumsum(rng.standard_normal(L)).astype(dtype) for L in lens]
    centroid = np.cumsum(rng.standard_normal(1500)).astype(dtype)
    mean, counts, delta, paths = _round(env, centroid, members, os_, oe)
    w_mean, w_counts, _, w_delta = O.dba_update(centroid, members, os_, oe, fma_mode=1)
    assert np.array_equal(_bits(mean), _bits(w_mean))
    assert np.array_equal(counts.astype(np.uint32), w_counts)
    assert delta == w_delta
    for k, seq in enumerate(members):
        t = O.path_triples(centroid, seq, os_, oe, fma_mode=1)
        assert np.array_equal(paths[k], t.astype(np.int32)), f"member {k}"


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", list(MODES))
def test_round_padded_last_swath_vs_oracle(env, dtype, mode):
    # last swaths 864-896 columns wide, which the float round sweeps at the
    # full 32 columns per lane (the extra columns are never walked): the
    # 1900-sample centroid's (876), and with the open end the flipped
    # members' (1904: 880, 2940: 892); both walks (ranges, path listing)
    rng = np.random.default_rng(1900 + list(MODES).index(mode))
    os_, oe = MODES[mode]
    lens = [5, 870, 1100, 1900, 1904, 2940, 3000]
    members = [np.cumsum(rng.standard_normal(L)).astype(dtype) for L in lens]
    centroid = np.cumsum(rng.standard_normal(1900)).astype(dtype)
    w_mean, w_counts, _, w_delta = O.dba_update(centroid, members, os_, oe, fma_mode=1)
    for with_paths in (False, True):
        mean, counts, delta, paths = _round(env, centroid, members, os_, oe, with_paths)
        assert np.array_equal(_bits(mean), _bits(w_mean)), with_paths
        assert np.array_equal(counts.astype(np.uint32), w_counts)
        assert delta == w_delta
    for k, seq in enumerate(members):
        t = O.path_triples(centroid, seq, os_, oe, fma_mode=1)
        assert np.array_equal(paths[k], t.astype(np.int32)), f"member {k}"


@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_round_open_end_shortcut_lane_matches_reference_gpu(env, sfx):
    # a 629-row centroid against longer members: the double build's shortcut
    # reads warp-0 lane 16's partial minimum (rows r % 1024 >= 512), which
    # changes this round's paths (the full minimum would not)
    members = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_members.odbs"))
    centroid = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_centroid.odbs"))[0]
    ref = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_open_end.mean.odbs"))[0]
    with open(os.path.join(GOLDEN, f"sc_dba_{sfx}_open_end.delta.txt")) as f:
        ref_delta = float(f.read())
    mean, counts, delta, paths = _round(env, centroid, members, 0, 1)
    assert np.array_equal(_bits(mean), _bits(ref))
    assert delta == ref_delta
    gold = np.load(os.path.join(GOLDEN, f"sc_dba_{sfx}_open_end.paths.npz"))
    for k, seq in enumerate(members):
        ij = gold[f"ij{k}"].copy()
        if len(centroid) < len(seq):
            ij[:-1] = ij[:-1, ::-1]
        assert np.array_equal(paths[k][:, :2], ij), f"member {k} path cells"
        assert np.array_equal(paths[k][:, 2].astype(np.uint8), gold[f"mv{k}"]), f"member {k} moves"


def test_round_open_end_shortcut_fires(env):
    # a short member against a long flat centroid: the top row becomes the
    # column minimum early, so the reference's shortcut decides the path end
    rng = np.random.default_rng(5)
    centroid = np.concatenate([np.cumsum(rng.standard_normal(300)), np.zeros(3000)]).astype(np.float32)
    members = [centroid[:300].copy() + 0.01 * rng.standard_normal(300).astype(np.float32),
               centroid[:250].copy()]
    mean, counts, delta, paths = _round(env, centroid, members, 0, 1)
    w_mean, w_counts, _, w_delta = O.dba_update(centroid, members, 0, 1, fma_mode=1)
    assert np.array_equal(_bits(mean), _bits(w_mean))
    for k, seq in enumerate(members):
        t = O.path_triples(centroid, seq, 0, 1, fma_mode=1)
        assert np.array_equal(paths[k], t.astype(np.int32))
        assert (paths[k][:, 2] == 4).sum() > 1000  # a long OPEN_RIGHT run on the top row


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_round_split_into_ranges_and_reduce_equals_whole_round(env, sfx, mode):
    # the multi-GPU round's two halves on one GPU: members dealt into three
    # blocks (sharding.member_shards), ranges per block through
    # odba_dba_round_ranges_*, concatenated in member order, reduced by
    # odba_dba_reduce_ranges_* -- bit-identical to odba_dba_round_*, and the
    # ranges equal the oracle's walk
    torch, api = env
    from opendba_b200 import sharding
    os_, oe = MODES[mode]
    dt = np.float32 if sfx == "f32" else np.float64
    rng = np.random.default_rng(808 + len(mode))
    members = [rng.standard_normal(int(L)).astype(dt) for L in rng.integers(200, 2600, size=14)]
    centroid = rng.standard_normal(1300).astype(dt)
    ds = api.DeviceSeries.from_host(members)
    c = torch.from_numpy(centroid).cuda()
    want_mean, want_counts, want_delta, _ = api.dba_round(c, ds, os_, oe)
    shards = sharding.member_shards(ds.host_lens, 3)
    parts = [api.dba_round_ranges(c, ds.subset(b, e), os_, oe) for b, e in shards]
    ranges = torch.cat(parts, dim=0)
    assert np.array_equal(ranges.cpu().numpy(), O.member_ranges(centroid, members, os_, oe))
    mean, counts, delta = api.dba_reduce_ranges(c, ds, ranges, os_, oe)
    assert np.array_equal(_bits(mean.cpu().numpy()), _bits(want_mean.cpu().numpy()))
    assert np.array_equal(counts.cpu().numpy(), want_counts.cpu().numpy())
    assert delta == want_delta
    mean1, _, delta1 = sharding.dba_round_sharded(c, ds, 0, 1, os_, oe)
    assert np.array_equal(_bits(mean1.cpu().numpy()), _bits(want_mean.cpu().numpy()))
    assert delta1 == want_delta


@pytest.mark.parametrize("nb", [2, 3, 8])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", list(MODES))
def test_round_row_bands_vs_oracle(env, nb, dtype, mode):
    # the path DTW's rows cut into bands (odba_round_set_bands): bands of at
    # least 1024 rows, so these members make 1 to 5 bands, last bands of 1, 2,
    # 4 or 53 rows among them; flipped members (open end, member longer than
    # the 2500-sample centroid) band the centroid's rows
    torch, api = env
    from opendba_b200 import _native
    lib = _native.lib()
    rng = np.random.default_rng(4242 + nb + list(MODES).index(mode))
    os_, oe = MODES[mode]
    lens = [5, 900, 2047, 2048, 2049, 2050, 3001, 4100, 2600, 1025]
    members = [np.cumsum(rng.standard_normal(L)).astype(dtype) for L in lens]
    centroid = np.cumsum(rng.standard_normal(2500)).astype(dtype)
    w_mean, w_counts, _, w_delta = O.dba_update(centroid, members, os_, oe, fma_mode=1)
    assert lib.odba_round_set_bands(nb) == 0
    try:
        for with_paths in (False, True):
            mean, counts, delta, paths = _round(env, centroid, members, os_, oe, with_paths)
            assert np.array_equal(_bits(mean), _bits(w_mean)), with_paths
            assert np.array_equal(counts.astype(np.uint32), w_counts)
            assert delta == w_delta
        for k, seq in enumerate(members):
            t = O.path_triples(centroid, seq, os_, oe, fma_mode=1)
            assert np.array_equal(paths[k], t.astype(np.int32)), f"member {k}"
    finally:
        lib.odba_round_set_bands(0)


@pytest.mark.parametrize("nb", [1, 2, 4])
def test_round_row_bands_keep_the_open_end_shortcut(env, nb):
    # a 1500-row member against a long flat centroid: the shortcut's minimum
    # is the least over both bands of the swath's right edge
    torch, api = env
    from opendba_b200 import _native
    lib = _native.lib()
    rng = np.random.default_rng(6)
    centroid = np.concatenate([np.cumsum(rng.standard_normal(1500)), np.zeros(4000)]).astype(np.float32)
    members = [centroid[:1500] + 0.01 * rng.standard_normal(1500).astype(np.float32),
               centroid[:1300].copy()]
    assert lib.odba_round_set_bands(nb) == 0
    try:
        mean, counts, delta, paths = _round(env, centroid, members, 0, 1)
    finally:
        lib.odba_round_set_bands(0)
    w_mean, w_counts, _, w_delta = O.dba_update(centroid, members, 0, 1, fma_mode=1)
    assert np.array_equal(_bits(mean), _bits(w_mean))
    assert delta == w_delta
    for k, seq in enumerate(members):
        t = O.path_triples(centroid, seq, 0, 1, fma_mode=1)
        assert np.array_equal(paths[k], t.astype(np.int32))
    assert (paths[0][:, 2] == 4).sum() > 1000  # the shortcut's OPEN_RIGHT run

