"""Complete linkage, dendrogram cuts and per-cluster medoids of the medoid
pass (clustering.cpp, host code in the C-ABI library) against the CPU oracle
(oracle/clustering_oracle.py).  No GPU needed."""
import ctypes

import numpy as np
import pytest

from oracle import clustering_oracle as CO


@pytest.fixture(scope="module")
def lib():
    from opendba_b200 import _native, build
    build.build_library()
    return _native.lib()


def _vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _linkage(lib, n, D):
    merge = np.zeros(2 * (n - 1), dtype=np.int32)
    height = np.zeros(max(n - 1, 1))
    D = np.ascontiguousarray(D, dtype=np.float64)
    assert lib.odba_complete_linkage(n, _vp(D), _vp(merge), _vp(height)) == 0
    return merge.reshape(2, n - 1).T, height[: n - 1]


@pytest.mark.parametrize("n", [2, 3, 4, 10, 41])
def test_complete_linkage_matches_plain_agglomeration(lib, n):
    rng = np.random.default_rng(n)
    D = rng.random(n * (n - 1) // 2)  # tie-free
    got_m, got_h = _linkage(lib, n, D)
    want_m, want_h = CO.complete_linkage(n, D)
    assert np.array_equal(got_m, want_m)
    assert np.array_equal(got_h, want_h)


def test_complete_linkage_on_points_in_the_plane(lib):
    rng = np.random.default_rng(7)
    pts = np.concatenate([rng.normal(c, 0.3, size=(12, 2)) for c in ((0, 0), (5, 0), (0, 5))])
    n = len(pts)
    D = np.array([np.hypot(*(pts[i] - pts[j])) for i in range(n) for j in range(i + 1, n)])
    got_m, got_h = _linkage(lib, n, D)
    want_m, want_h = CO.complete_linkage(n, D)
    assert np.array_equal(got_m, want_m) and np.array_equal(got_h, want_h)
    assert np.all(np.diff(got_h) >= 0)
    # three well separated groups: a cut between the within- and between-group heights
    labels = np.zeros(n, dtype=np.int32)
    flat = np.ascontiguousarray(got_m.T.reshape(-1), dtype=np.int32)
    assert lib.odba_cutree_cdist(n, _vp(flat), _vp(np.ascontiguousarray(got_h)), ctypes.c_double(3.0),
                                 _vp(labels)) == 0
    assert sorted(np.bincount(labels)) == [12, 12, 12]
    assert labels[0] == 0 and labels[12] == 1 and labels[24] == 2


@pytest.mark.parametrize("n", [5, 23])
def test_cuts_match_oracle(lib, n):
    rng = np.random.default_rng(100 + n)
    D = rng.random(n * (n - 1) // 2)
    m, h = _linkage(lib, n, D)
    flat = np.ascontiguousarray(m.T.reshape(-1), dtype=np.int32)
    labels = np.zeros(n, dtype=np.int32)
    for k in range(0, n + 2):
        assert lib.odba_cutree_k(n, _vp(flat), k, _vp(labels)) == 0
        assert np.array_equal(labels, CO.cutree_k(n, m, k)), k
    for c in (0.0, 0.1, 0.3, 0.5, 0.9, 2.0):
        assert lib.odba_cutree_cdist(n, _vp(flat), _vp(np.ascontiguousarray(h)), ctypes.c_double(c),
                                     _vp(labels)) == 0
        assert np.array_equal(labels, CO.cutree_cdist(n, m, h, c)), c


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("cdist", [1.0, 0.0, 0.35, 0.6, 2.0, 3.0, 7.0, -1.0])
def test_memberships_and_medoids_match_oracle(lib, dtype, cdist):
    rng = np.random.default_rng(31)
    n = 30
    lens = rng.integers(100, 900, size=n).astype(np.uint64)
    # three families: distances small within, large between (plus noise)
    fam = rng.integers(0, 3, size=n)
    d = []
    for i in range(n):
        for j in range(i + 1, n):
            base = 1.0 if fam[i] == fam[j] else 4.0
            d.append(base + rng.random())
    dists = np.array(d, dtype=dtype)
    memb = np.zeros(n, dtype=np.int32)
    meds = np.zeros(n, dtype=np.int32)
    ncl = ctypes.c_int(0)
    sfx = "f32" if dtype == np.float32 else "f64"
    rc = getattr(lib, f"odba_cluster_medoids_{sfx}")(n, _vp(dists), _vp(lens), ctypes.c_double(cdist),
                                                      _vp(memb), _vp(meds), ctypes.byref(ncl))
    assert rc == 0
    want_memb, want_meds = CO.cluster_and_medoids(dists, lens, cdist)
    assert np.array_equal(memb, want_memb)
    assert ncl.value == len(want_meds)
    assert list(meds[: ncl.value]) == want_meds
    if cdist == 3.0:
        assert ncl.value >= 3
