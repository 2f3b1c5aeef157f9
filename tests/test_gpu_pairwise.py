"""Parity of the CUDA medoid pass (all-pairs DTW, medoid, z-norm) on a B200.

Bit-exact against (a) the reference's own GPU outputs (tests/golden/ref/) and
(b) the CPU oracle on seeded random cases, through the C ABI.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}


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


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_pairwise_matches_reference_gpu(api, sfx, mode):
    series = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}_{mode}.dist.odbs"))[0]
    ds = api.DeviceSeries.from_host(series)
    got = api.pairwise(ds, *MODES[mode]).cpu().numpy()
    bad = np.nonzero(_bits(got) != _bits(ref))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]} got {got[bad[:5]]} want {ref[bad[:5]]}"


@pytest.mark.parametrize("mode", ["global", "open_end"])
def test_pairwise_plain_dba_workload_matches_reference_gpu(api, mode):
    series = O.read_bundle(os.path.join(GOLDEN, "pw_c1_f32.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"pw_c1_f32_{mode}.dist.odbs"))[0]
    ds = api.DeviceSeries.from_host(series)
    got = api.pairwise(ds, *MODES[mode]).cpu().numpy()
    assert np.array_equal(_bits(got), _bits(ref))
    sos, med = api.medoid(api.pairwise(ds, *MODES[mode]), ds)
    want_med, want_sos = O.medoid(ref, np.array([len(s) for s in series], dtype=np.uint64))
    assert med == want_med
    assert np.array_equal(_bits(sos.cpu().numpy()), _bits(want_sos))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", list(MODES))
def test_pairwise_random_lengths_vs_oracle(api, dtype, mode):
    rng = np.random.default_rng(1234 + list(MODES).index(mode))
    lens = list(rng.integers(1, 2600, size=14)) + [1, 2, 31, 32, 33, 1024, 1025, 2048]
    rng.shuffle(lens)
    series = [rng.standard_normal(int(L)).astype(dtype) for L in lens]
    ds = api.DeviceSeries.from_host(series)
    got = api.pairwise(ds, *MODES[mode]).cpu().numpy()
    want = O.pairwise(series, *MODES[mode], fma_mode=1)
    bad = np.nonzero(_bits(got) != _bits(want))[0]
    assert bad.size == 0, f"{bad.size} mismatches of {len(want)}"


def test_pairwise_two_series_and_ties(api):
    # identical series: every cost path ties; distance must be exactly 0
    x = np.linspace(-1, 1, 1500).astype(np.float32)
    ds = api.DeviceSeries.from_host([x, x.copy(), x[:700]])
    got = api.pairwise(ds, 0, 0).cpu().numpy()
    want = O.pairwise([x, x, x[:700]], 0, 0, fma_mode=1)
    assert got[0] == 0.0
    assert np.array_equal(_bits(got), _bits(want))


@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_znorm_matches_reference_gpu(api, sfx):
    series = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.norm.odbs"))
    ref_m = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.means.odbs"))[0]
    ref_s = O.read_bundle(os.path.join(GOLDEN, f"znorm_{sfx}.sigmas.odbs"))[0]
    ds = api.DeviceSeries.from_host(series)
    means, sigmas = api.znorm_(ds)
    for a, b in zip(ds.to_host(), ref):
        assert np.array_equal(_bits(a), _bits(b))
    assert np.array_equal(means.cpu().numpy(), ref_m)
    assert np.array_equal(sigmas.cpu().numpy(), ref_s)


def test_medoid_pass_host_end_to_end(api):
    rng = np.random.default_rng(77)
    series = [np.cumsum(rng.standard_normal(int(L))).astype(np.float32) + 40
              for L in rng.integers(300, 1800, size=12)]
    dists, med, means, sigmas = api.medoid_pass_host(series, 0, 1, norm=1)
    normed, m_want, s_want = O.znorm(series)
    want = O.pairwise(normed, 0, 1, fma_mode=1)
    want_med, _ = O.medoid(want, np.array([len(s) for s in series], dtype=np.uint64))
    assert np.array_equal(_bits(dists), _bits(want))
    assert med == want_med
    assert np.array_equal(means, m_want) and np.array_equal(sigmas, s_want)


def test_rejects_bad_arguments(api):
    from opendba_b200 import _native
    with pytest.raises(ValueError):
        api.medoid_pass_host([np.zeros(0, np.float32), np.ones(3, np.float32)])
    # the C entry point itself rejects an empty series
    flat = np.ones(3, np.float32)
    lens = np.array([0, 3], dtype=np.uint64)
    with pytest.raises(_native.OdbaError):
        api.medoid_pass_host(None, flat=flat, lens=lens)
    rc = _native.lib().odba_dtw_pairwise_f32(None, None, None, 5, 10, 0, 0, None, None, 0, None)
    assert rc == 1
    # a workspace smaller than required is refused before any launch
    ds = api.DeviceSeries.from_host([np.ones(40, np.float32), np.ones(50, np.float32)])
    import torch
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(_native.OdbaError) as e:
        api.pairwise(ds, workspace=small)
    assert e.value.status == 4
