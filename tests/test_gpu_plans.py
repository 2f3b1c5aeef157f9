"""Launch plans of the pair kernels (one warp per pair, half-width swaths, and
the swath pipeline with many warps per pair) and their autotuner, on a B200.

Every plan must give the reference's distances bit for bit: the plan is pinned
through the tuning table for the key of each case and the result compared with
the reference's own GPU outputs (tests/golden/ref/) or the CPU oracle.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}
PLANS = {"whole": 1, "half": 2, "pipeline": 3}


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api as A
    from opendba_b200 import build
    build.build_library()
    return A


@pytest.fixture
def pin(api):
    from opendba_b200 import _native
    lib = _native.lib()
    keys = []

    def _pin(elem, max_len, npairs, plan):
        key = (elem, int(max_len).bit_length() - 1, int(npairs).bit_length() - 1)
        assert lib.odba_tune_set(*key, plan) == 0
        keys.append(key)

    yield _pin
    for k in keys:
        lib.odba_tune_set(*k, 0)


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def _plan_in_use(elem, max_len, npairs, ws_bytes):
    import ctypes
    from opendba_b200 import _native
    plan = ctypes.c_int(-1)
    rates = (ctypes.c_double * 4)()
    _native.check(_native.lib().odba_tune_query(elem, max_len, npairs, ws_bytes,
                                                ctypes.addressof(plan), ctypes.addressof(rates)))
    return plan.value, list(rates)


@pytest.mark.parametrize("plan", list(PLANS))
@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_every_plan_matches_reference_gpu(api, pin, plan, sfx, mode):
    series = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}_{mode}.dist.odbs"))[0]
    ds = api.DeviceSeries.from_host(series)
    elem = 4 if sfx == "f32" else 8
    npairs = len(series) * (len(series) - 1) // 2
    pin(elem, ds.max_len, npairs, PLANS[plan])
    ws = api.pairwise_workspace(ds)
    assert _plan_in_use(elem, ds.max_len, npairs, ws.numel())[0] == PLANS[plan]
    got = api.pairwise(ds, *MODES[mode], workspace=ws).cpu().numpy()
    bad = np.nonzero(_bits(got) != _bits(ref))[0]
    assert bad.size == 0, f"{plan}: {bad.size} mismatches, first {bad[:5]}"


@pytest.mark.parametrize("plan", list(PLANS))
@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_open_end_shortcut_lanes_every_plan(api, pin, plan, sfx):
    # short-by-long open-end pairs where the reference's shortcut fires: its
    # float build checks the full edge minimum, its double build lane 16's
    # partial one; one-row pairs whose result the reference reads from
    # unwritten shared memory are checked against the oracle instead
    from test_oracle_stripe import undefined_single_row
    series = O.read_bundle(os.path.join(GOLDEN, f"sc_mix_{sfx}.odbs"))
    ref = O.read_bundle(os.path.join(GOLDEN, f"sc_mix_{sfx}_open_end.dist.odbs"))[0]
    ds = api.DeviceSeries.from_host(series)
    elem = 4 if sfx == "f32" else 8
    npairs = len(series) * (len(series) - 1) // 2
    pin(elem, ds.max_len, npairs, PLANS[plan])
    ws = api.pairwise_workspace(ds)
    assert _plan_in_use(elem, ds.max_len, npairs, ws.numel())[0] == PLANS[plan]
    got = api.pairwise(ds, 0, 1, workspace=ws).cpu().numpy()
    want = O.pairwise(series, 0, 1, fma_mode=1)
    p = 0
    for i in range(len(series) - 1):
        for j in range(i + 1, len(series)):
            exp = want[p] if undefined_single_row(len(series[i]), len(series[j]), sfx) else ref[p]
            assert got[p].tobytes() == np.asarray(exp, dtype=got.dtype).tobytes(), (plan, i, j)
            p += 1


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", list(MODES))
def test_pipeline_long_series_vs_oracle(api, pin, dtype, mode):
    # few long pairs: 5 series, 10 pairs, up to 30 swaths per pair
    rng = np.random.default_rng(4321 + list(MODES).index(mode))
    lens = [30001, 17408, 9000, 1, 20480] if mode == "open_start" else [30001, 17408, 9000, 2, 20480]
    series = [np.cumsum(rng.standard_normal(L)).astype(dtype) * 0.1 for L in lens]
    ds = api.DeviceSeries.from_host(series)
    elem = np.dtype(dtype).itemsize
    pin(elem, ds.max_len, 10, PLANS["pipeline"])
    ws = api._torch().empty(_ws_n(elem, 5, ds.max_len), dtype=api._torch().uint8, device="cuda")
    assert _plan_in_use(elem, ds.max_len, 10, ws.numel())[0] == PLANS["pipeline"]
    got = api.pairwise(ds, *MODES[mode], workspace=ws).cpu().numpy()
    want = O.pairwise(series, *MODES[mode], fma_mode=1)
    bad = np.nonzero(_bits(got) != _bits(want))[0]
    assert bad.size == 0, f"{bad.size} mismatches of {len(want)}: got {got[bad]} want {want[bad]}"
    # the error word of the launch stays clear
    assert int(ws[8:12].cpu().numpy().view(np.uint32)[0]) == 0


def _ws_n(elem, n, max_len):
    from opendba_b200 import _native
    return _native.lib().odba_dtw_pairwise_workspace_bytes_n(elem, n, max_len)


def test_default_plan_for_few_long_series_is_the_pipeline(api):
    elem, max_len, npairs = 4, 4_000_000, 120
    ws = _ws_n(elem, 16, max_len)
    plan, _ = _plan_in_use(elem, max_len, npairs, ws)
    assert plan == PLANS["pipeline"]
    # per-pair edge buffers: two per pair, far below one pair of buffers per warp
    from opendba_b200 import _native
    assert ws < _native.lib().odba_dtw_pairwise_workspace_bytes(elem, max_len) / 10
    # many medium pairs stay one warp per pair
    assert _plan_in_use(4, 8000, 1_999_000, 1 << 40)[0] == PLANS["whole"]


def test_pair_list_pipeline_mixed_modes_vs_oracle(api, pin):
    import torch
    from opendba_b200 import _native
    rng = np.random.default_rng(99)
    lens = [12000, 7000, 3000, 5000, 9000, 600]
    series = [rng.standard_normal(L).astype(np.float32) for L in lens]
    ds = api.DeviceSeries.from_host(series)
    pairs = [(0, 1, 0, 0), (1, 0, 0, 1), (2, 4, 1, 0), (4, 3, 1, 1), (5, 0, 0, 1), (3, 3, 0, 0)]
    tasks = np.zeros(len(pairs), dtype=[("first", "<u4"), ("second", "<u4"), ("out", "<u8")])
    for k, (a, b, os_, oe) in enumerate(pairs):
        tasks[k] = (a, b, k | (os_ << 62) | (oe << 63))
    pin(4, ds.max_len, len(pairs), PLANS["pipeline"])
    d_tasks = torch.from_numpy(tasks.view(np.uint8)).cuda()
    out = torch.empty(len(pairs), dtype=torch.float32, device="cuda")
    ws = api.pairwise_workspace(ds)
    _native.call("odba_dtw_pairlist_f32", ds.data.data_ptr(), ds.offsets.data_ptr(),
                 ds.lens.data_ptr(), d_tasks.data_ptr(), len(pairs), ds.max_len, out.data_ptr(),
                 ws.data_ptr(), ws.numel(), None)
    got = out.cpu().numpy()
    want = np.array([O.dtw_pair(series[a], series[b], os_, oe) for a, b, os_, oe in pairs],
                    dtype=np.float32)
    assert np.array_equal(_bits(got), _bits(want)), (got, want)


def test_tuning_mode_measures_each_plan_and_keeps_results(api):
    from opendba_b200 import _native
    lib = _native.lib()
    rng = np.random.default_rng(5)
    series = [rng.standard_normal(int(L)).astype(np.float32) for L in rng.integers(4100, 8100, 12)]
    ds = api.DeviceSeries.from_host(series)
    npairs = 66
    ws = api.pairwise_workspace(ds)
    lb, cb = ds.max_len.bit_length() - 1, npairs.bit_length() - 1
    lib.odba_tune_set(4, lb, cb, 0)
    outs = []
    lib.odba_tune_mode(1)
    try:
        for _ in range(4):
            outs.append(api.pairwise(ds, 0, 0, workspace=ws).cpu().numpy())
        assert lib.odba_tune_flush() == 0
    finally:
        lib.odba_tune_mode(0)
    plan, rates = _plan_in_use(4, ds.max_len, npairs, ws.numel())
    assert all(r > 0 for r in rates[1:]), rates
    assert plan == 1 + int(np.argmax(rates[1:]))
    for o in outs[1:]:
        assert np.array_equal(_bits(o), _bits(outs[0]))
    assert np.array_equal(_bits(outs[0]), _bits(O.pairwise(series, 0, 0, fma_mode=1)))


def test_bounded_wait_runs_out_and_reports(api):
    import time
    from opendba_b200 import _native
    t0 = time.perf_counter()
    rc = _native.lib().odba_selftest_wait_timeout(50_000_000, None)  # 50 ms
    dt = time.perf_counter() - t0
    assert rc == 6, _native.lib().odba_last_error()
    assert 0.04 < dt < 5.0
    # the context is still usable afterwards
    ds = api.DeviceSeries.from_host([np.ones(40, np.float32), np.arange(50, dtype=np.float32)])
    assert np.isfinite(api.pairwise(ds).cpu().numpy()).all()


@pytest.mark.parametrize("plan", ["whole", "pipeline"])
def test_pair_ranges_assemble_to_the_full_triangle(api, pin, plan):
    import torch
    from opendba_b200 import _native, sharding
    rng = np.random.default_rng(17)
    series = sorted([rng.standard_normal(int(L)).astype(np.float32)
                     for L in rng.integers(500, 5000, size=30)], key=len)
    ds = api.DeviceSeries.from_host(series)
    n = len(series)
    npairs = n * (n - 1) // 2
    full = api.pairwise(ds, 0, 1).cpu().numpy()
    ws = api.pairwise_workspace(ds)
    out = torch.full((npairs,), float("nan"), dtype=torch.float32, device="cuda")
    for b, e in sharding.shard_ranges([len(s) for s in series], 3):
        pin(4, ds.max_len, max(e - b, 1), PLANS[plan])
        _native.call("odba_dtw_pairwise_range_f32", ds.data.data_ptr(), ds.offsets.data_ptr(),
                     ds.lens.data_ptr(), n, ds.max_len, 0, 1, b, e, out.data_ptr(), ws.data_ptr(),
                     ws.numel(), None)
    got = out.cpu().numpy()
    assert np.array_equal(_bits(got), _bits(full))
    from opendba_b200 import _native as N
    with pytest.raises(N.OdbaError):
        N.call("odba_dtw_pairwise_range_f32", ds.data.data_ptr(), ds.offsets.data_ptr(),
               ds.lens.data_ptr(), n, ds.max_len, 0, 1, 5, npairs + 1, out.data_ptr(),
               ws.data_ptr(), ws.numel(), None)


def test_sharded_medoid_pass_single_rank(api):
    from opendba_b200 import sharding
    rng = np.random.default_rng(21)
    series = sorted([rng.standard_normal(int(L)).astype(np.float32)
                     for L in rng.integers(300, 2000, size=25)], key=len)
    ds = api.DeviceSeries.from_host(series)
    full, med = sharding.medoid_pass_sharded(ds, [len(s) for s in series], 0, 1)
    want = O.pairwise(series, 0, 0, fma_mode=1)
    assert np.array_equal(_bits(full.cpu().numpy()), _bits(want))
    assert med == O.medoid(want, np.array([len(s) for s in series], dtype=np.uint64))[0]
