"""The no-allocation all-pairs entry point, odba_dtw_pairwise_noalloc_f32.

It serves callers that cannot allocate device memory where they call the
library -- a serving or real-time loop that forbids allocation after start-up,
or a host that owns the whole device memory budget and gives plugins no
allocator -- by keeping its scratch (work counter and swath-edge buffers) in a
fixed array inside the library.  This test calls it through the C ABI twice in
a row and checks each result against the regular entry point
(odba_dtw_pairwise_f32) bit for bit, the tolerance every DTW test here uses.
It also checks that a series longer than the array's limit is refused.
The file name sorts last so that a stop-at-first-failure run has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api, build, _native
    build.build_library()
    return torch, api, _native


def _noalloc(native, ds, out, open_start, open_end, stream):
    return native.lib().odba_dtw_pairwise_noalloc_f32(
        ds.data.data_ptr(), ds.offsets.data_ptr(), ds.lens.data_ptr(), ds.n, ds.max_len,
        open_start, open_end, out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("open_start,open_end", [(0, 0), (0, 1)])
def test_noalloc_matches_regular_entry_point_twice(env, open_start, open_end):
    torch, api, native = env
    rng = np.random.default_rng(4242 + open_end)
    lens = list(rng.integers(2, 3000, size=30)) + [1025, 2049]
    series = [rng.standard_normal(int(L)).astype(np.float32) for L in lens]
    ds = api.DeviceSeries.from_host(series)
    stream = torch.cuda.current_stream()
    want = api.pairwise(ds, open_start, open_end).cpu().numpy()
    npairs = len(want)
    for _ in range(2):  # the second call reuses the array the first one left behind
        out = torch.full((npairs,), float("nan"), dtype=torch.float32, device="cuda")
        rc = _noalloc(native, ds, out, open_start, open_end, stream)
        assert rc == 0, native.lib().odba_last_error()
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_noalloc_rejects_series_beyond_its_limit(env):
    torch, api, native = env
    ds = api.DeviceSeries.from_host([np.ones(8, np.float32), np.ones(9, np.float32)])
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    lib = native.lib()
    rc = lib.odba_dtw_pairwise_noalloc_f32(ds.data.data_ptr(), ds.offsets.data_ptr(),
                                           ds.lens.data_ptr(), 2, 3_000_000, 0, 0,
                                           out.data_ptr(), None)
    assert rc == 1
    assert b"limit" in lib.odba_last_error()
