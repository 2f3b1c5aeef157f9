"""The no-allocation all-pairs entry point, odba_dtw_pairwise_noalloc_f32.

It serves callers that cannot allocate device memory where they call the
library -- a serving or real-time loop that forbids allocation after start-up,
or a host that owns the whole device memory budget and gives plugins no
allocator -- by keeping its scratch (work counter and swath-edge buffers) in a
fixed array inside the library.  The tests call it through the C ABI and check
its results against the regular entry point (odba_dtw_pairwise_f32) bit for
bit, the tolerance every DTW test here uses:
  * two calls in a row (the second reuses what the first left in the array),
    with series long enough that fewer warps fit the array than the regular
    launch runs;
  * a max_len so large that one block of warps fills the array, and the
    largest max_len it accepts;
  * a call, a device reset, and a call again, in a child process (the array's
    address is looked up again in the new context);
and that a max_len one past the limit is refused.
The file name sorts last so that a stop-at-first-failure run has already run
every other test; it also passes when run alone in a fresh process.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# The array holds one block of 4 warps' ping-pong swath edges (8 columns of
# (max_len + 63) // 32 * 32 floats) up to 64 MiB minus its 256-byte header.
LIMIT = 2_097_088


def _blocks_that_fit(max_len):
    stride = (max_len + 63) // 32 * 32
    return ((64 << 20) - 256) // (4 * 2 * stride * 4)


def test_limit_arithmetic():
    assert _blocks_that_fit(LIMIT) == 1
    assert _blocks_that_fit(LIMIT + 1) == 0
    assert _blocks_that_fit(1_500_000) == 1
    assert _blocks_that_fit(9000) < 444  # fewer blocks than a B200's regular launch


def test_rejects_max_len_past_the_limit_without_a_device():
    # the size check comes before any device work, so it needs no GPU
    from opendba_b200 import _native
    lib = _native.lib()
    dummy = ctypes.c_void_p(256)  # never dereferenced: the call is refused first
    rc = lib.odba_dtw_pairwise_noalloc_f32(dummy, dummy, dummy, 2, LIMIT + 1, 0, 0, dummy, None)
    assert rc == 1  # ODBA_ERR_INVALID_ARGUMENT
    assert b"limit" in lib.odba_last_error()


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api, build, _native
    build.build_library()
    return torch, api, _native


def _noalloc(native, ds, out, open_start, open_end, stream, max_len=None):
    return native.lib().odba_dtw_pairwise_noalloc_f32(
        ds.data.data_ptr(), ds.offsets.data_ptr(), ds.lens.data_ptr(), ds.n,
        ds.max_len if max_len is None else max_len, open_start, open_end, out.data_ptr(),
        ctypes.c_void_p(stream.cuda_stream))


def _check(env, series, open_start, open_end, max_len=None, calls=2):
    torch, api, native = env
    ds = api.DeviceSeries.from_host(series)
    stream = torch.cuda.current_stream()
    want = api.pairwise(ds, open_start, open_end).cpu().numpy()
    for _ in range(calls):
        out = torch.full((len(want),), float("nan"), dtype=torch.float32, device="cuda")
        rc = _noalloc(native, ds, out, open_start, open_end, stream, max_len)
        assert rc == 0, native.lib().odba_last_error()
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("open_start,open_end", [(0, 0), (0, 1)])
def test_noalloc_matches_regular_entry_point_twice(env, open_start, open_end):
    rng = np.random.default_rng(4242 + open_end)
    lens = list(rng.integers(2, 9000, size=30)) + [1025, 2049, 8999]
    series = [rng.standard_normal(int(L)).astype(np.float32) for L in lens]
    _check(env, series, open_start, open_end)


@pytest.mark.gpu
@pytest.mark.parametrize("max_len", [1_500_000, LIMIT])
def test_noalloc_one_block_at_large_max_len(env, max_len):
    rng = np.random.default_rng(77)
    series = [rng.standard_normal(int(L)).astype(np.float32) for L in rng.integers(100, 2000, 8)]
    _check(env, series, 0, 0, max_len=max_len)


@pytest.mark.gpu
def test_noalloc_rejects_series_beyond_its_limit(env):
    torch, api, native = env
    ds = api.DeviceSeries.from_host([np.ones(8, np.float32), np.ones(9, np.float32)])
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    lib = native.lib()
    rc = lib.odba_dtw_pairwise_noalloc_f32(ds.data.data_ptr(), ds.offsets.data_ptr(),
                                           ds.lens.data_ptr(), 2, LIMIT + 1, 0, 0,
                                           out.data_ptr(), None)
    assert rc == 1
    assert b"limit" in lib.odba_last_error()


# A child process with its own context: plain CUDA runtime calls (no torch,
# whose allocations a device reset would invalidate), a call, a reset, a call.
_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, ROOT)
from opendba_b200 import _native
lib = _native.lib()
rt = ctypes.CDLL("libcudart.so.12")
rng = np.random.default_rng(5)
series = [rng.standard_normal(int(L)).astype(np.float32) for L in rng.integers(50, 6000, 12)]
lens = np.array([len(s) for s in series], dtype=np.uint64)
offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
flat = np.concatenate(series + [np.zeros(16, np.float32)])
npairs = len(series) * (len(series) - 1) // 2
max_len = int(lens.max())

def dev(nbytes):
    p = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(nbytes)) == 0
    return p

def h2d(p, a):
    assert rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes), 1) == 0

def d2h(a, p):
    assert rt.cudaMemcpy(a.ctypes.data_as(ctypes.c_void_p), p, ctypes.c_size_t(a.nbytes), 2) == 0

def run(noalloc):
    d_s, d_o, d_l = dev(flat.nbytes), dev(offs.nbytes), dev(lens.nbytes)
    d_out = dev(4 * npairs)
    h2d(d_s, flat); h2d(d_o, offs); h2d(d_l, lens)
    if noalloc:
        rc = lib.odba_dtw_pairwise_noalloc_f32(d_s, d_o, d_l, len(series), max_len, 0, 0, d_out, None)
    else:
        ws_bytes = lib.odba_dtw_pairwise_workspace_bytes(4, max_len)
        d_ws = dev(ws_bytes)
        rc = lib.odba_dtw_pairwise_f32(d_s, d_o, d_l, len(series), max_len, 0, 0, d_out, d_ws,
                                       ws_bytes, None)
    assert rc == 0, lib.odba_last_error()
    assert rt.cudaDeviceSynchronize() == 0
    out = np.empty(npairs, np.float32)
    d2h(out, d_out)
    return out

want = run(False)
first = run(True)
assert rt.cudaDeviceReset() == 0
second = run(True)
assert np.array_equal(first.view(np.uint32), want.view(np.uint32)), "before the reset"
assert np.array_equal(second.view(np.uint32), want.view(np.uint32)), "after the reset"
print("ok")
"""


@pytest.mark.gpu
def test_noalloc_call_reset_call_in_a_child_process(env):
    code = "ROOT = %r\n" % ROOT + _RESET_CHILD
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    assert p.stdout.strip().endswith("ok")
