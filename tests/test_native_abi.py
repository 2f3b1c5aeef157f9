"""The C-ABI library loads and exports every symbol its headers declare (CPU only,
no compute calls)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(inc, fn)) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(odba_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


@pytest.fixture(scope="module")
def native():
    from opendba_b200 import build
    build.build_library()
    return ctypes.CDLL(os.path.join(ROOT, "opendba_b200", "libopendba_b200.so"))


def test_header_declares_entry_points():
    names = _declared_functions()
    assert "odba_dtw_pairwise_f32" in names and "odba_medoid_pass_host_f64" in names
    assert len(names) >= 12


def test_library_exports_every_declared_symbol(native):
    missing = [n for n in _declared_functions() if not hasattr(native, n)]
    assert not missing, missing


def test_binding_table_matches_header():
    from opendba_b200 import _native
    assert set(_native.SIGNATURES) == set(_declared_functions())


def test_status_strings_without_gpu(native):
    native.odba_status_string.restype = ctypes.c_char_p
    native.odba_abi_version.restype = ctypes.c_int
    assert native.odba_abi_version() == 1
    assert native.odba_status_string(0) == b"ok"
    assert native.odba_status_string(4) == b"workspace too small"


def test_tuning_table_set_save_load_without_gpu(native, tmp_path):
    from opendba_b200 import _native
    lib = _native.lib()
    path = str(tmp_path / "tune.txt").encode()
    assert lib.odba_tune_set(4, 21, 6, 3) == 0
    assert lib.odba_tune_set(8, 12, 20, 1) == 0
    assert lib.odba_tune_set(3, 12, 20, 1) == 1          # bad element size
    assert lib.odba_tune_set(4, 12, 20, 9) == 1          # bad plan
    assert lib.odba_tune_save(path) == 0
    lines = [l.split() for l in open(path) if not l.startswith("#")]
    assert ["4", "21", "6", "3"] == lines[0][:4] and ["8", "12", "20", "1"] == lines[1][:4]
    assert lib.odba_tune_set(4, 21, 6, 0) == 0 and lib.odba_tune_set(8, 12, 20, 0) == 0
    assert lib.odba_tune_load(path) == 0
    assert lib.odba_tune_save(path) == 0
    again = [l.split() for l in open(path) if not l.startswith("#")]
    assert again == lines
    bad = tmp_path / "bad.txt"
    bad.write_text("4 21 6\n")
    assert lib.odba_tune_load(str(bad).encode()) == 7
    lib.odba_tune_set(4, 21, 6, 0)
    lib.odba_tune_set(8, 12, 20, 0)


def test_round_band_setting_without_gpu(native):
    lib = native
    assert lib.odba_round_set_bands(9) == 1   # invalid argument
    assert lib.odba_round_set_bands(-1) == 1
    u64 = ctypes.c_uint64
    lens = (u64 * 3)(3000, 5000, 8000)
    auto = lib.odba_dba_round_workspace_bytes(4, lens, 3, 6012, 0, 0)
    try:
        assert lib.odba_round_set_bands(1) == 0
        one = lib.odba_dba_round_workspace_bytes(4, lens, 3, 6012, 0, 0)
        assert lib.odba_round_set_bands(4) == 0
        four = lib.odba_dba_round_workspace_bytes(4, lens, 3, 6012, 0, 0)
    finally:
        assert lib.odba_round_set_bands(0) == 0
    # bands add row buffers; 18 (member, swath) tasks fit one wave of warps
    # and are not banded automatically
    assert one < four and auto == one
    assert lib.odba_dba_round_workspace_bytes(4, lens, 3, 6012, 0, 0) == auto


def test_stripe_workspace_sizes_without_gpu(native):
    # host-only size queries of the stripe-mode round: an open end adds the
    # per-(member, centroid index) extra samples and, for double (512-column
    # swaths), a second move buffer; members longer than the centroid are
    # flipped, so their rows are the centroid's
    f = native.odba_dba_round_stripe_workspace_bytes
    f.restype = ctypes.c_size_t
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                  ctypes.c_int, ctypes.c_int]
    short = (ctypes.c_uint64 * 3)(5000, 11000, 9000)  # all shorter than the centroid
    for elem in (4, 8):
        g = f(elem, short, 3, 12000, 0, 0, 1024)
        o = f(elem, short, 3, 12000, 0, 1, 1024)
        assert g > 0 and o > g
        assert f(elem, short, 3, 12000, 0, 0, 48) == 0  # not a power of two
        assert f(elem, short, 3, 12000, 0, 0, 0) == f(elem, short, 3, 12000, 0, 0, 4096)
    # double's second move buffer: one swath of moves for the longest row count
    extra_f = f(4, short, 3, 12000, 0, 1, 1024) - f(4, short, 3, 12000, 0, 0, 1024)
    extra_d = f(8, short, 3, 12000, 0, 1, 1024) - f(8, short, 3, 12000, 0, 0, 1024)
    assert extra_d > extra_f
    # a member longer than the centroid: with an open end its rows are the
    # centroid's 12000 instead of its own 40000, so the move buffer shrinks
    long = (ctypes.c_uint64 * 2)(5000, 40000)
    assert f(4, long, 2, 12000, 0, 1, 1024) < f(4, long, 2, 12000, 0, 0, 1024)
