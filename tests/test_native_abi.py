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
