"""ctypes binding of libopendba_b200.so (the C ABI in include/opendba_b200.h).

The library is built in-tree by ``opendba_b200.build.build_library()``.  There
is no fallback: if the shared library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libopendba_b200.so")

ODBA_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
    4: "workspace too small", 5: "unsupported device", 6: "timed out", 7: "I/O error",
}

_lib = None

P = ctypes.c_void_p
U64 = ctypes.c_uint64
I32 = ctypes.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "odba_abi_version": (I32, []),
    "odba_status_string": (ctypes.c_char_p, [I32]),
    "odba_last_error": (ctypes.c_char_p, []),
    "odba_device_check": (I32, []),
    "odba_dtw_pairwise_workspace_bytes": (ctypes.c_size_t, [I32, U64]),
    "odba_dtw_pairwise_workspace_bytes_n": (ctypes.c_size_t, [I32, I32, U64]),
    "odba_dtw_pairwise_range_f32": (I32, [P, P, P, I32, U64, I32, I32, U64, U64, P, P, ctypes.c_size_t, P]),
    "odba_dtw_pairwise_range_f64": (I32, [P, P, P, I32, U64, I32, I32, U64, U64, P, P, ctypes.c_size_t, P]),
    "odba_complete_linkage": (I32, [I32, P, P, P]),
    "odba_cutree_k": (I32, [I32, P, I32, P]),
    "odba_cutree_cdist": (I32, [I32, P, P, ctypes.c_double, P]),
    "odba_cluster_medoids_f32": (I32, [I32, P, P, ctypes.c_double, P, P, P]),
    "odba_cluster_medoids_f64": (I32, [I32, P, P, ctypes.c_double, P, P, P]),
    "odba_prefix_chop_workspace_bytes": (ctypes.c_size_t, [I32, P, I32, U64]),
    "odba_prefix_chop_f32": (I32, [P, U64, P, P, P, P, I32, P, P, P, ctypes.c_size_t, P]),
    "odba_prefix_chop_f64": (I32, [P, U64, P, P, P, P, I32, P, P, P, ctypes.c_size_t, P]),
    "odba_tune_set": (I32, [I32, I32, I32, I32]),
    "odba_round_set_bands": (I32, [I32]),
    "odba_tune_query": (I32, [I32, U64, U64, ctypes.c_size_t, P, P]),
    "odba_tune_mode": (None, [I32]),
    "odba_tune_flush": (I32, []),
    "odba_tune_save": (I32, [ctypes.c_char_p]),
    "odba_tune_load": (I32, [ctypes.c_char_p]),
    "odba_selftest_wait_timeout": (I32, [U64, P]),
    "odba_dtw_pairwise_f32": (I32, [P, P, P, I32, U64, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_dtw_pairwise_f64": (I32, [P, P, P, I32, U64, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_dtw_pairlist_f32": (I32, [P, P, P, P, U64, U64, P, P, ctypes.c_size_t, P]),
    "odba_dtw_pairlist_f64": (I32, [P, P, P, P, U64, U64, P, P, ctypes.c_size_t, P]),
    "odba_dtw_pairwise_noalloc_f32": (I32, [P, P, P, I32, U64, I32, I32, P, P]),
    "odba_medoid_f32": (I32, [P, P, I32, P, P, P]),
    "odba_medoid_f64": (I32, [P, P, I32, P, P, P]),
    "odba_znorm_f32": (I32, [P, P, P, I32, P, P, P]),
    "odba_znorm_f64": (I32, [P, P, P, I32, P, P, P]),
    "odba_dba_round_workspace_bytes": (ctypes.c_size_t, [I32, P, I32, U64, I32, I32]),
    "odba_dba_round_stripe_workspace_bytes": (ctypes.c_size_t, [I32, P, I32, U64, I32, I32, I32]),
    "odba_dba_round_stripe_f32": (I32, [P, U64, P, P, P, P, I32, I32, I32, I32, P, P, P, P, P, P,
                                        ctypes.c_size_t, P]),
    "odba_dba_round_stripe_f64": (I32, [P, U64, P, P, P, P, I32, I32, I32, I32, P, P, P, P, P, P,
                                        ctypes.c_size_t, P]),
    "odba_dba_round_f32": (I32, [P, U64, P, P, P, P, I32, I32, I32, P, P, P, P, P, P,
                                 ctypes.c_size_t, P]),
    "odba_dba_round_f64": (I32, [P, U64, P, P, P, P, I32, I32, I32, P, P, P, P, P, P,
                                 ctypes.c_size_t, P]),
    "odba_dba_round_ranges_f32": (I32, [P, U64, P, P, P, P, I32, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_dba_round_ranges_f64": (I32, [P, U64, P, P, P, P, I32, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_dba_reduce_workspace_bytes": (ctypes.c_size_t, [I32, I32]),
    "odba_dba_reduce_ranges_f32": (I32, [P, U64, P, P, P, I32, I32, I32, P, P, P, P, P,
                                         ctypes.c_size_t, P]),
    "odba_dba_reduce_ranges_f64": (I32, [P, U64, P, P, P, I32, I32, I32, P, P, P, P, P,
                                         ctypes.c_size_t, P]),
    "odba_dba_batch_workspace_bytes": (ctypes.c_size_t, [I32, P, P, I32, P, P, I32]),
    "odba_dba_batch_round_f32": (I32, [P, P, P, P, P, P, I32, I32, P, P, P, P, P, P, I32, P, P, P, P,
                                       P, P, P, P, P, P, ctypes.c_size_t, P]),
    "odba_dba_batch_round_f64": (I32, [P, P, P, P, P, P, I32, I32, P, P, P, P, P, P, I32, P, P, P, P,
                                       P, P, P, P, P, P, ctypes.c_size_t, P]),
    "odba_segment_capacity": (ctypes.c_size_t, [P, I32, I32]),
    "odba_segment_workspace_bytes": (ctypes.c_size_t, [I32]),
    "odba_segment_blocks_f32": (I32, [P, P, P, P, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_segment_blocks_f64": (I32, [P, P, P, P, I32, I32, P, P, ctypes.c_size_t, P]),
    "odba_perform_dba_f32": (I32, [P, I32, P, P, I32, I32, ctypes.c_char_p, I32, ctypes.c_double,
                                   I32]),
    "odba_perform_dba_f64": (I32, [P, I32, P, P, I32, I32, ctypes.c_char_p, I32, ctypes.c_double,
                                   I32]),
    "odba_setup_and_run": (I32, [I32, ctypes.c_char_p, P, I32, ctypes.c_char_p, I32, I32, I32,
                                 ctypes.c_char_p, I32, ctypes.c_double, I32, I32, I32]),
    "odba_segment_host_f32": (I32, [P, P, I32, I32, I32, P, P]),
    "odba_segment_host_f64": (I32, [P, P, I32, I32, I32, P, P]),
    "odba_dba_jobs_f32": (I32, [P, P, P, P, P, I32, I32, I32, I32, P, P, P, P, P, P]),
    "odba_dba_jobs_f64": (I32, [P, P, P, P, P, I32, I32, I32, I32, P, P, P, P, P, P]),
    "odba_server_create": (P, [I32, ctypes.c_size_t, I32]),
    "odba_server_destroy": (None, [P]),
    "odba_server_add_centroid": (I32, [P, P, U64]),
    "odba_server_submit_query": (ctypes.c_int64, [P, P, P, I32, P, I32, I32]),
    "odba_server_submit_job": (ctypes.c_int64, [P, P, P, I32, I32, I32]),
    "odba_server_poll": (I32, [P, ctypes.c_int64]),
    "odba_server_wait": (I32, [P, ctypes.c_int64, ctypes.c_double]),
    "odba_server_take": (I32, [P, ctypes.c_int64, P, U64, P, P, P, P]),
    "odba_server_stats": (I32, [P, P, P, P]),
    "odba_medoid_pass_host_f32": (I32, [P, P, I32, I32, I32, I32, P, P, P, P, P]),
    "odba_medoid_pass_host_f64": (I32, [P, P, I32, I32, I32, I32, P, P, P, P, P]),
}


class OdbaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> ctypes.CDLL:
    """Loads the native library (once).  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OdbaError(2, f"native library not built: {LIB_PATH} (run opendba_b200.build)")
        _lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def check(status: int) -> None:
    if status != ODBA_OK:
        raise OdbaError(status, lib().odba_last_error().decode(errors="replace"))


def call(name: str, *args) -> int:
    """Calls an entry point that returns an odba_status and raises on failure."""
    check(getattr(lib(), name)(*args))
    return 0
