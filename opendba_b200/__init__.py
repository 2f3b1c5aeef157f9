"""OpenDBA's data-parallel hot path on NVIDIA B200 (sm_100a).

DTW all-vs-all distances and medoid, z-normalisation and the DBA round, as
hand-written CUDA kernels behind a C ABI (include/opendba_b200.h), with the
reference's templated C++ entry points and CLI on top.
"""
from ._native import OdbaError, lib  # noqa: F401

__all__ = ["OdbaError", "lib"]
