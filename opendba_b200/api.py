"""Python host API over the C ABI.

Mirrors the reference's entry points for the hot path (names and argument
meaning of dba.hpp / gpu_utils.hpp): all-vs-all DTW distances and the medoid
(approximateMedoidIndices, dba.hpp:37), z-normalisation (normalizeSequences,
gpu_utils.hpp:133).  Device memory comes from PyTorch tensors; PyTorch is only
the allocator and stream provider here, every computation runs in
libopendba_b200.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native

_SFX = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64"}


def _torch():
    import torch  # noqa: WPS433 (deferred: only device-side helpers need it)
    return torch


def _stream_ptr(stream) -> int | None:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def pack_host(series, dtype=None):
    """Concatenates a ragged list of 1-D arrays: (flat, offsets, lens) numpy arrays."""
    dtype = np.dtype(dtype or np.asarray(series[0]).dtype)
    if dtype not in _SFX:
        raise TypeError("series must be float32 or float64")
    lens = np.array([len(s) for s in series], dtype=np.uint64)
    if np.any(lens == 0):
        raise ValueError("every series needs at least one sample")
    offsets = np.zeros(len(series), dtype=np.uint64)
    if len(series) > 1:
        offsets[1:] = np.cumsum(lens)[:-1]
    flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=dtype) for s in series]))
    return flat, offsets, lens


@dataclass
class DeviceSeries:
    """A ragged set of series resident in device memory (concatenated)."""
    data: "object"      # torch tensor, float32/float64, on cuda
    offsets: "object"   # torch uint64 tensor (device)
    lens: "object"      # torch uint64 tensor (device)
    host_lens: np.ndarray
    dtype: np.dtype

    @property
    def n(self) -> int:
        return len(self.host_lens)

    @property
    def max_len(self) -> int:
        return int(self.host_lens.max()) if self.n else 0

    @classmethod
    def from_host(cls, series, dtype=None, device="cuda") -> "DeviceSeries":
        torch = _torch()
        flat, offsets, lens = pack_host(series, dtype)
        # pad the tail so vector loads past the last sample stay inside the allocation
        padded = np.concatenate([flat, np.zeros(16, dtype=flat.dtype)])
        data = torch.from_numpy(padded).to(device)
        off = torch.from_numpy(offsets.view(np.int64)).to(device)
        ln = torch.from_numpy(lens.view(np.int64)).to(device)
        return cls(data, off, ln, lens, flat.dtype)

    def subset(self, begin: int, end: int) -> "DeviceSeries":
        """Series begin..end-1 as a view sharing this set's device data."""
        return DeviceSeries(self.data, self.offsets[begin:end], self.lens[begin:end],
                            self.host_lens[begin:end], self.dtype)

    def to_host(self) -> list[np.ndarray]:
        flat = self.data.cpu().numpy()
        offs = self.offsets.cpu().numpy().view(np.uint64)
        return [flat[int(o):int(o) + int(L)].copy() for o, L in zip(offs, self.host_lens)]


def pairwise_workspace(ds: DeviceSeries):
    torch = _torch()
    nbytes = _native.lib().odba_dtw_pairwise_workspace_bytes(ds.dtype.itemsize, ds.max_len)
    return torch.empty(nbytes, dtype=torch.uint8, device=ds.data.device)


def pairwise(ds: DeviceSeries, open_start: int = 0, open_end: int = 0, out=None, workspace=None,
             stream=None):
    """All pair distances (upper triangle, reference order) as a device tensor."""
    torch = _torch()
    n = ds.n
    npairs = n * (n - 1) // 2
    if out is None:
        out = torch.empty(max(npairs, 1), dtype=ds.data.dtype, device=ds.data.device)
    if workspace is None:
        workspace = pairwise_workspace(ds)
    _native.call(f"odba_dtw_pairwise_{_SFX[ds.dtype]}", ds.data.data_ptr(), ds.offsets.data_ptr(),
                 ds.lens.data_ptr(), n, ds.max_len, int(open_start), int(open_end), out.data_ptr(),
                 workspace.data_ptr(), workspace.numel(), _stream_ptr(stream))
    return out[:npairs]


def medoid(dists, ds: DeviceSeries, stream=None):
    """(sums of squares tensor, medoid index) for one cluster of ds."""
    torch = _torch()
    sos = torch.empty(ds.n, dtype=ds.data.dtype, device=ds.data.device)
    med = torch.empty(1, dtype=torch.int32, device=ds.data.device)
    _native.call(f"odba_medoid_{_SFX[ds.dtype]}", dists.data_ptr() if dists.numel() else None,
                 ds.lens.data_ptr(), ds.n, sos.data_ptr(), med.data_ptr(), _stream_ptr(stream))
    return sos, int(med.item())


def znorm_(ds: DeviceSeries, stream=None):
    """Z-normalises ds in place; returns (means, sigmas) device tensors (float64)."""
    torch = _torch()
    means = torch.empty(ds.n, dtype=torch.float64, device=ds.data.device)
    sigmas = torch.empty(ds.n, dtype=torch.float64, device=ds.data.device)
    _native.call(f"odba_znorm_{_SFX[ds.dtype]}", ds.data.data_ptr(), ds.offsets.data_ptr(),
                 ds.lens.data_ptr(), ds.n, means.data_ptr(), sigmas.data_ptr(), _stream_ptr(stream))
    return means, sigmas


def medoid_pass_host(series, open_start: int = 0, open_end: int = 0, norm: int = 1,
                     dtype=None, flat=None, lens=None, dists_out=None, stream=None):
    """End-to-end medoid pass through the host-buffer C entry point.

    Either a list of series, or pre-packed ``flat``/``lens`` host arrays (pinned
    or pageable) may be given.  Returns (dists, medoid, means, sigmas)."""
    if flat is None:
        flat, _, lens = pack_host(series, dtype)
    dt = np.dtype(flat.dtype)
    n = len(lens)
    npairs = n * (n - 1) // 2
    if dists_out is None:
        dists_out = np.empty(max(npairs, 1), dtype=dt)
    med = np.zeros(1, dtype=np.int32)
    means = np.zeros(n, dtype=np.float64)
    sigmas = np.zeros(n, dtype=np.float64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _native.call(f"odba_medoid_pass_host_{_SFX[dt]}", vp(flat), vp(np.ascontiguousarray(lens, dtype=np.uint64)),
                 n, int(open_start), int(open_end), int(norm), vp(dists_out), vp(med),
                 vp(means), vp(sigmas), stream)
    return dists_out[:npairs], int(med[0]), means, sigmas


def dba_round(centroid, members: DeviceSeries, open_start: int = 0, open_end: int = 0,
              with_paths: bool = False, workspace=None, stream=None, stripe_rows=None):
    """One DBA round of ``members`` against ``centroid`` (DBAUpdate, dba.hpp:434).

    centroid: device tensor (same dtype as members).  Returns (new_centroid,
    counts, delta, paths) where paths is None or a list of (k, 3) int32 numpy
    arrays (row, column, move) in the order of the reference's path files.
    stripe_rows: None for the full-path round, else the stripe-mode round with
    that many rows per recomputed tile (a power of two; 0 = the default)."""
    torch = _torch()
    Lc = int(centroid.numel())
    dev = members.data.device
    lib = _native.lib()
    h_lens = np.ascontiguousarray(members.host_lens, dtype=np.uint64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    if workspace is None:
        if stripe_rows is None:
            nbytes = lib.odba_dba_round_workspace_bytes(members.dtype.itemsize, vp(h_lens),
                                                        members.n, Lc, int(open_start), int(open_end))
        else:
            nbytes = lib.odba_dba_round_stripe_workspace_bytes(members.dtype.itemsize, vp(h_lens),
                                                               members.n, Lc, int(open_start),
                                                               int(open_end), int(stripe_rows))
        workspace = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    mean = torch.empty(Lc, dtype=members.data.dtype, device=dev)
    counts = torch.empty(Lc, dtype=torch.int32, device=dev)
    delta = torch.empty(1, dtype=torch.float64, device=dev)
    tri = cnt = None
    if with_paths:
        cap = int(h_lens.sum()) + members.n * (Lc + 1)
        tri = torch.empty(3 * cap, dtype=torch.int32, device=dev)
        cnt = torch.empty(members.n, dtype=torch.int64, device=dev)
    mode_args = (int(open_start), int(open_end))
    name = f"odba_dba_round_{_SFX[members.dtype]}"
    if stripe_rows is not None:
        mode_args += (int(stripe_rows),)
        name = f"odba_dba_round_stripe_{_SFX[members.dtype]}"
    _native.call(name, centroid.data_ptr(), Lc,
                 members.data.data_ptr(), members.offsets.data_ptr(), members.lens.data_ptr(),
                 vp(h_lens), members.n, *mode_args, mean.data_ptr(),
                 counts.data_ptr(), delta.data_ptr(), tri.data_ptr() if tri is not None else None,
                 cnt.data_ptr() if cnt is not None else None, workspace.data_ptr(),
                 workspace.numel(), _stream_ptr(stream))
    paths = None
    if with_paths:
        t = tri.cpu().numpy()
        c = cnt.cpu().numpy()
        paths, pos = [], 0
        for k in range(members.n):
            if c[k] < 0:
                raise _native.OdbaError(2, f"backtrack of member {k} failed")
            paths.append(t[3 * pos:3 * (pos + int(c[k]))].reshape(-1, 3))
            pos += int(h_lens[k]) + Lc + 1
    return mean, counts.view(torch.int32), float(delta.item()), paths


def dba_round_ranges(centroid, members: DeviceSeries, open_start: int = 0, open_end: int = 0,
                     workspace=None, stream=None):
    """The first half of a DBA round for a share of the members: path DTW and
    backtrack (odba_dba_round_ranges_*).  Returns an int32 device tensor
    [n, len(centroid), 2]: per member and centroid index the first and last
    member sample index it receives ((1, 0): none)."""
    torch = _torch()
    Lc = int(centroid.numel())
    dev = members.data.device
    h_lens = np.ascontiguousarray(members.host_lens, dtype=np.uint64)
    if members.n == 0:
        return torch.zeros((0, Lc, 2), dtype=torch.int32, device=dev)
    if workspace is None:
        nbytes = _native.lib().odba_dba_round_workspace_bytes(
            members.dtype.itemsize, h_lens.ctypes.data_as(ctypes.c_void_p), members.n, Lc,
            int(open_start), int(open_end))
        workspace = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    ranges = torch.empty((members.n, Lc, 2), dtype=torch.int32, device=dev)
    _native.call(f"odba_dba_round_ranges_{_SFX[members.dtype]}", centroid.data_ptr(), Lc,
                 members.data.data_ptr(), members.offsets.data_ptr(), members.lens.data_ptr(),
                 h_lens.ctypes.data_as(ctypes.c_void_p), members.n, int(open_start), int(open_end),
                 ranges.data_ptr(), workspace.data_ptr(), workspace.numel(), _stream_ptr(stream))
    return ranges


def dba_reduce_ranges(centroid, members: DeviceSeries, ranges, open_start: int = 0,
                      open_end: int = 0, stream=None):
    """The second half: the ordered reducer over every member's ranges
    (odba_dba_reduce_ranges_*).  Returns (new_centroid, counts, delta) as the
    whole round does."""
    torch = _torch()
    Lc = int(centroid.numel())
    dev = members.data.device
    ws = torch.empty(max(_native.lib().odba_dba_reduce_workspace_bytes(members.dtype.itemsize,
                                                                        members.n), 1),
                     dtype=torch.uint8, device=dev)
    mean = torch.empty(Lc, dtype=members.data.dtype, device=dev)
    counts = torch.empty(Lc, dtype=torch.int32, device=dev)
    delta = torch.empty(1, dtype=torch.float64, device=dev)
    ranges = ranges.contiguous()
    _native.call(f"odba_dba_reduce_ranges_{_SFX[members.dtype]}", centroid.data_ptr(), Lc,
                 members.data.data_ptr(), members.offsets.data_ptr(), members.lens.data_ptr(),
                 members.n, int(open_start), int(open_end), ranges.data_ptr(), mean.data_ptr(),
                 counts.data_ptr(), delta.data_ptr(), ws.data_ptr(), ws.numel(), _stream_ptr(stream))
    return mean, counts, float(delta.item())


def perform_dba(series, names, output_prefix: str, open_start: int = 0, open_end: int = 0,
                norm: int = 1, cdist: float = 1.0, algo_mode: int = 3):
    """performDBA<T> (dba.hpp:863) on host series: writes the reference's
    output files under ``output_prefix``.  Ends the process on the reference's
    fatal errors, like the reference does."""
    dt = np.dtype(np.asarray(series[0]).dtype)
    arrs = [np.ascontiguousarray(s, dtype=dt) for s in series]
    n = len(arrs)
    ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
    lens = (ctypes.c_size_t * n)(*[len(a) for a in arrs])
    cnames = [ctypes.create_string_buffer(str(nm).encode()) for nm in names]
    name_ptrs = (ctypes.c_char_p * n)(*[ctypes.addressof(c) for c in cnames])
    _native.call(f"odba_perform_dba_{_SFX[dt]}", ptrs, n, lens, name_ptrs, int(open_start),
                 int(open_end), output_prefix.encode(), int(norm), float(cdist), int(algo_mode))
    return [a for a in arrs]


def setup_and_run(files, output_prefix: str, read_mode: int = 0, open_start: int = 0,
                  open_end: int = 0, min_segment_length: str = "0", norm: int = 1,
                  cdist: float = 1.0, dtype=np.float32, seqprefix_file=None, prefix_start: int = 0,
                  prefix_length: int = 0, is_short: bool = False):
    """setupAndRun<T> (openDBA.cuh:15): read_mode 0 text, 1 binary, 2 TSV."""
    n = len(files)
    bufs = [ctypes.create_string_buffer(f.encode()) for f in files]
    arr = (ctypes.c_char_p * n)(*[ctypes.addressof(b) for b in bufs])
    _native.call("odba_setup_and_run", np.dtype(dtype).itemsize,
                 seqprefix_file.encode() if seqprefix_file else None, arr, n,
                 output_prefix.encode(), int(read_mode), int(open_start), int(open_end),
                 str(min_segment_length).encode(), int(norm), float(cdist), int(prefix_start),
                 int(prefix_length), int(is_short))


def segment_host(series, min_segment_length: int, prefix_skip: int = 0):
    """adaptive_segmentation<T> (segmentation.hpp:340): segment medians per series."""
    flat, _, lens = pack_host(series)
    dt = np.dtype(flat.dtype)
    cap = _native.lib().odba_segment_capacity(lens.ctypes.data_as(ctypes.c_void_p), len(lens),
                                              int(min_segment_length))
    out = np.zeros(max(int(cap), 1), dtype=dt)
    out_lens = np.zeros(len(lens), dtype=np.uint64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _native.call(f"odba_segment_host_{_SFX[dt]}", vp(flat), vp(lens), len(lens),
                 int(min_segment_length), int(prefix_skip), vp(out), vp(out_lens))
    res, pos = [], 0
    for L in out_lens:
        res.append(out[pos:pos + int(L)].copy())
        pos += int(L)
    return res


def dba_jobs(jobs, flags=None, norm: int = 1, batched: bool = True, max_rounds: int = 250,
             dtype=None):
    """Many independent DBA jobs (odba_dba_jobs_*): each job a list of series.

    flags[j]: bit 0 open start, bit 1 open end.  Returns a list of dicts with
    the medoid (index within the job), centroid, rounds and last delta."""
    dtype = np.dtype(dtype or np.asarray(jobs[0][0]).dtype)
    flat_list, lens, jb, je = [], [], [], []
    for job in jobs:
        jb.append(len(lens))
        for s in job:
            a = np.ascontiguousarray(s, dtype=dtype)
            flat_list.append(a)
            lens.append(len(a))
        je.append(len(lens))
    flat = np.ascontiguousarray(np.concatenate(flat_list))
    lens = np.array(lens, dtype=np.uint64)
    jb = np.array(jb, dtype=np.int32)
    je = np.array(je, dtype=np.int32)
    fl = np.array(flags if flags is not None else [0] * len(jobs), dtype=np.int32)
    nj = len(jobs)
    cap = int(sum(max(len(s) for s in job) for job in jobs))
    med = np.zeros(nj, dtype=np.int32)
    coff = np.zeros(nj, dtype=np.uint64)
    cent = np.zeros(max(cap, 1), dtype=dtype)
    rounds = np.zeros(nj, dtype=np.int32)
    deltas = np.zeros(nj, dtype=np.float64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _native.call(f"odba_dba_jobs_{_SFX[dtype]}", vp(flat), vp(lens), vp(jb), vp(je), vp(fl), nj,
                 int(norm), int(max_rounds), int(bool(batched)), vp(med), vp(coff), vp(cent),
                 vp(rounds), vp(deltas), None)
    out = []
    for j, job in enumerate(jobs):
        L = len(job[int(med[j])])
        # truncation of a too-large last sample shortens the medoid by one
        o = int(coff[j])
        nxt = int(coff[j + 1]) if j + 1 < nj else None
        if nxt is not None:
            L = nxt - o
        out.append({"medoid": int(med[j]), "centroid": cent[o:o + L].copy(), "rounds": int(rounds[j]),
                    "delta": float(deltas[j])})
    return out


class Server:
    """Serving loop with continuous batching (odba_server_*)."""

    def __init__(self, dtype=np.float32, hbm_budget_bytes: int = 8 << 30, device: int = 0):
        self.dtype = np.dtype(dtype)
        self._lib = _native.lib()
        self._h = self._lib.odba_server_create(self.dtype.itemsize, int(hbm_budget_bytes), int(device))
        self._keep = {}

    def close(self):
        if self._h:
            self._lib.odba_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_centroid(self, centroid) -> int:
        c = np.ascontiguousarray(centroid, dtype=self.dtype)
        cid = self._lib.odba_server_add_centroid(self._h, c.ctypes.data, len(c))
        if cid < 0:
            raise _native.OdbaError(-cid, "add_centroid")
        return cid

    def submit_query(self, reads, centroid_ids, open_start=0, open_end=0) -> int:
        flat, _, lens = pack_host(reads, self.dtype)
        ids = np.ascontiguousarray(centroid_ids, dtype=np.int32)
        rid = self._lib.odba_server_submit_query(self._h, flat.ctypes.data, lens.ctypes.data,
                                                 len(lens), ids.ctypes.data, len(ids),
                                                 int(open_start) | (int(open_end) << 1))
        if rid < 0:
            raise _native.OdbaError(-rid, "submit_query")
        self._keep[rid] = ("q", len(lens) * len(ids))
        return rid

    def submit_job(self, series, open_start=0, open_end=0, norm=1) -> int:
        flat, _, lens = pack_host(series, self.dtype)
        rid = self._lib.odba_server_submit_job(self._h, flat.ctypes.data, lens.ctypes.data, len(lens),
                                               int(open_start) | (int(open_end) << 1), int(norm))
        if rid < 0:
            raise _native.OdbaError(-rid, "submit_job")
        self._keep[rid] = ("j", int(max(lens)))
        return rid

    def poll(self, rid) -> int:
        return self._lib.odba_server_poll(self._h, rid)

    def wait(self, rid, timeout_s=600.0) -> int:
        return self._lib.odba_server_wait(self._h, rid, float(timeout_s))

    def take(self, rid):
        kind, cap = self._keep.pop(rid)
        out = np.zeros(max(cap, 1), dtype=self.dtype)
        n = ctypes.c_uint64(0)
        med = ctypes.c_int(-1)
        rounds = ctypes.c_int(0)
        lat = ctypes.c_double(0)
        rc = self._lib.odba_server_take(self._h, rid, out.ctypes.data, cap, ctypes.byref(n),
                                        ctypes.byref(med), ctypes.byref(rounds), ctypes.byref(lat))
        _native.check(rc)
        return {"result": out[:n.value].copy(), "medoid": med.value, "rounds": rounds.value,
                "latency_s": lat.value}

    def stats(self):
        it, cells, busy = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_double(0)
        _native.check(self._lib.odba_server_stats(self._h, ctypes.byref(it), ctypes.byref(cells),
                                                  ctypes.byref(busy)))
        return {"iterations": it.value, "cells": cells.value, "busy_s": busy.value}
