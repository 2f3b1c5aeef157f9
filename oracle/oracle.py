"""ctypes access to the CPU oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  It also reads and writes the "series
bundle" fixture container described in oracle/series_bundle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libodba_oracle.so")

NIL, DIAGONAL, RIGHT, UP, OPEN_RIGHT, NIL_OPEN_RIGHT = 255, 1, 2, 3, 4, 5
MOVE_NAMES = {DIAGONAL: "DIAG", RIGHT: "RIGHT", UP: "UP", OPEN_RIGHT: "OPEN_RIGHT",
              NIL: "NIL", NIL_OPEN_RIGHT: "NIL_OPEN_RIGHT"}

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        for sfx in ("f32", "f64"):
            f = getattr(_lib, f"oracle_dtw_pair_{sfx}")
            f.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, P, P]
            f.restype = ctypes.c_int
            f = getattr(_lib, f"oracle_pairwise_{sfx}")
            f.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P,
                          ctypes.c_int64, ctypes.c_int]
            f.restype = ctypes.c_int
            f = getattr(_lib, f"oracle_pairwise_fast_{sfx}")
            f.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int64,
                          ctypes.c_int]
            f.restype = ctypes.c_int
            f = getattr(_lib, f"oracle_medoid_{sfx}")
            f.argtypes = [P, ctypes.c_int, P, P]
            f.restype = ctypes.c_int
            f = getattr(_lib, f"oracle_dba_update_{sfx}")
            f.argtypes = [P, ctypes.c_size_t, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, P, P, P]
            f.restype = ctypes.c_double
            f = _lib.oracle_set_shortcut_lanes
            f.argtypes = [ctypes.c_int, ctypes.c_int]
            f.restype = None
            f = getattr(_lib, f"oracle_dba_update_stripe_{sfx}")
            f.argtypes = [P, ctypes.c_size_t, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, P, P, P, ctypes.c_int64, P, P]
            f.restype = ctypes.c_double
            f = getattr(_lib, f"oracle_path_triples_{sfx}")
            f.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, P, ctypes.c_int64]
            f.restype = ctypes.c_int64
            f = getattr(_lib, f"oracle_segment_{sfx}")
            f.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]
            f.restype = ctypes.c_int64
            f = getattr(_lib, f"oracle_znorm_{sfx}")
            f.argtypes = [P, P, P, ctypes.c_int, P, P]
            f.restype = ctypes.c_int
        f = _lib.oracle_pairwise_fp64ref
        f.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P,
                      ctypes.c_int64, ctypes.c_int]
        f.restype = ctypes.c_int
    return _lib


def _sfx(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def pack(series: list[np.ndarray], dtype=None):
    """Concatenate a ragged list; returns (flat, offsets, lens) as numpy arrays."""
    dtype = np.dtype(dtype or series[0].dtype)
    lens = np.array([len(s) for s in series], dtype=np.uint64)
    offsets = np.zeros(len(series), dtype=np.uint64)
    if len(series) > 1:
        offsets[1:] = np.cumsum(lens)[:-1]
    flat = np.concatenate([np.asarray(s, dtype=dtype) for s in series]) if series else \
        np.zeros(0, dtype)
    return np.ascontiguousarray(flat), offsets, lens


def dtw_pair(first, second, open_start=0, open_end=0, fma_mode=1, with_path=False):
    first = np.ascontiguousarray(first)
    second = np.ascontiguousarray(second, dtype=first.dtype)
    d = np.zeros(1, dtype=first.dtype)
    path = np.zeros(len(first) * len(second), dtype=np.uint8) if with_path else None
    rc = getattr(lib(), f"oracle_dtw_pair_{_sfx(first.dtype)}")(
        _ptr(first), len(first), _ptr(second), len(second), open_start, open_end, fma_mode,
        _ptr(d), _ptr(path) if with_path else None)
    assert rc == 0
    if with_path:
        return d[0], path.reshape(len(first), len(second))
    return d[0]


def pairwise(series, open_start=0, open_end=0, fma_mode=1, pair_list=None, threads=0):
    flat, offsets, lens = pack(series)
    n = len(series)
    out = np.zeros(n * (n - 1) // 2, dtype=flat.dtype)
    pl = None if pair_list is None else np.ascontiguousarray(pair_list, dtype=np.int64)
    rc = getattr(lib(), f"oracle_pairwise_{_sfx(flat.dtype)}")(
        _ptr(flat), _ptr(offsets), _ptr(lens), n, open_start, open_end, fma_mode, _ptr(out),
        _ptr(pl) if pl is not None else None, 0 if pl is None else len(pl), threads)
    assert rc == 0
    return out


def pairwise_fast(series, open_start=0, open_end=0, pair_list=None, threads=0):
    """Distance-only restatement (the timed CPU baseline); same values as pairwise()."""
    flat, offsets, lens = pack(series)
    n = len(series)
    out = np.zeros(n * (n - 1) // 2, dtype=flat.dtype)
    pl = None if pair_list is None else np.ascontiguousarray(pair_list, dtype=np.int64)
    rc = getattr(lib(), f"oracle_pairwise_fast_{_sfx(flat.dtype)}")(
        _ptr(flat), _ptr(offsets), _ptr(lens), n, open_start, open_end, _ptr(out),
        _ptr(pl) if pl is not None else None, 0 if pl is None else len(pl), threads)
    assert rc == 0
    return out


def pairwise_fp64ref(series, open_start=0, open_end=0, pair_list=None, threads=0, for_f32=None):
    """FP64 reference distances (the same recurrence in double, double square
    root); entries outside pair_list are left 0."""
    if for_f32 is None:
        for_f32 = np.dtype(series[0].dtype) == np.float32
    flat, offsets, lens = pack(series, np.float64)
    n = len(series)
    out = np.zeros(n * (n - 1) // 2, dtype=np.float64)
    pl = None if pair_list is None else np.ascontiguousarray(pair_list, dtype=np.int64)
    rc = lib().oracle_pairwise_fp64ref(
        _ptr(flat), _ptr(offsets), _ptr(lens), n, open_start, open_end, int(bool(for_f32)), _ptr(out),
        _ptr(pl) if pl is not None else None, 0 if pl is None else len(pl), threads)
    assert rc == 0
    return out


def rel_error(got, ref):
    """Relative error of results against FP64 reference values: max, median
    and count (pairs whose reference is 0 compare absolutely)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.where(ref != 0, np.abs(ref), 1.0)
    rel = np.abs(got - ref) / den
    return {"max_rel": float(rel.max()) if rel.size else 0.0,
            "median_rel": float(np.median(rel)) if rel.size else 0.0,
            "pairs": int(rel.size)}


def medoid(dists, lens):
    dists = np.ascontiguousarray(dists)
    lens = np.ascontiguousarray(lens, dtype=np.uint64)
    n = len(lens)
    sos = np.zeros(n, dtype=dists.dtype)
    m = getattr(lib(), f"oracle_medoid_{_sfx(dists.dtype)}")(_ptr(dists), n, _ptr(lens), _ptr(sos))
    return m, sos


def dba_update(centroid, members, open_start=0, open_end=0, fma_mode=1):
    centroid = np.ascontiguousarray(centroid)
    flat, offsets, lens = pack(members, centroid.dtype)
    Lc = len(centroid)
    mean = np.zeros(Lc, dtype=centroid.dtype)
    counts = np.zeros(Lc, dtype=np.uint32)
    sums = np.zeros(Lc, dtype=centroid.dtype)
    delta = getattr(lib(), f"oracle_dba_update_{_sfx(centroid.dtype)}")(
        _ptr(centroid), Lc, _ptr(flat), _ptr(offsets), _ptr(lens), len(members), open_start,
        open_end, fma_mode, _ptr(mean), _ptr(counts), _ptr(sums))
    return mean, counts, sums, delta


# which warp-0 lane's partial minimum the reference's open-end shortcut reads
# (dtw.hpp:97-105): lane 0 (the full minimum) in its float build, lane 16 in
# its double build, pinned by its stripe-mode runs (tests/golden/ref/stripe_*)
SHORTCUT_LANE = {np.dtype(np.float32): 0, np.dtype(np.float64): 16}


def set_shortcut_lanes(lane_f32=0, lane_f64=16):
    """Which lane's partial minimum the open-end shortcut reads (see
    SHORTCUT_LANE); the defaults are the reference's."""
    lib().oracle_set_shortcut_lanes(lane_f32, lane_f64)


def dba_update_stripe(centroid, members, open_start=0, open_end=0, fma_mode=1, lane=None):
    """One DBA round in the reference's stripe mode (dba.hpp:515-763), with the
    open-end rules its stripe re-run applies at the backtrack height.  Returns
    (mean, counts, delta, paths, hazards): paths[k] is member k's (row, column,
    move) cells in walk order, hazards[k] its walk's row-0 stripe exits."""
    centroid = np.ascontiguousarray(centroid)
    if lane is None:
        lane = SHORTCUT_LANE[centroid.dtype]
    flat, offsets, lens = pack(members, centroid.dtype)
    Lc = len(centroid)
    mean = np.zeros(Lc, dtype=centroid.dtype)
    counts = np.zeros(Lc, dtype=np.uint32)
    n = len(members)
    cap = int(sum(Lc + len(x) + 2 for x in members))
    tri = np.zeros(3 * cap, dtype=np.int64)
    tcnt = np.zeros(n, dtype=np.int64)
    hz = np.zeros(n, dtype=np.int64)
    delta = getattr(lib(), f"oracle_dba_update_stripe_{_sfx(centroid.dtype)}")(
        _ptr(centroid), Lc, _ptr(flat), _ptr(offsets), _ptr(lens), n, open_start, open_end,
        fma_mode, lane, _ptr(mean), _ptr(counts), _ptr(tri), cap, _ptr(tcnt), _ptr(hz))
    assert (tcnt >= 0).all()
    paths, o = [], 0
    for k in range(n):
        paths.append(tri[3 * o:3 * (o + tcnt[k])].reshape(-1, 3))
        o += int(tcnt[k])
    return mean, counts, delta, paths, hz


def path_triples(centroid, seq, open_start=0, open_end=0, fma_mode=1):
    centroid = np.ascontiguousarray(centroid)
    seq = np.ascontiguousarray(seq, dtype=centroid.dtype)
    cap = len(centroid) + len(seq) + 2
    tri = np.zeros(3 * cap, dtype=np.int64)
    k = getattr(lib(), f"oracle_path_triples_{_sfx(centroid.dtype)}")(
        _ptr(centroid), len(centroid), _ptr(seq), len(seq), open_start, open_end, fma_mode,
        _ptr(tri), cap)
    assert k >= 0
    return tri[:3 * k].reshape(k, 3)


def member_ranges(centroid, members, open_start=0, open_end=0, fma_mode=1):
    """Per member and centroid index, the first and last member sample index
    that centroid index receives in updateCentroid's walk (dba.hpp:374-423),
    as int32 [n, Lc, 2] ((1, 0) where none): the walk of path_triples, with
    OPEN_RIGHT cells skipped and the start cell added unless NIL_OPEN_RIGHT."""
    Lc = len(centroid)
    out = np.zeros((len(members), Lc, 2), dtype=np.int32)
    out[:, :, 0] = 1
    for k, seq in enumerate(members):
        flip = bool(open_end) and Lc < len(seq)  # dba.hpp:497-501
        tri = path_triples(centroid, seq, open_start, open_end, fma_mode)
        lo = np.full(Lc, np.iinfo(np.int32).max, dtype=np.int64)
        hi = np.full(Lc, -1, dtype=np.int64)
        for i, j, mv in tri[:-1]:
            if mv == OPEN_RIGHT:
                continue
            t, s = (i, j) if flip else (j, i)
            lo[t] = min(lo[t], s)
            hi[t] = max(hi[t], s)
        if tri[-1][2] != NIL_OPEN_RIGHT:
            lo[0] = min(lo[0], 0)
            hi[0] = max(hi[0], 0)
        got = hi >= 0
        out[k, got, 0] = lo[got]
        out[k, got, 1] = hi[got]
    return out


def reduce_ranges(centroid, members, ranges):
    """The ordered centroid update from member ranges: per centroid index the
    member samples added in T, members in order, each member's samples from
    its last index down (the order of the reference's single-thread pile-up,
    dba.hpp:374-423), then sum / count in T and max |old - new| in double of
    the difference taken in T (dba.hpp:817-836).  Returns (mean, counts,
    delta)."""
    centroid = np.asarray(centroid)
    T = centroid.dtype.type
    Lc = len(centroid)
    mean = np.zeros(Lc, dtype=centroid.dtype)
    counts = np.zeros(Lc, dtype=np.uint32)
    delta = 0.0
    with np.errstate(invalid="ignore", divide="ignore"):
        for t in range(Lc):
            acc, cnt = T(0), 0
            for k, seq in enumerate(members):
                lo, hi = int(ranges[k, t, 0]), int(ranges[k, t, 1])
                for i in range(hi, lo - 1, -1):
                    acc = T(acc + seq[i])
                cnt += max(0, hi - lo + 1)
            mean[t] = T(acc / T(cnt))
            counts[t] = cnt
            d = abs(float(T(centroid[t] - mean[t])))
            if d > delta:
                delta = d
    return mean, counts, delta


def znorm(series):
    flat, offsets, lens = pack(series)
    n = len(series)
    means = np.zeros(n)
    sigmas = np.zeros(n)
    getattr(lib(), f"oracle_znorm_{_sfx(flat.dtype)}")(_ptr(flat), _ptr(offsets), _ptr(lens), n,
                                                        _ptr(means), _ptr(sigmas))
    out = [flat[int(o):int(o) + int(L)].copy() for o, L in zip(offsets, lens)]
    return out, means, sigmas


B200_SMEM_OPTIN = 232448  # cudaDevAttrMaxSharedMemoryPerBlockOptin on B200


def segment(series, minseg, prefix_skip=0, smem=B200_SMEM_OPTIN):
    """k-segmentation medians per series (adaptive_segmentation)."""
    flat, offsets, lens = pack(series)
    n = len(series)
    dw = (minseg + 2) // 3
    spb = 256 * dw
    k_max = int((256 + minseg / dw - 1) / (minseg / dw))
    cap = sum(k_max * ((int(L) + spb - 1) // spb) for L in lens) + 1
    out = np.zeros(cap, dtype=flat.dtype)
    out_lens = np.zeros(n, dtype=np.uint64)
    getattr(lib(), f"oracle_segment_{_sfx(flat.dtype)}")(
        _ptr(flat), _ptr(offsets), _ptr(lens), n, minseg, prefix_skip, smem, _ptr(out),
        _ptr(out_lens))
    res, pos = [], 0
    for L in out_lens:
        res.append(out[pos:pos + int(L)].copy())
        pos += int(L)
    return res


# ---- series bundle I/O (layout in oracle/series_bundle.h) ----

def write_bundle(path: str, series: list[np.ndarray], dtype=None) -> None:
    dtype = np.dtype(dtype or (series[0].dtype if series else np.float32))
    with open(path, "wb") as f:
        f.write(b"ODBS")
        f.write(struct.pack("<IQ", dtype.itemsize, len(series)))
        f.write(np.array([len(s) for s in series], dtype="<u8").tobytes())
        for s in series:
            f.write(np.ascontiguousarray(s, dtype=dtype).tobytes())


def read_bundle(path: str) -> list[np.ndarray]:
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:4] == b"ODBS", path
    esize, n = struct.unpack_from("<IQ", raw, 4)
    lens = np.frombuffer(raw, dtype="<u8", count=n, offset=16)
    dtype = np.float64 if esize == 8 else np.float32
    pos = 16 + 8 * n
    out = []
    for L in lens:
        L = int(L)
        out.append(np.frombuffer(raw, dtype=dtype, count=L, offset=pos).copy())
        pos += L * esize
    return out


def perform_dba(series, open_start=0, open_end=0, norm=1, fma_mode=1, max_rounds=250):
    """CPU restatement of performDBA for one cluster (cdist == 1), dba.hpp:863-1189.

    Returns a dict with the sorted order, the medoid index (in sorted order),
    the pair distances, the final centroid (rescaled when norm), the number of
    rounds run and each round's delta."""
    dtype = series[0].dtype
    tmax = np.finfo(dtype).max
    work = []
    for s in series:
        s = np.array(s, dtype=dtype)
        if s[-1] >= np.sqrt(tmax):  # dba.hpp:868-872
            s = s[:-1]
        work.append(s)
    order = sorted(range(len(work)), key=lambda i: len(work[i]))  # stable, dba.hpp:882-883
    work = [work[i] for i in order]
    means = sigmas = None
    if norm:
        work, means, sigmas = znorm(work)
    dists = pairwise(work, open_start, open_end, fma_mode)
    lens = np.array([len(s) for s in work], dtype=np.uint64)
    med, _ = medoid(dists, lens)
    centroid = work[med].copy()
    prev = two_prev = np.zeros_like(centroid)
    deltas = []
    new = centroid
    rounds = 0
    for i in range(max_rounds):
        new, _, _, delta = dba_update(centroid, work, open_start, open_end, fma_mode)
        rounds += 1
        deltas.append(delta)
        if delta == 0:
            break
        if open_start or open_end:
            if i >= 1 and new.tobytes() == two_prev.tobytes():
                break
            if i > 1:
                two_prev = prev.copy()
            if i > 0:
                prev = new.copy()
        centroid = new
    out = new.copy()
    if norm:
        out = (np.float64(means[med]) + out.astype(np.float64) * np.float64(sigmas[med])).astype(dtype)
    return {"order": order, "medoid": med, "dists": dists, "centroid": out, "rounds": rounds,
            "deltas": deltas, "means": means, "sigmas": sigmas}
