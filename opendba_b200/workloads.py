"""Benchmark workloads beyond the medoid pass: many DBA jobs (batched vs the
plain per-job path) and a Poisson request stream through the serving loop
(continuous batching vs plain first-come-first-served).

Seeded synthetic data stands in for nanopore reads: no public suite exists.
Cells are full m x n DTW matrices (medoid pairs, query pairs, and member x
centroid per DBA round), counted the same way for both paths.
"""
from __future__ import annotations

import math
import statistics
import threading
import time

import numpy as np

from . import api, synth


def _logu_int(rng, lo, hi, size=None):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=size)).astype(np.int64)


def _step(rng, L):
    return synth.step_signal(rng, int(L), 90.0, 12.0, 10.0, 2.0).astype(np.float32)


def make_jobs(n_jobs, count_lo, count_hi, len_lo, len_hi, seed):
    """Independent averaging jobs: per job a log-uniform count of series with
    log-uniform lengths (step signals: N(90,12) levels, dwell 10, noise 2)."""
    rng = np.random.default_rng(seed)
    counts = _logu_int(rng, count_lo, count_hi + 1, n_jobs)
    return [synth.step_signals(rng, _logu_int(rng, len_lo, len_hi + 1, int(c)), 90.0, 12.0, 10.0, 2.0)
            for c in counts]


def job_cells(job, rounds, centroid_len):
    lens = np.array([len(s) for s in job], dtype=np.float64)
    tot = lens.sum()
    pair_cells = (tot * tot - (lens * lens).sum()) / 2.0
    return pair_cells + rounds * tot * centroid_len


def run_batched_vs_plain(n_jobs=256, count_lo=8, count_hi=512, len_lo=200, len_hi=20000,
                         open_end=1, seed=synth.SEED_BASE + 3, plain_sample=24):
    """Many DBA jobs (open end, float32): batched vs plain; returns a dict.
    Defaults: 256 jobs of 8-512 series (log-uniform count), lengths
    log-uniform in [200, 20000].  The batched path runs every job; the plain
    path (one job after another, a synchronisation every round) runs a seeded
    sample of ``plain_sample`` jobs, whose results must equal the batched
    ones, and its throughput (cells per second) is measured on that sample."""
    import sys
    jobs = make_jobs(n_jobs, count_lo, count_hi, len_lo, len_hi, seed)
    flags = [2 if open_end else 0] * len(jobs)
    api.dba_jobs(jobs[:2], flags[:2], norm=1, batched=True)   # warm-up (module loading)
    api.dba_jobs(jobs[:2], flags[:2], norm=1, batched=False)
    t0 = time.perf_counter()
    res_b = api.dba_jobs(jobs, flags, norm=1, batched=True)
    tb = time.perf_counter() - t0
    cells = sum(job_cells(j, r["rounds"], len(r["centroid"])) for j, r in zip(jobs, res_b))
    print(f"batched: {len(jobs)} jobs, {cells:.3e} cells in {tb:.1f} s", file=sys.stderr, flush=True)
    rng = np.random.default_rng(seed + 1)
    pick = sorted(rng.choice(len(jobs), size=min(plain_sample, len(jobs)), replace=False).tolist())
    t0 = time.perf_counter()
    res_p = api.dba_jobs([jobs[i] for i in pick], [flags[i] for i in pick], norm=1, batched=False)
    tp = time.perf_counter() - t0
    pcells = sum(job_cells(jobs[i], r["rounds"], len(r["centroid"])) for i, r in zip(pick, res_p))
    print(f"plain: {len(pick)} jobs, {pcells:.3e} cells in {tp:.1f} s", file=sys.stderr, flush=True)
    same = all(res_b[i]["medoid"] == b["medoid"] and res_b[i]["rounds"] == b["rounds"] and
               np.array_equal(res_b[i]["centroid"].view(np.uint32), b["centroid"].view(np.uint32))
               for i, b in zip(pick, res_p))
    bg, pg = cells / tb / 1e9, pcells / tp / 1e9
    return {"workload": f"{len(jobs)} DBA jobs of {count_lo}-{count_hi} series (log-uniform), lengths "
                        f"log-uniform [{len_lo},{len_hi}], open end, float32, z-normalised",
            "cells": cells, "batched_s": tb, "batched_gcups": bg,
            "plain_sample_jobs": len(pick), "plain_sample_cells": pcells, "plain_sample_s": tp,
            "plain_gcups": pg, "speedup": bg / pg, "identical_results_on_sample": bool(same),
            "rounds_mean": float(np.mean([r["rounds"] for r in res_b])),
            "rounds_max": int(max(r["rounds"] for r in res_b))}


def make_requests(n, seed, n_centroids=32, centroid_len=4000, query_frac=0.7,
                  reads_max=64, read_lo=500, read_hi=50000, job_lo=16, job_hi=256,
                  job_len=(500, 2000)):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        if rng.uniform() < query_frac:
            k = int(_logu_int(rng, 1, reads_max + 1))
            reads = [_step(rng, L) for L in _logu_int(rng, read_lo, read_hi + 1, k)]
            reqs.append(("q", reads))
        else:
            k = int(_logu_int(rng, job_lo, job_hi + 1))
            reqs.append(("j", [_step(rng, L) for L in rng.integers(job_len[0], job_len[1] + 1, k)]))
    cents = [_step(rng, centroid_len) for _ in range(n_centroids)]
    return reqs, cents


def _request_cells(kind, data, cents, rounds=0, clen=0):
    if kind == "q":
        return float(sum(len(r) for r in data)) * float(sum(len(c) for c in cents))
    return job_cells(data, rounds, clen)


def run_serving(rate_hz, n_requests=60, seed=0x0DBA0005, budget=32 << 30, detail=False, **kw):
    """Poisson arrivals through the server; returns latency percentiles and
    throughput, plus the plain FCFS path on the same requests."""
    reqs, cents = make_requests(n_requests, seed, **kw)
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0 / rate_hz, size=len(reqs))
    srv = api.Server(np.float32, hbm_budget_bytes=budget)
    ids = [srv.add_centroid(c) for c in cents]
    # warm-up
    w = srv.submit_query([cents[0][:500]], ids[:2])
    srv.wait(w, 300)
    srv.take(w)
    submitted = []
    t_start = time.perf_counter()

    def producer():
        for (kind, data), g in zip(reqs, gaps):
            time.sleep(g)
            rid = srv.submit_query(data, ids) if kind == "q" else srv.submit_job(data)
            submitted.append((rid, kind, data))

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    lats, cells, rounds = [], 0.0, []
    for rid, kind, data in submitted:
        assert srv.wait(rid, 1200) == 1
        r = srv.take(rid)
        lats.append(r["latency_s"])
        rounds.append(r["rounds"])
        cells += _request_cells(kind, data, cents, r["rounds"], len(r["result"]) if kind == "j" else 0)
    wall = time.perf_counter() - t_start
    sstats = srv.stats()
    srv.close()
    # plain: the same requests one after another through the drop-in paths
    t0 = time.perf_counter()
    plain_lat, plain_dur, clock = [], [], 0.0
    arrivals = np.cumsum(gaps)
    for (kind, data), arr in zip(reqs, arrivals):
        s0 = time.perf_counter()
        if kind == "q":
            ds = api.DeviceSeries.from_host(list(data) + cents)
            n = len(data)
            import torch
            tasks = np.zeros(n * len(cents), dtype=[("first", "<u4"), ("second", "<u4"), ("out", "<u8")])
            k = 0
            for i in range(n):
                for c in range(len(cents)):
                    tasks[k] = (i, n + c, k)
                    k += 1
            d_tasks = torch.from_numpy(tasks.view(np.uint8)).cuda()
            out = torch.empty(k, dtype=torch.float32, device="cuda")
            wsz = api._native.lib().odba_dtw_pairwise_workspace_bytes(4, max(len(r) for r in data))
            ws = torch.empty(wsz, dtype=torch.uint8, device="cuda")
            api._native.call("odba_dtw_pairlist_f32", ds.data.data_ptr(), ds.offsets.data_ptr(),
                             ds.lens.data_ptr(), d_tasks.data_ptr(), k, max(len(r) for r in data),
                             out.data_ptr(), ws.data_ptr(), ws.numel(),
                             torch.cuda.current_stream().cuda_stream)
            out.cpu()
        else:
            api.dba_jobs([data], [0], norm=1, batched=False)
        dur = time.perf_counter() - s0
        plain_dur.append(dur)
        clock = max(clock, arr) + dur
        plain_lat.append(clock - arr)
    plain_wall = time.perf_counter() - t0
    pct = lambda v, p: float(np.percentile(np.array(v), p))  # noqa: E731
    out = {"rate_hz": rate_hz, "requests": len(reqs), "cells": cells,
            "served_wall_s": wall, "served_gcups": cells / wall / 1e9,
            "p50_ms": 1e3 * pct(lats, 50), "p99_ms": 1e3 * pct(lats, 99),
            "plain_busy_s": plain_wall, "plain_gcups": cells / plain_wall / 1e9,
            "plain_p50_ms": 1e3 * pct(plain_lat, 50), "plain_p99_ms": 1e3 * pct(plain_lat, 99),
            "server_iterations": sstats["iterations"], "server_busy_s": sstats["busy_s"]}
    if detail:
        out["requests_detail"] = [
            {"kind": k, "n": len(d), "samples": int(sum(len(x) for x in d)), "rounds": rr,
             "served_ms": 1e3 * l, "plain_ms": 1e3 * pd}
            for (k, d), rr, l, pd in zip(reqs, rounds, lats, plain_dur)]
    return out


def run_long(n_series=16, len_lo=1_000_000, len_hi=4_000_000, dtypes=("f32", "f64"), minseg=4,
             seed=0x0DBA0002 + 2, with_round=True, round_open_end=0):
    """Few very long series: the k-segmentation DP on each raw series, then
    all-vs-all DTW (global, z-normalised) in float32 and float64, which the
    planner runs as the swath pipeline.  Device time by CUDA events."""
    import torch
    from . import _native
    rng = np.random.default_rng(seed)
    lens = rng.integers(len_lo, len_hi + 1, size=n_series)
    raw = synth.step_signals(rng, lens, 90.0, 12.0, 8.0, 1.5, np.float32)
    raw.sort(key=len)
    L = np.array([len(s) for s in raw], dtype=np.float64)
    cells = float((L.sum() ** 2 - (L ** 2).sum()) / 2.0)
    out = {"workload": f"{n_series} series, lengths U[{len_lo},{len_hi}], step signals (dwell 8, "
                       f"noise 1.5), global DTW of all {n_series * (n_series - 1) // 2} pairs",
           "samples": int(L.sum()), "cells": cells}
    t0 = time.perf_counter()
    segs = api.segment_host(raw, minseg)
    out["segmentation"] = {"min_segment_length": minseg, "seconds": time.perf_counter() - t0,
                           "segments": int(sum(len(s) for s in segs)),
                           "msamples_per_s": L.sum() / (time.perf_counter() - t0) / 1e6,
                           "api": "odba_segment_host_f32 (host series in, medians out)"}
    lib = _native.lib()
    for name in dtypes:
        dt = np.float32 if name == "f32" else np.float64
        ds = api.DeviceSeries.from_host([s.astype(dt) for s in raw])
        api.znorm_(ds)
        elem = np.dtype(dt).itemsize
        ws = torch.empty(lib.odba_dtw_pairwise_workspace_bytes_n(elem, n_series, ds.max_len),
                         dtype=torch.uint8, device="cuda")
        import ctypes
        plan = ctypes.c_int(0)
        lib.odba_tune_query(elem, ds.max_len, n_series * (n_series - 1) // 2, ws.numel(),
                            ctypes.addressof(plan), None)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        d = api.pairwise(ds, 0, 0, workspace=ws)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        err = int(ws[8:12].cpu().numpy().view(np.uint32)[0])
        dh = d.cpu().numpy()
        out[name] = {"seconds": ms / 1e3, "gcups": cells / ms / 1e6, "plan": plan.value,
                     "workspace_gb": ws.numel() / 1e9, "wait_error": err,
                     "finite": bool(np.isfinite(dh).all()), "checksum": float(dh.astype(np.float64).sum())}
        del ds, ws, d
        torch.cuda.empty_cache()
    if with_round:
        out["dba_round_stripe"] = _long_round(raw, round_open_end)
    return out


def _long_round(raw, open_end=0):
    """One stripe-mode DBA round (float32, global or open end): all series
    aligned to the middle-length one as the centroid (the full 2-bit path
    would need ~sum(len) * len(centroid) / 4 bytes); with an open end the
    longer members are flipped (centroid on the rows)."""
    import torch
    from . import _native
    ds = api.DeviceSeries.from_host(raw)
    api.znorm_(ds)
    mid = len(raw) // 2
    cen = ds.data[int(ds.offsets[mid]):int(ds.offsets[mid]) + len(raw[mid])].clone()
    L = np.array([len(s) for s in raw], dtype=np.float64)
    h = np.ascontiguousarray(ds.host_lens, dtype=np.uint64)
    lib = _native.lib()
    import os
    rows = int(os.environ.get("ODBA_STRIPE_ROWS", "1024"))
    nbytes = lib.odba_dba_round_stripe_workspace_bytes(4, h.ctypes.data, len(raw), len(cen), 0,
                                                       int(open_end), rows)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    mean, counts, delta, _ = api.dba_round(cen, ds, 0, int(open_end), workspace=ws, stripe_rows=rows)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    cells = float(L.sum()) * len(cen)
    full_path_tb = float(L.sum()) * len(cen) / 4 / 1e12
    return {"centroid_len": len(cen), "members": len(raw), "tile_rows": rows or 4096,
            "mode": "open_end" if open_end else "global",
            "seconds": ms / 1e3,
            "forward_cells": cells, "gcups": cells / ms / 1e6, "workspace_gb": nbytes / 1e9,
            "full_path_would_need_tb": full_path_tb, "delta": float(delta),
            "finite_mean": bool(torch.isfinite(mean).all().item())}


def run_round(n_members=400, len_lo=3000, len_hi=8000, seed=synth.SEED_BASE + 6, reps=3):
    """One full-path DBA round (float32, global): n_members z-normalised step
    signals of U[len_lo, len_hi] samples against member 7 as the centroid;
    CUDA-event time per round over ``reps`` rounds after two warm-up rounds."""
    import torch
    rng = np.random.default_rng(seed)
    mem = synth.step_signals(rng, rng.integers(len_lo, len_hi + 1, n_members), 90, 12, 10, 2)
    ds = api.DeviceSeries.from_host(mem)
    api.znorm_(ds)
    c = ds.data[int(ds.offsets[7]):int(ds.offsets[7]) + len(mem[7])].clone()
    for _ in range(2):
        api.dba_round(c, ds, 0, 0)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        api.dba_round(c, ds, 0, 0)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    cells = float(sum(len(m) for m in mem)) * len(c)
    return {"workload": f"one DBA round, {n_members} members U[{len_lo},{len_hi}] vs a {len(c)}-sample "
                        "centroid, global, float32", "round_ms": ms, "cells": cells,
            "gcups": cells / ms / 1e6}
