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
            "plain_basis": (f"sample rate: a seeded sample of {len(pick)} of the {len(jobs)} jobs run "
                            "one after another through the plain per-job path, cells / seconds on "
                            "that sample"),
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


def _arrival_schedule(n, rate_hz, seed):
    """Poisson arrival offsets (seconds from the first request's slot)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0, size=n)) / rate_hz


def _drive(offsets, submit):
    """Calls submit(k) for every request k at its arrival offset (from a
    producer thread, absolute schedule so the gaps do not drift) and returns
    the perf_counter time of each submission."""
    times = [0.0] * len(offsets)

    def producer():
        t0 = time.perf_counter()
        for k, off in enumerate(offsets):
            delay = t0 + off - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            times[k] = time.perf_counter()
            submit(k)

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    return times


class PlainServing:
    """The plain per-job path as a first-come-first-served server, with the
    same device residency the served path gets: the centroids are uploaded
    once; each query copies only its reads into a preallocated device buffer,
    builds its task list with numpy and runs one pair-list launch
    (odba_dtw_pairlist_f32) on a preallocated workspace; each averaging job
    runs through the plain drop-in path (odba_dba_jobs_f32, one job)."""

    def __init__(self, reqs, cents):
        import torch
        from . import _native
        self.torch, self.native = torch, _native
        nc = len(cents)
        clens = np.array([len(c) for c in cents], dtype=np.uint64)
        self.nc = nc
        read_cap = max([sum(len(r) for r in d) for k, d in reqs if k == "q"] + [1])
        max_first = max([len(r) for k, d in reqs if k == "q" for r in d] + [1])
        self.ctotal = int(clens.sum())
        self.data = torch.zeros(self.ctotal + read_cap + 16, dtype=torch.float32, device="cuda")
        self.data[:self.ctotal].copy_(torch.from_numpy(np.concatenate(cents)))
        self.host = torch.empty(read_cap, dtype=torch.float32).pin_memory()
        self.clens = clens
        self.coffs = np.concatenate([[0], np.cumsum(clens)[:-1]]).astype(np.uint64)
        max_reads = max([len(d) for k, d in reqs if k == "q"] + [1])
        self.out = torch.empty(max_reads * nc, dtype=torch.float32, device="cuda")
        wsz = _native.lib().odba_dtw_pairwise_workspace_bytes(4, max_first)
        self.ws = torch.empty(wsz, dtype=torch.uint8, device="cuda")
        self.stream = torch.cuda.current_stream()

    def query(self, reads):
        torch = self.torch
        k = len(reads)
        rl = np.array([len(r) for r in reads], dtype=np.uint64)
        flat = np.concatenate(reads)
        self.host[:len(flat)].copy_(torch.from_numpy(flat))
        self.data[self.ctotal:self.ctotal + len(flat)].copy_(self.host[:len(flat)], non_blocking=True)
        # series table: centroids 0..nc-1, then the reads (the read is the
        # first series, as in the serving loop)
        offs = np.concatenate([self.coffs, self.ctotal + np.concatenate([[0], np.cumsum(rl)[:-1]])])
        lens = np.concatenate([self.clens, rl])
        tasks = np.empty(k * self.nc, dtype=[("first", "<u4"), ("second", "<u4"), ("out", "<u8")])
        tasks["first"] = np.repeat(np.arange(k, dtype=np.uint32) + self.nc, self.nc)
        tasks["second"] = np.tile(np.arange(self.nc, dtype=np.uint32), k)
        tasks["out"] = np.arange(k * self.nc, dtype=np.uint64)
        d_offs = torch.from_numpy(offs.astype(np.uint64).view(np.int64)).cuda()
        d_lens = torch.from_numpy(lens.astype(np.uint64).view(np.int64)).cuda()
        d_tasks = torch.from_numpy(tasks.view(np.uint8)).cuda()
        self.native.call("odba_dtw_pairlist_f32", self.data.data_ptr(), d_offs.data_ptr(),
                         d_lens.data_ptr(), d_tasks.data_ptr(), k * self.nc, int(rl.max()),
                         self.out.data_ptr(), self.ws.data_ptr(), self.ws.numel(),
                         self.stream.cuda_stream)
        return self.out[:k * self.nc].cpu().numpy()

    def job(self, series):
        r = api.dba_jobs([series], [0], norm=1, batched=False)[0]
        return r["centroid"], r["medoid"], r["rounds"]


def _pct(v, p):
    return float(np.percentile(np.asarray(v, dtype=np.float64), p))


def run_serving(rates=(8.0, 32.0, 128.0, 512.0), n_requests=300, seed=0x0DBA0005,
                budget=32 << 30, detail=False, **kw):
    """Poisson request streams at several arrival rates through the serving
    loop (continuous batching) and through the plain per-job path run as a
    first-come-first-served server (PlainServing), same requests, same
    arrival schedule, both timed by the host clock: latency = completion -
    arrival per request, throughput = cells / (last completion - first
    arrival).  Every served result must equal the plain one bit for bit."""
    import queue

    import torch
    reqs, cents = make_requests(n_requests, seed, **kw)
    srv = api.Server(np.float32, hbm_budget_bytes=budget)
    ids = [srv.add_centroid(c) for c in cents]
    w = srv.submit_query([cents[0][:500]], ids[:2])  # warm-up
    srv.wait(w, 300)
    srv.take(w)
    plain = PlainServing(reqs, cents)
    plain.query([cents[0][:500]])  # warm-up (module loading)
    plain.job([cents[0][:500], cents[1][:600], cents[2][:700]])
    torch.cuda.synchronize()
    results = []
    for rate in rates:
        offsets = _arrival_schedule(len(reqs), rate, seed + 1)
        # served: submit at the arrival times, collect afterwards
        rids = [None] * len(reqs)

        def submit(k):
            kind, data = reqs[k]
            rids[k] = srv.submit_query(data, ids) if kind == "q" else srv.submit_job(data)

        sub_t = _drive(offsets, submit)
        s_lat, s_done, s_res, cells = [], [], [], 0.0
        for k, rid in enumerate(rids):
            assert srv.wait(rid, 1200) == 1
            r = srv.take(rid)
            s_lat.append(r["latency_s"])
            s_done.append(sub_t[k] + r["latency_s"])
            s_res.append(r)
            kind, data = reqs[k]
            cells += _request_cells(kind, data, cents, r["rounds"], len(r["result"]) if kind == "j" else 0)
        s_span = max(s_done) - min(sub_t)
        # plain: a first-come-first-served consumer fed at the same arrival times
        q = queue.Queue()
        arrivals = [0.0] * len(reqs)

        def produce():
            arrivals[:] = _drive(offsets, q.put)

        prod = threading.Thread(target=produce)
        prod.start()
        p_done, same = [0.0] * len(reqs), True
        for _ in range(len(reqs)):
            k = q.get()
            kind, data = reqs[k]
            if kind == "q":
                got = plain.query(data)
                same &= np.array_equal(got.view(np.uint32), s_res[k]["result"].view(np.uint32))
            else:
                cen, med, rounds = plain.job(data)
                same &= (med == s_res[k]["medoid"] and rounds == s_res[k]["rounds"] and
                         np.array_equal(cen.view(np.uint32), s_res[k]["result"].view(np.uint32)))
            p_done[k] = time.perf_counter()
        prod.join()
        p_lat = [p_done[k] - arrivals[k] for k in range(len(reqs))]
        p_span = max(p_done) - min(arrivals)
        rec = {"rate_hz": rate, "requests": len(reqs), "cells": cells,
               "served": {"gcups": cells / s_span / 1e9, "span_s": s_span,
                          "p50_ms": 1e3 * _pct(s_lat, 50), "p99_ms": 1e3 * _pct(s_lat, 99)},
               "plain": {"gcups": cells / p_span / 1e9, "span_s": p_span,
                         "p50_ms": 1e3 * _pct(p_lat, 50), "p99_ms": 1e3 * _pct(p_lat, 99)},
               "identical_results": bool(same)}
        rec["speedup"] = rec["served"]["gcups"] / rec["plain"]["gcups"]
        if detail:
            rec["requests_detail"] = [
                {"kind": kd, "n": len(d), "samples": int(sum(len(x) for x in d)),
                 "served_ms": 1e3 * sl, "plain_ms": 1e3 * pl}
                for (kd, d), sl, pl in zip(reqs, s_lat, p_lat)]
        results.append(rec)
    sstats = srv.stats()
    srv.close()
    return {"workload": f"{len(reqs)} Poisson requests per rate: 70 % read-vs-centroid queries of 1-64 reads "
                        "(lengths log-uniform [500,50000]) against 32 resident centroids of 4000 samples, "
                        "30 % averaging jobs of 16-256 series of 500-2000 samples; float32",
            "latency": "completion - arrival per request (host clock); throughput: cells / "
                       "(last completion - first arrival), the same for both arms",
            "plain": "first-come-first-served: centroids resident, one pair-list launch per query, "
                     "the plain per-job path per averaging job",
            "queries": sum(1 for k, _ in reqs if k == "q"), "jobs": sum(1 for k, _ in reqs if k == "j"),
            "server_iterations": sstats["iterations"], "rates": results}


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
