"""Benchmark: all-vs-all DTW (the medoid pass) on one or more B200s.

Workload (the metric's configuration): 2000 nanopore-like series, lengths
uniform in [2000, 8000], piecewise-constant levels ~ N(90, 12) pA with
geometric dwells of mean 10 samples plus N(0, 2) noise, z-normalised; global
(unbanded) DTW of all 1,999,000 pairs in float32, then the medoid.  Seeded
synthetic data (seed 0x0DBA0002 + rank) stands in for nanopore reads.

A step is one full medoid pass: every pair's DTW distance plus the medoid
(sums of squares, argmin).  ``value`` is whole-job DTW cell updates per second
(GCUPS) with the z-normalised series already resident in HBM; ``e2e`` is the
same metric through the host-buffer C entry point odba_medoid_pass_host_f32
(pinned host series in, distances/medoid/means/sigmas out, z-normalisation on
the device), copies inside the timed region.

Multi-GPU (torchrun): one medoid pass over all ranks ("strong" scaling, the
job is fixed): every rank holds the same series, computes a contiguous range
of the pair triangle holding ~1/N of the DTW cells
(odba_dtw_pairwise_range_f32), the ranges are exchanged with one NCCL
all-gather of the distance triangle (8 MB), and every rank takes the medoid
of the full triangle.  The step time is the max over ranks.

After the timed region, on one GPU, the line also carries:
  parity          the last timed step's distances against the oracle on the
                  CPU baseline's pair sample (bit for bit), their SHA-256 and
                  the medoid against the reference's own run on this
                  workload (tests/golden/ref/c2_medoid_ref.json), and the
                  device z-normalisation against the oracle's;
  fp64_error      relative error of those sampled distances against the same
                  recurrence evaluated in float64;
  cpu_baseline    the oracle's distance-only C restatement on all host cores;
  reference_gpu   the reference's own GPU code (its sources built for sm_100a)
                  on the first 200 rows of the triangle, distances compared;
  batched_vs_plain, serving   the batched and served forms against the plain
                  per-job path (opendba_b200/workloads.py); --no-extras drops
                  them.

``--impl reference`` times the reference's DTW recurrence restated in C
(oracle/, OpenMP on all host cores, the reference itself has no CPU
implementation) on a bounded random sample of the same workload's pairs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "all-vs-all DTW GCUPS (2000×2–8k, fp32); batched/served vs plain, p50/p99, 1 B200"
N_SERIES, LEN_LO, LEN_HI = 2000, 2000, 8000
SEED = 0x0DBA0002
SMS, FP32_LANES, OPS_PER_CELL = 148, 128, 5
MIN_CPU_CELLS = 1.0e11  # the CPU baseline's smallest sample
SM_MAX_MHZ = 1965.0


def workload(rank: int, n_series: int = N_SERIES):
    from opendba_b200 import synth
    return synth.medoid_workload(n_series, LEN_LO, LEN_HI, SEED + rank), synth


def cells_of(lens) -> float:
    lens = np.asarray(lens, dtype=np.float64)
    tot = lens.sum()
    return float((tot * tot - (lens * lens).sum()) / 2.0)


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.out.flush()

    def summary(self):
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        clocks, reasons, maxc = [], set(), SM_MAX_MHZ
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                clocks.append(float(r[1]))
                maxc = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not clocks:
            return {"sm_mhz": None, "sm_max_mhz": SM_MAX_MHZ, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(clocks), "sm_max_mhz": maxc, "reasons": sorted(reasons),
                "samples": len(clocks)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(series, target_secs: float, seed: int = 7):
    """Times the C restatement (OpenMP, all host threads) on a random pair sample."""
    from oracle import oracle as O
    O.lib()
    n = len(series)
    npairs = n * (n - 1) // 2
    lens = np.array([len(s) for s in series], dtype=np.float64)
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n - 1), np.arange(n - 1, 0, -1))
    starts = np.concatenate([[0], np.cumsum(np.arange(n - 1, 0, -1))])[:-1]
    cols = np.arange(npairs) - np.repeat(starts, np.arange(n - 1, 0, -1)) + rows + 1
    threads = os.cpu_count() or 1
    # calibrate on a small sample, then size the measured sample to ~target_secs
    probe = rng.choice(npairs, size=max(threads, 8), replace=False)
    t0 = time.perf_counter()
    O.pairwise_fast(series, 0, 0, pair_list=probe, threads=threads)
    dt = time.perf_counter() - t0
    rate = float((lens[rows[probe]] * lens[cols[probe]]).sum()) / max(dt, 1e-6)
    per_pair = float((lens[rows] * lens[cols]).mean())
    # at least MIN_CPU_CELLS cells, whatever the calibration says (it runs one
    # pair per thread, so it underestimates the rate of a long sample)
    k = int(max(threads, min(npairs, max(target_secs * rate, MIN_CPU_CELLS) / per_pair)))
    sample = np.sort(rng.choice(npairs, size=k, replace=False))
    cells = float((lens[rows[sample]] * lens[cols[sample]]).sum())
    t0 = time.perf_counter()
    d = O.pairwise_fast(series, 0, 0, pair_list=sample, threads=threads)
    dt = time.perf_counter() - t0
    rec = {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": threads, "kind": "port",
           "sample": f"{k} random pairs of the same workload ({cells:.3e} cells, {dt:.1f} s), "
                     "distance-only C restatement of dtw.hpp:158-239, OpenMP over pairs"}
    return rec, sample, d[sample]


def fp64_error(series, sample, got):
    """Relative error of the float32 distances `got` of the pairs `sample`
    against the FP64 reference (the same recurrence in double, double square
    root), on all host threads."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    ref = O.pairwise_fp64ref(series, 0, 0, pair_list=sample, threads=os.cpu_count() or 1)[sample]
    err = O.rel_error(got, ref)
    err["seconds"] = time.perf_counter() - t0
    err["reference"] = "DTW recurrence of dtw.hpp:158-239 in float64, square root in float64"
    return err


def c2_golden(n_series):
    """The reference's own result on this workload (2000 series only), run
    with the reference's sources built for sm_100a: digest of all distances
    and the medoid (tests/golden/ref/c2_medoid_ref.json)."""
    path = os.path.join(ROOT, "tests", "golden", "ref", "c2_medoid_ref.json")
    if n_series != N_SERIES or not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def reference_gpu(series, ours, rows, device_index):
    """The reference's own all-pairs launch loop (dba.hpp:67-161, compiled
    from its sources for sm_100a by oracle/Makefile into oracle/_ref) on the
    first `rows` rows of the same input, timed by the host clock between two
    device synchronisations; its distances are compared with ours bit for bit.
    A context figure: extrapolated to the whole triangle by cells."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return {"unavailable": "oracle/_ref/ref_harness is not built (built from the reference's "
                               "sources where they are present)"}
    from oracle import oracle as O
    with tempfile.TemporaryDirectory() as d:
        inp, outp = os.path.join(d, "in.odbs"), os.path.join(d, "out.odbs")
        O.write_bundle(inp, series)
        with ClockSampler(device_index) as clk:
            p = subprocess.run([harness, "pairwise", inp, outp, "0", "0", str(rows)],
                               capture_output=True, text=True, timeout=1200)
        if p.returncode != 0:
            return {"unavailable": f"reference harness exited {p.returncode}: {p.stderr[-300:]}"}
        rec = json.loads(p.stdout.strip().splitlines()[-1])
        ref = O.read_bundle(outp)[0]
    n = len(series)
    k = rows * n - rows * (rows + 1) // 2  # pairs of the first `rows` rows
    mism = int(np.count_nonzero(ref[:k].view(np.uint32) != ours[:k].view(np.uint32)))
    total = cells_of([len(s) for s in series])
    return {"value": rec["gcups"], "unit": "GCUPS", "rows": rows, "pairs": k, "cells": rec["cells"],
            "seconds": rec["ms"] / 1e3, "clocks": clk.summary(),
            "full_pass_seconds_extrapolated": total / (rec["gcups"] * 1e9),
            "distance_mismatches_vs_ours": mism,
            "basis": f"the reference's DTWDistance launch loop on the first {rows} rows of the triangle "
                     "(shortest first series against all later ones), host clock between device "
                     "synchronisations; extrapolated to the full triangle by cells"}


def checks_and_baselines(args, series_raw, ds, out, medoid_idx, device_index):
    """After the timed region (1 GPU): parity of the last timed step's
    distances and medoid against the oracle's pair sample and the reference's
    own result on this workload, their error against FP64, the CPU baseline,
    and the reference's GPU code timed on the same input."""
    import hashlib
    from oracle import oracle as O
    res = {}
    normed, _, _ = O.znorm(series_raw)
    ours = out.cpu().numpy()
    flat = np.concatenate(normed)
    dev_flat = ds.data[:len(flat)].cpu().numpy()
    parity = {"znorm_bits_match_oracle": bool(np.array_equal(dev_flat.view(np.uint32),
                                                             flat.view(np.uint32)))}
    golden = c2_golden(args.n_series)
    if golden is not None:
        parity["distances_sha256_match_ref"] = (
            hashlib.sha256(ours.tobytes()).hexdigest() == golden["dist_sha256"])
        parity["medoid_ref"] = golden["medoid"]
        parity["medoid_matches_ref"] = medoid_idx == golden["medoid"]
        parity["ref_source"] = ("the reference's sources built for sm_100a, run on this workload "
                                "(tests/golden/ref/c2_medoid_ref.json)")
    if not args.no_cpu:
        cb, sample, cpu_d = cpu_baseline(normed, args.cpu_secs)
        res["cpu_baseline"] = cb
        parity["pairs_checked_vs_oracle"] = int(len(sample))
        parity["mismatches_vs_oracle"] = int(np.count_nonzero(
            cpu_d.view(np.uint32) != ours[sample].view(np.uint32)))
        sub = sample[:: max(1, len(sample) // 2000)]  # at most ~2000 pairs in float64
        res["fp64_error"] = fp64_error(normed, sub, ours[sub])
    res["parity"] = parity
    if not args.no_ref_gpu:
        res["reference_gpu"] = reference_gpu(normed, ours, args.ref_gpu_rows, device_index)
    return res


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O
    series, _, _ = O.znorm(workload(0)[0])
    per_step = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(series, per_step * 0.3, seed=11)
    vals, secs = [], []
    for i in range(args.steps):
        t0 = time.perf_counter()
        cb = cpu_baseline(series, per_step, seed=100 + i)[0]
        secs.append(time.perf_counter() - t0)
        vals.append(cb["value"])
    v = float(statistics.mean(vals))
    cb["value"] = v
    line = {
        "metric": METRIC, "value": v, "unit": "GCUPS", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded nanopore-like step signals)",
        "config": {"workload": f"medoid all-vs-all: {N_SERIES} series, lengths U[{LEN_LO},{LEN_HI}], "
                               "global DTW, float32, z-normalised",
                   "series": N_SERIES, "len_range": [LEN_LO, LEN_HI], "mode": "global",
                   "sample": "random pairs per step (CPU)"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def extra_results(which):
    from opendba_b200 import workloads
    out = {}
    if which in ("batched", "all"):
        out["batched_vs_plain"] = workloads.run_batched_vs_plain()
    if which in ("serving", "all"):
        out["serving"] = workloads.run_serving()
    if which == "long":
        out["long_pairs"] = workloads.run_long()
    if which == "long_round":
        out["long_pairs"] = workloads.run_long(dtypes=())
    if which == "long_round_open_end":
        out["long_pairs"] = workloads.run_long(dtypes=(), round_open_end=1)
    if which == "round":
        out["dba_round"] = workloads.run_round()
    if which == "long_small":
        out["long_pairs"] = workloads.run_long(len_lo=20_000, len_hi=40_000, with_round=False)
    return out


def run_extra(args, world, rank, local):
    """The batched and served forms against the plain per-job path (1 GPU)."""
    import torch
    torch.cuda.set_device(local)
    if rank != 0:
        return 0
    from opendba_b200 import build, _native
    if not os.path.exists(_native.LIB_PATH):
        build.build_library()
    with ClockSampler(local) as clk:
        res = extra_results(args.workload)
    line = {"metric": METRIC, "workload": args.workload, "n_gpus": 1, "dtype": "f32",
            "data": "synthetic (seeded nanopore-like step signals)", **res,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-secs", type=float, default=30.0,
                    help="CPU baseline sample budget (30 s: about 1e11 cells on 16 host threads)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="end-to-end steps (default: --steps, at most 5)")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the batched-jobs and serving comparisons (about 6 minutes)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="leave out the timing of the reference's own GPU code")
    ap.add_argument("--ref-gpu-rows", type=int, default=200,
                    help="rows of the pair triangle the reference's GPU code is timed on")
    ap.add_argument("--n-series", type=int, default=N_SERIES,
                    help="development only: fewer series than the benchmark configuration")
    ap.add_argument("--workload", default="medoid", choices=["medoid", "batched", "serving", "long", "long_round",
                                                             "long_round_open_end", "long_small", "round",
                             "all"],
                    help="medoid: the metric's configuration, with the batched-jobs and serving "
                         "comparisons unless --no-extras (default; all is the same); batched: many DBA jobs, "
                         "batched vs plain; serving: Poisson request stream, served vs plain; "
                         "long: 16 series of 1M-4M samples, segmentation then all-vs-all f32 and "
                         "f64 and one stripe-mode DBA round (several minutes); long_round: the "
                         "segmentation and the DBA round only (long_round_open_end: that round with "
                         "an open end); round: one full-path DBA round of 400 "
                         "members of 3k-8k samples; long_small: the long workload's all-vs-all "
                         "with 20k-40k samples (a profiling case)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload in ("batched", "serving", "long", "long_round", "long_round_open_end", "long_small",
                         "round"):
        return run_extra(args, world, rank, local)

    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=device)
    from opendba_b200 import api, build, _native
    if not os.path.exists(_native.LIB_PATH):
        build.build_library()
    series_raw, synth = workload(0, args.n_series)  # one job shared by all ranks
    lens = [len(s) for s in series_raw]
    cells = cells_of(lens)
    stream = torch.cuda.current_stream()

    # resident, z-normalised inputs for the device-side value
    ds = api.DeviceSeries.from_host(series_raw)
    api.znorm_(ds)
    ws = api.pairwise_workspace(ds)
    out = torch.empty(len(lens) * (len(lens) - 1) // 2, dtype=torch.float32, device=device)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MiB > L2

    from opendba_b200 import sharding
    ranges = sharding.shard_ranges(lens, world)
    rb, re_ = ranges[rank]

    def step(evk=None):
        if evk is not None:
            evk[0].record(stream)
        if world == 1:
            api.pairwise(ds, 0, 0, out=out, workspace=ws, stream=stream)
        else:
            _native.call("odba_dtw_pairwise_range_f32", ds.data.data_ptr(), ds.offsets.data_ptr(),
                         ds.lens.data_ptr(), ds.n, ds.max_len, 0, 0, rb, re_, out.data_ptr(),
                         ws.data_ptr(), ws.numel(), stream.cuda_stream)
        if evk is not None:
            evk[1].record(stream)
        full = out if world == 1 else sharding.gather_triangle(out, ranges, rank, world)
        return api.medoid(full, ds, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    step_ms, kern_ms = [], []
    medoid_idx = None
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            _, medoid_idx = step((k0, k1))
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            kern_ms.append(k0.elapsed_time(k1))
    clocks = clk.summary()
    barrier(world)
    ms = max_over_ranks(statistics.mean(step_ms), world, device)
    kms = max_over_ranks(statistics.mean(kern_ms), world, device)
    value = cells / (ms * 1e-3) / 1e9

    # end to end through the host-buffer C entry point (pinned host input)
    flat, _, hl = api.pack_host(series_raw)
    pinned = torch.from_numpy(flat).pin_memory()
    flat_p = pinned.numpy()
    npairs = len(lens) * (len(lens) - 1) // 2
    dists_h = torch.empty(npairs, dtype=torch.float32).pin_memory().numpy()
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else min(args.steps, 5)
    dists_pin = torch.from_numpy(dists_h)

    def e2e_step():
        if world == 1:
            return api.medoid_pass_host(None, 0, 0, 1, flat=flat_p, lens=hl, dists_out=dists_h)[1]
        # host series in (pinned), z-norm, this rank's range, all-gather, medoid, distances out
        ds.data[: pinned.numel()].copy_(pinned, non_blocking=True)
        api.znorm_(ds)
        full, med = sharding.medoid_pass_sharded(ds, lens, rank, world, workspace=ws, stream=stream)
        dists_pin.copy_(full, non_blocking=True)
        torch.cuda.synchronize()
        return med

    e2e_step()  # warm-up
    barrier(world)
    e2e_s, med_e2e = [], None
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        med_e2e = e2e_step()
        e2e_s.append(time.perf_counter() - t0)
    e2e_sec = max_over_ranks(statistics.mean(e2e_s), world, device) if e2e_s else float("nan")
    e2e_value = cells / e2e_sec / 1e9
    h2d = flat.nbytes + 2 * 8 * len(lens)
    d2h = npairs * 4 + 4 + 2 * 8 * len(lens)

    f_mhz = clocks["sm_mhz"] or SM_MAX_MHZ
    peak = SMS * FP32_LANES * f_mhz * 1e6 / OPS_PER_CELL / 1e9
    peak_max = SMS * FP32_LANES * SM_MAX_MHZ * 1e6 / OPS_PER_CELL / 1e9
    # the kernel of one rank processes its range: ~cells / world (balanced to 1%)
    achieved = cells / world / (kms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "pairwise_dtw_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")
    hbm_gbs = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            hbm_gbs = json.load(f).get("hbm_gbs")
    except OSError:
        pass

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded nanopore-like step signals)",
            "config": {"workload": f"medoid all-vs-all: {args.n_series} series, lengths U[{LEN_LO},{LEN_HI}], "
                                   "global DTW, float32, z-normalised",
                       "series": args.n_series, "pairs": npairs, "cells": cells,
                       "cells_per_gpu": cells / world, "len_range": [LEN_LO, LEN_HI], "mode": "global",
                       "parallelism": ("pairs dp1" if world == 1 else
                                       f"cell-balanced pair ranges x{world} + NCCL all-gather of the triangle"),
                       "l2": "256 MiB buffer written between timed steps"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "GCUPS",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_basis": f"{SMS} SMs x {FP32_LANES} FP32 lanes x {f_mhz:.0f} MHz "
                                       f"(median sampled) / {OPS_PER_CELL} ops per cell",
                         "frac_at_max_clock": achieved / peak_max,
                         "kernel": "pairwise_kernel<float,32,4>", "kernel_ms": kms,
                         "hbm_peak_gbs_measured": hbm_gbs},
            "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "seconds_per_step": e2e_sec,
                    "api": ("odba_medoid_pass_host_f32 (z-norm + pairwise + medoid, pinned host buffers)"
                            if world == 1 else "pinned host series -> z-norm -> pair range -> all-gather "
                            "-> medoid -> distances to pinned host, on every rank")},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
            "medoid": medoid_idx, "medoid_e2e": med_e2e,
        }
        if world == 1:
            line.update(checks_and_baselines(args, series_raw, ds, out, medoid_idx, local))
        if world == 1 and not args.no_extras:
            line.update(extra_results("all"))
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
