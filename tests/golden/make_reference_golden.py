"""Generate golden fixtures by running the reference's own GPU build.

Test infrastructure.  Runs oracle/_ref/ref_harness (the reference's sources
compiled for sm_100a by oracle/Makefile) on seeded inputs and stores its
outputs under the given output directory (inside the repository).  The
committed copy lives in tests/golden/ref/; tests compare the CUDA path and
the CPU oracle against it.

Run on a B200 box from the repository root:
    python tests/golden/make_reference_golden.py out_dir [--clusters-only | --chop-only |
                                                          --stripe-only | --shortcut-only |
                                                          --configs-only]
"""
from __future__ import annotations

import glob
import gzip
import json
import os
import shutil
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from opendba_b200 import synth  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}
FIXTURES = "tests/golden/ref_fixtures"


OUT = None  # the output directory, written "<out>" in the logs


def _logged(a) -> str:
    """An argument as the log records it: paths under the output directory as
    <out>/..., other paths under the repository relative to its root."""
    a = str(a)
    if OUT and a.startswith(OUT + os.sep):
        return "<out>/" + os.path.relpath(a, OUT)
    if a.startswith(ROOT + os.sep):
        return os.path.relpath(a, ROOT)
    return a


def run(args, log, cwd=None, env=None):
    t0 = time.time()
    p = subprocess.run([HARNESS] + [str(a) for a in args], capture_output=True, text=True, cwd=cwd,
                       env=env)
    log.write(json.dumps({"args": [_logged(a) for a in args], "rc": p.returncode,
                          "secs": round(time.time() - t0, 3), "stdout": p.stdout[-2000:],
                          "stderr": p.stderr[-2000:]}) + "\n")
    log.flush()
    return p


def mix_series(dtype, seed):
    """Lengths that hit the swath edges (1024, 2048), tiny series and odd sizes; unsorted."""
    lens = [2, 3, 7, 33, 100, 511, 1023, 1024, 1025, 1500, 2047, 2048, 2049, 2500, 3100,
            700, 1200, 64, 1030, 2000]
    rng = np.random.default_rng(seed)
    out = []
    for i, L in enumerate(lens):
        if i % 2:
            x = np.cumsum(rng.standard_normal(L))
        else:
            x = synth.step_signal(rng, L, 90.0, 12.0, 10.0, 2.0)
        sd = x.std()
        out.append(((x - x.mean()) / (sd if sd else 1.0)).astype(dtype))
    return out


def paths_to_npz(prefix, dst):
    files = sorted(glob.glob(prefix + ".path*.txt"),
                   key=lambda f: int(f.rsplit(".path", 1)[1].split(".")[0]))
    arrays = {}
    for f in files:
        k = int(f.rsplit(".path", 1)[1].split(".")[0])
        rows = []
        with open(f) as fh:
            fh.readline()
            for line in fh:
                a = line.rstrip("\n").split("\t")
                rows.append((int(a[0]), int(a[2]), a[4]))
        names = {v: k2 for k2, v in O.MOVE_NAMES.items()}
        arrays[f"ij{k}"] = np.array([(r[0], r[1]) for r in rows], dtype=np.int32)
        arrays[f"mv{k}"] = np.array([names.get(r[2], 0) for r in rows], dtype=np.uint8)
    np.savez_compressed(dst, **arrays)


def gz(src, dst):
    with open(src, "rb") as f, gzip.open(dst, "wb", compresslevel=9) as g:
        g.write(f.read())


def family_series(dtype, seed, n_per=(9, 8, 7)):
    """Three families of warped, noisy copies of three random-walk templates."""
    rng = np.random.default_rng(seed)
    out = []
    for f, cnt in enumerate(n_per):
        tmpl = np.cumsum(rng.standard_normal(600)) + 80.0 + 15.0 * f
        for _ in range(cnt):
            L = int(rng.integers(300, 900))
            t = np.sort(rng.random(L)) * (len(tmpl) - 1)
            x = np.interp(t, np.arange(len(tmpl)), tmpl) + rng.normal(0, 0.8, L)
            out.append(x.astype(dtype))
    order = rng.permutation(len(out))
    return [out[i] for i in order]


def chop_inputs(dirname, seed):
    """A leader (step signal, 300 samples) and reads that start with a warped,
    noisy copy of it followed by a random tail; text files as setupAndRun reads."""
    rng = np.random.default_rng(seed)
    leader = synth.step_signal(rng, 300, 90.0, 12.0, 10.0, 2.0)
    paths = []
    os.makedirs(dirname, exist_ok=True)
    for i in range(8):
        L = int(rng.integers(220, 420))
        t = np.sort(rng.random(L)) * (len(leader) - 1)
        head = np.interp(t, np.arange(len(leader)), leader) + rng.normal(0, 1.5, L)
        tail = synth.step_signal(rng, int(rng.integers(400, 1500)), 90.0, 12.0, 10.0, 2.0)
        x = np.concatenate([head, tail])
        p = os.path.join(dirname, f"read{i}.txt")
        with open(p, "w") as f:
            f.write("\n".join("%.4f" % v for v in x) + "\n")
        paths.append(p)
    lp = os.path.join(dirname, "leader.txt")
    with open(lp, "w") as f:
        f.write("\n".join("%.4f" % v for v in leader) + "\n")
    return lp, paths


def chop_cases(out, tmp, log):
    """setupAndRun with a leader file: prefix_chop.txt, then DBA on the tails."""
    d = os.path.join(out, "chop_inputs")
    lp, paths = chop_inputs(d, synth.SEED_BASE + 606)
    for norm in (1, 0):
        pfx = os.path.join(tmp, f"chop_n{norm}")
        env = dict(os.environ, ODBA_HARNESS_SEQPREFIX=lp)
        t0 = time.time()
        # file names relative to the input directory: the series names are the
        # file names up to the first "." (openDBA.cuh:58-59)
        p = subprocess.run([HARNESS, "setupandrun", pfx, "0", "0", str(norm)] +
                           [os.path.basename(x) for x in paths],
                           capture_output=True, text=True, env=env, cwd=d)
        log.write(json.dumps({"args": ["setupandrun", _logged(pfx), 0, 0, norm], "rc": p.returncode,
                              "secs": round(time.time() - t0, 3), "stderr": p.stderr[-2000:]}) + "\n")
        for ext in (".prefix_chop.txt", ".avg.txt", ".pair_dists.txt"):
            if os.path.exists(pfx + ext):
                shutil.copy(pfx + ext, os.path.join(out, f"chop_n{norm}{ext}"))


def cluster_cases(out, tmp, log):
    """performDBA with clustering thresholds other than 1 (dba.hpp:219-343,
    951-962): membership file, per-cluster averages and pair distances."""
    cases = [(np.float32, "f32", "global", 0.3), (np.float32, "f32", "global", 3.0),
             (np.float32, "f32", "global", 0.0), (np.float64, "f64", "open_end", 0.45)]
    for dt, sfx, mode, cdist in cases:
        ser = family_series(dt, synth.SEED_BASE + 505)
        name = f"cluster_{sfx}_{mode}_c{cdist:g}"
        O.write_bundle(os.path.join(out, f"cluster_{sfx}.odbs"), ser)
        pfx = os.path.join(tmp, name)
        os_, oe = MODES[mode]
        run(["performdba", os.path.join(out, f"cluster_{sfx}.odbs"), pfx, os_, oe, 1, cdist], log)
        for ext in (".avg.txt", ".pair_dists.txt", ".cluster_membership.txt"):
            if os.path.exists(pfx + ext):
                shutil.copy(pfx + ext, os.path.join(out, name + ext))


def warped_copy(rng, base, L, noise):
    """base resampled to L samples along a random monotone time warp, plus
    N(0, noise) noise, z-normalised."""
    w = np.cumsum(rng.uniform(0.3, 1.7, L))
    w = (w - w[0]) / (w[-1] - w[0]) * (len(base) - 1)
    x = np.interp(w, np.arange(len(base)), base) + rng.normal(0, noise, L)
    return (x - x.mean()) / x.std()


# stripe-mode sets: seed offset, centroid length, member lengths (shorter and
# longer than the centroid, so both orientations of the open-end flip occur)
STRIPE_SETS = {"a": (606, 2300, [1500, 2100, 2900, 3600, 4700, 5200, 2400, 1900]),
               "b": (607, 1800, [1200, 2500, 3900, 6100, 1790, 2950, 4400, 800]),
               "c": (608, 3100, [2000, 3300, 5000, 7000, 2600, 4100]),
               "d": (616, 2600, [1700, 3000, 4300, 5600, 2200, 3500, 6400, 2500]),
               "e": (704, 2835, [5602, 5527, 1051, 1367, 2651, 3002, 5156, 1361]),
               "f": (713, 3064, [3040, 4863, 1153, 5175, 6223, 2152, 6333, 1267]),
               "g": (708, 2626, [4473, 3479, 2927, 4931, 5622, 3683, 6785, 5564]),
               "h": (719, 3326, [6668, 3906, 3632, 5977, 2595, 3609, 3562, 5240])}


def stripe_inputs(dtype, tag):
    seed, Lc, lens = STRIPE_SETS[tag]
    rng = np.random.default_rng(synth.SEED_BASE + seed)
    base = synth.step_signal(rng, Lc, 90.0, 12.0, 10.0, 2.0).astype(np.float64)
    base = (base - base.mean()) / base.std()
    members = [warped_copy(rng, base, L, 0.3).astype(dtype) for L in lens]
    return base.astype(dtype), members


def stripe_safe(centroid, members, os_, oe):
    """True if no walk of the oracle's stripe restatement leaves a stripe past
    the first on row 0, whichever warp-0 lane the shortcut check reads: there
    the reference's stripe walk reads one byte before its stripe path buffer
    (dba.hpp:403 with j = -1, i = 0)."""
    lanes = range(32) if (oe and not os_) else (0,)
    return all(not O.dba_update_stripe(centroid, members, os_, oe, lane=lane)[4].any()
               for lane in lanes)


def _sha(b: bytes) -> str:
    import hashlib
    return hashlib.sha256(b).hexdigest()


# Every C2_SAMPLE_STRIDE-th pair distance of the medoid configuration is kept
# verbatim (bit patterns) beside the digest of all of them.
C2_SAMPLE_STRIDE = 997


def c2_inputs():
    """The medoid benchmark configuration: 2000 step signals of U[2000, 8000]
    samples (synth.medoid_workload, seed 0x0DBA0002), z-normalised by the
    oracle's restatement of normalizeSequences (float32)."""
    raw = synth.medoid_workload(2000, 2000, 8000, synth.SEED_BASE + 2)
    normed, _, _ = O.znorm(raw)
    return normed


def c2_cases(out, tmp, log):
    """The reference on the medoid benchmark configuration itself (global,
    float32): the full distance triangle from the launch loop of
    approximateMedoidIndices (pairwise mode), then approximateMedoidIndices
    (medoid and pair_dists.txt).  Kept as digests, the medoid, a strided
    sample of distances and the timing in c2_medoid_ref.json."""
    series = c2_inputs()
    inp = os.path.join(tmp, "c2_input.odbs")
    O.write_bundle(inp, series)
    dist_path = os.path.join(tmp, "c2.dist.odbs")
    p = run(["pairwise", inp, dist_path, 0, 0], log)
    timing = json.loads(p.stdout.strip().splitlines()[-1])
    d = O.read_bundle(dist_path)[0]
    pfx = os.path.join(tmp, "c2_medoid")
    t0 = time.time()
    run(["medoid", inp, pfx, 0, 0], log)
    medoid_secs = time.time() - t0
    with open(pfx + ".medoid.txt") as f:
        medoid_ref = int(f.read().split()[0])
    with open(pfx + ".pair_dists.txt", "rb") as f:
        txt_sha = _sha(f.read())
    lens = np.array([len(s) for s in series], dtype=np.uint64)
    med_from_dists, _ = O.medoid(d, lens)
    idx = np.arange(0, len(d), C2_SAMPLE_STRIDE, dtype=np.int64)
    rec = {"config": "2000 series, lengths U[2000,8000], global, float32",
           "input": "synth.medoid_workload(2000, 2000, 8000, 0x0DBA0002) z-normalised by oracle.znorm",
           "input_sha256": _sha(np.concatenate(series).tobytes()),
           "lens_sha256": _sha(lens.tobytes()),
           "pairs": int(len(d)), "dist_sha256": _sha(np.ascontiguousarray(d, np.float32).tobytes()),
           "medoid": medoid_ref, "medoid_from_dists": int(med_from_dists),
           "pair_dists_txt_sha256": txt_sha,
           "sample_stride": C2_SAMPLE_STRIDE,
           "sample_bits": [int(v) for v in d[idx].view(np.uint32)],
           "reference_timing": timing, "reference_medoid_pass_secs": round(medoid_secs, 1)}
    with open(os.path.join(out, "c2_medoid_ref.json"), "w") as f:
        json.dump(rec, f)
        f.write("\n")


def c1_perform_cases(out, tmp, log):
    """performDBA on the plain-DBA configuration (64 Gaussian random walks of
    U[512, 1024] samples, seed 0x0DBA0001, raw values, z-normalisation on,
    global, float32) until it converges: avg.txt, pair_dists.txt and the last
    round's path of every member."""
    ser = synth.random_walks(64, 512, 1024, synth.SEED_BASE + 1)
    src = os.path.join(out, "perform_c1_f32.odbs")
    O.write_bundle(src, ser)
    pfx = os.path.join(tmp, "perform_c1_f32_global")
    run(["performdba", src, pfx, 0, 0, 1], log)
    for ext in (".avg.txt", ".pair_dists.txt"):
        if os.path.exists(pfx + ext):
            shutil.copy(pfx + ext, os.path.join(out, f"perform_c1_f32_global{ext}"))
    paths_to_npz(pfx + ".0", os.path.join(out, "perform_c1_f32_global.paths.npz"))


def path_digest(ij: np.ndarray, mv: np.ndarray) -> str:
    """sha256 of one path listing: (row, column) as int32 pairs, then moves as bytes."""
    return _sha(np.ascontiguousarray(ij, dtype=np.int32).tobytes() +
                np.ascontiguousarray(mv, dtype=np.uint8).tobytes())


def stripe_summary(out):
    """Digests of the stripe-mode outputs (stripe_ref.json): input bundles,
    mean bytes, delta and every member's path, so the fixtures stay small;
    set "a" also keeps its raw outputs for diagnosis."""
    summary = {"sets": {k: list(v) for k, v in STRIPE_SETS.items()}, "inputs": {}, "cases": {}}
    for tag in STRIPE_SETS:
        for sfx in ("f32", "f64"):
            for part in ("members", "centroid"):
                f = os.path.join(out, f"stripe_{tag}_{sfx}_{part}.odbs")
                with open(f, "rb") as fh:
                    summary["inputs"][f"{tag}_{sfx}_{part}"] = _sha(fh.read())
            for mode in MODES:
                name = f"stripe_{tag}_{sfx}_{mode}"
                if not os.path.exists(os.path.join(out, name + ".mean.odbs")):
                    continue
                mean = O.read_bundle(os.path.join(out, name + ".mean.odbs"))[0]
                with open(os.path.join(out, name + ".delta.txt")) as fh:
                    delta = fh.read().strip()
                gp = np.load(os.path.join(out, name + ".paths.npz"))
                paths = []
                k = 0
                while f"ij{k}" in gp:
                    paths.append(path_digest(gp[f"ij{k}"], gp[f"mv{k}"]))
                    k += 1
                summary["cases"][f"{tag}_{sfx}_{mode}"] = {
                    "mean": _sha(mean.tobytes()), "delta": delta, "paths": paths}
    with open(os.path.join(out, "stripe_ref.json"), "w") as fh:
        json.dump(summary, fh, indent=1, sort_keys=True)


def stripe_cases(out, tmp, log):
    """One DBAUpdate round in the reference's stripe mode (dba.hpp:515-763),
    forced by the harness, all four modes, float and double."""
    env = dict(os.environ, ODBA_HARNESS_FORCE_STRIPE="1")
    for tag in STRIPE_SETS:
        for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
            centroid, members = stripe_inputs(dt, tag)
            mfile = os.path.join(out, f"stripe_{tag}_{sfx}_members.odbs")
            cfile = os.path.join(out, f"stripe_{tag}_{sfx}_centroid.odbs")
            O.write_bundle(mfile, members)
            O.write_bundle(cfile, [centroid])
            for mode, (os_, oe) in MODES.items():
                name = f"stripe_{tag}_{sfx}_{mode}"
                if not stripe_safe(centroid, members, os_, oe):
                    log.write(json.dumps({"skipped": name, "why": "row-0 stripe exit"}) + "\n")
                    continue
                pfx = os.path.join(tmp, name)
                run(["dbaupdate", mfile, cfile, pfx, os_, oe], log, env=env)
                for ext in (".mean.odbs", ".delta.txt"):
                    if os.path.exists(pfx + ext):
                        shutil.copy(pfx + ext, os.path.join(out, name + ext))
                paths_to_npz(pfx, os.path.join(out, name + ".paths.npz"))


def shortcut_mix_series(dtype):
    """Lengths around and past 512 rows and a single sample, so that the
    open-end shortcut (dtw.hpp:74-129) is checked on short-by-long pairs."""
    rng = np.random.default_rng(5)
    lens = [1, 2, 600, 700, 900, 1100, 1500, 530, 3000, 4100, 2600, 5200, 800, 1700]
    out = []
    for i, L in enumerate(lens):
        x = synth.step_signal(rng, L, 90.0, 12.0, 10.0, 2.0) if i % 2 else np.cumsum(rng.standard_normal(L))
        sd = x.std()
        out.append(((x - x.mean()) / (sd if sd else 1.0)).astype(dtype))
    return out


# a short centroid (629 rows after the open-end flip) against longer members
SHORTCUT_DBA_SET = (800, 629, [4871, 4272, 660, 6390, 1776, 2009, 1535, 2535])


def shortcut_cases(out, tmp, log):
    """Open-end pair distances and one full-path DBA round where the
    shortcut's partial minimum (which lane of warp 0 the check reads,
    dtw.hpp:97-105) changes the result."""
    for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
        mix = shortcut_mix_series(dt)
        O.write_bundle(os.path.join(out, f"sc_mix_{sfx}.odbs"), mix)
        run(["pairwise", os.path.join(out, f"sc_mix_{sfx}.odbs"),
             os.path.join(out, f"sc_mix_{sfx}_open_end.dist.odbs"), 0, 1], log)
        seed, Lc, lens = SHORTCUT_DBA_SET
        STRIPE_SETS["sc"] = SHORTCUT_DBA_SET
        centroid, members = stripe_inputs(dt, "sc")
        del STRIPE_SETS["sc"]
        mfile = os.path.join(out, f"sc_dba_{sfx}_members.odbs")
        cfile = os.path.join(out, f"sc_dba_{sfx}_centroid.odbs")
        O.write_bundle(mfile, members)
        O.write_bundle(cfile, [centroid])
        pfx = os.path.join(tmp, f"sc_dba_{sfx}_open_end")
        run(["dbaupdate", mfile, cfile, pfx, 0, 1], log)
        for ext in (".mean.odbs", ".delta.txt"):
            if os.path.exists(pfx + ext):
                shutil.copy(pfx + ext, os.path.join(out, f"sc_dba_{sfx}_open_end{ext}"))
        paths_to_npz(pfx, os.path.join(out, f"sc_dba_{sfx}_open_end.paths.npz"))


def main():
    if len(sys.argv) < 2 or sys.argv[1].startswith("--"):
        sys.exit("usage: make_reference_golden.py out_dir [--clusters-only | --chop-only | "
                 "--stripe-only | --shortcut-only | --configs-only | --timing]")
    global OUT
    out = os.path.abspath(sys.argv[1])
    OUT = out
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(out, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    if "--chop-only" in sys.argv:
        with open(os.path.join(out, "harness_log_chop.jsonl"), "w") as log:
            chop_cases(out, tmp, log)
        shutil.rmtree(tmp, ignore_errors=True)
        print("prefix chop golden written to", out)
        return
    if "--stripe-only" in sys.argv:
        with open(os.path.join(out, "harness_log_stripe.jsonl"), "w") as log:
            stripe_cases(out, tmp, log)
        stripe_summary(out)
        shutil.rmtree(tmp, ignore_errors=True)
        print("stripe golden written to", out)
        return
    if "--shortcut-only" in sys.argv:
        with open(os.path.join(out, "harness_log_shortcut.jsonl"), "w") as log:
            shortcut_cases(out, tmp, log)
        shutil.rmtree(tmp, ignore_errors=True)
        print("shortcut golden written to", out)
        return
    if "--configs-only" in sys.argv:
        with open(os.path.join(out, "harness_log_configs.jsonl"), "w") as log:
            c1_perform_cases(out, tmp, log)
            c2_cases(out, tmp, log)
        shutil.rmtree(tmp, ignore_errors=True)
        print("benchmark-configuration golden written to", out)
        return
    if "--clusters-only" in sys.argv:
        with open(os.path.join(out, "harness_log_clusters.jsonl"), "w") as log:
            cluster_cases(out, tmp, log)
        shutil.rmtree(tmp, ignore_errors=True)
        print("cluster golden written to", out)
        return
    log = open(os.path.join(out, "harness_log.jsonl"), "w")
    meta = {"harness": "oracle/_ref/ref_harness", "modes": MODES}

    # 1. pairwise distances, all modes, float and double, edge-case lengths
    for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
        mix = mix_series(dt, synth.SEED_BASE + 101)
        O.write_bundle(os.path.join(out, f"pw_mix_{sfx}.odbs"), mix)
        for mode, (os_, oe) in MODES.items():
            run(["pairwise", os.path.join(out, f"pw_mix_{sfx}.odbs"),
                 os.path.join(out, f"pw_mix_{sfx}_{mode}.dist.odbs"), os_, oe], log)

    # 2. plain DBA workload: 64 z-normalised random walks, lengths 512..1024, sorted
    c1 = synth.znorm_host(synth.random_walks(64, 512, 1024, synth.SEED_BASE + 1))
    c1 = sorted(c1, key=len)
    O.write_bundle(os.path.join(out, "pw_c1_f32.odbs"), c1)
    for mode in ("global", "open_end"):
        os_, oe = MODES[mode]
        run(["pairwise", os.path.join(out, "pw_c1_f32.odbs"),
             os.path.join(out, f"pw_c1_f32_{mode}.dist.odbs"), os_, oe], log)
    # approximateMedoidIndices itself: pair_dists.txt format and the medoid
    run(["medoid", os.path.join(out, "pw_c1_f32.odbs"), os.path.join(out, "medoid_c1_f32_global"), 0, 0], log)

    # 3. one DBA round, all modes, float and double (path moves as npz, two raw path files)
    for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
        rng = np.random.default_rng(synth.SEED_BASE + 202)
        lens = [200, 450, 900, 1030, 1300, 1800, 2100, 640]
        members = []
        for L in lens:
            x = synth.step_signal(rng, L, 90.0, 12.0, 10.0, 2.0)
            members.append(((x - x.mean()) / x.std()).astype(dt))
        c = synth.step_signal(rng, 1100, 90.0, 12.0, 10.0, 2.0)
        centroid = ((c - c.mean()) / c.std()).astype(dt)
        O.write_bundle(os.path.join(out, f"dba_{sfx}_members.odbs"), members)
        O.write_bundle(os.path.join(out, f"dba_{sfx}_centroid.odbs"), [centroid])
        for mode, (os_, oe) in MODES.items():
            pfx = os.path.join(tmp, f"dba_{sfx}_{mode}")
            run(["dbaupdate", os.path.join(out, f"dba_{sfx}_members.odbs"),
                 os.path.join(out, f"dba_{sfx}_centroid.odbs"), pfx, os_, oe], log)
            for ext in (".mean.odbs", ".delta.txt"):
                if os.path.exists(pfx + ext):
                    shutil.copy(pfx + ext, os.path.join(out, f"dba_{sfx}_{mode}{ext}"))
            paths_to_npz(pfx, os.path.join(out, f"dba_{sfx}_{mode}.paths.npz"))
            if sfx == "f32" and mode in ("global", "open_end"):
                for k in (0, 5):
                    src = f"{pfx}.path{k}.txt"
                    if os.path.exists(src):
                        gz(src, os.path.join(out, f"dba_{sfx}_{mode}.path{k}.txt.gz"))

    # 4. z-normalisation
    for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
        rng = np.random.default_rng(synth.SEED_BASE + 303)
        zs = [synth.step_signal(rng, L, 90.0, 12.0, 10.0, 2.0).astype(dt)
              for L in (5, 100, 1023, 1024, 1025, 3000, 10000)]
        O.write_bundle(os.path.join(out, f"znorm_{sfx}.odbs"), zs)
        run(["znorm", os.path.join(out, f"znorm_{sfx}.odbs"), os.path.join(out, f"znorm_{sfx}")], log)

    # 5. performDBA end to end (z-norm on), float global/open_end and double global
    for dt, sfx, mode in ((np.float32, "f32", "global"), (np.float32, "f32", "open_end"),
                          (np.float64, "f64", "global")):
        rng = np.random.default_rng(synth.SEED_BASE + 404)
        ser = [(np.cumsum(rng.standard_normal(int(L))) + 50.0).astype(dt)
               for L in rng.integers(100, 1300, size=10)]
        O.write_bundle(os.path.join(out, f"perform_{sfx}_{mode}.odbs"), ser)
        pfx = os.path.join(tmp, f"perform_{sfx}_{mode}")
        os_, oe = MODES[mode]
        run(["performdba", os.path.join(out, f"perform_{sfx}_{mode}.odbs"), pfx, os_, oe, 1], log)
        for ext in (".avg.txt", ".pair_dists.txt"):
            if os.path.exists(pfx + ext):
                shutil.copy(pfx + ext, os.path.join(out, f"perform_{sfx}_{mode}{ext}"))
        paths_to_npz(pfx + ".0", os.path.join(out, f"perform_{sfx}_{mode}.paths.npz"))

    # 6. the reference's own test sections through setupAndRun<float> (text inputs)
    sections = {
        "gsd": (0, 0, ["random_short1.txt", "random_short1.txt"]),
        "gdd": (0, 0, ["random_short1.txt", "random_short2.txt"]),
        "gtd": (0, 0, ["random_short1.txt", "random_short2.txt", "random_short3.txt"]),
        "gdtd": (0, 1, ["random_short1.txt", "random_trun_short2.txt"]),
        "gld": (0, 0, ["random_large0.txt", "random_large1.txt"]),
    }
    for name, (os_, oe, files) in sections.items():
        # a prefix relative to the repository root: the reference names its
        # outputs after the prefix up to its first '.'
        pfx = os.path.relpath(os.path.join(tmp, f"sar_{name}"), ROOT)
        args = ["setupandrun", pfx, os_, oe, 0] + [f"{FIXTURES}/{f}" for f in files]
        run(args, log, cwd=ROOT)
        for ext in (".avg.txt", ".pair_dists.txt"):
            src = os.path.join(ROOT, pfx + ext)
            if os.path.exists(src):
                shutil.copy(src, os.path.join(out, f"sar_{name}{ext}"))

    # 7. k-segmentation
    for dt, sfx in ((np.float32, "f32"), (np.float64, "f64")):
        rng = np.random.default_rng(synth.SEED_BASE + 505)
        ss = [synth.step_signal(rng, L, 90.0, 12.0, 8.0, 1.5).astype(dt) for L in (700, 3000, 9001)]
        O.write_bundle(os.path.join(out, f"seg_{sfx}.odbs"), ss)
        for minseg in (4, 6):
            run(["segment", os.path.join(out, f"seg_{sfx}.odbs"),
                 os.path.join(out, f"seg_{sfx}_m{minseg}.odbs"), minseg, 0], log)

    # 8. clustering thresholds other than 1
    with open(os.path.join(out, "harness_log_clusters.jsonl"), "w") as clog:
        cluster_cases(out, tmp, clog)
    # 9. prefix chop with a leader sequence
    with open(os.path.join(out, "harness_log_chop.jsonl"), "w") as clog:
        chop_cases(out, tmp, clog)

    with open(os.path.join(out, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    shutil.rmtree(tmp, ignore_errors=True)

    # 10. timing only (not a fixture): the reference's medoid launches on the first
    # 40 rows of the 2000-series nanopore-like workload.
    if "--timing" in sys.argv:
        c2 = synth.znorm_host(synth.nanopore_like(2000, 2000, 8000, synth.SEED_BASE + 2))
        c2 = sorted(c2, key=len)
        tpath = os.path.join(out, "c2_input.odbs")
        O.write_bundle(tpath, c2)
        p = run(["pairwise", tpath, os.path.join(out, "c2_ref_rows.dist.odbs"), 0, 0, 40], log)
        print("reference timing:", p.stdout.strip())
        os.remove(tpath)
    log.close()
    print("golden written to", out)


if __name__ == "__main__":
    main()
