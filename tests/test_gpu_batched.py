"""Batched forms on a B200: the pair-list launch and the multi-job DBA rounds
(CUDA-graph replays) give exactly the per-job results, which are exactly the
reference's performDBA results (CPU oracle)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api as A
    from opendba_b200 import build
    build.build_library()
    return A


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def test_pairlist_equals_per_job_all_pairs(api):
    import ctypes
    import torch
    from opendba_b200 import _native
    rng = np.random.default_rng(3)
    jobs = [[np.cumsum(rng.standard_normal(int(L))).astype(np.float32)
             for L in rng.integers(20, 2500, size=int(k))] for k in (2, 5, 9, 3)]
    modes = [0, 2, 1, 3]
    allser = [s for job in jobs for s in job]
    ds = api.DeviceSeries.from_host(allser)
    tasks, want, base, out = [], [], 0, 0
    for job, fl in zip(jobs, modes):
        d = O.pairwise(job, fl & 1, (fl >> 1) & 1, fma_mode=1)
        want.append(d)
        n = len(job)
        for s in range(n - 1):
            for t in range(s + 1, n):
                tasks.append((base + s, base + t, out | ((fl & 1) << 62) | (((fl >> 1) & 1) << 63)))
                out += 1
        base += n
    rng.shuffle(tasks)
    arr = np.zeros(len(tasks), dtype=[("first", "<u4"), ("second", "<u4"), ("out", "<u8")])
    for i, (a, b, o) in enumerate(tasks):
        arr[i] = (a, b, o)
    d_tasks = torch.from_numpy(arr.view(np.uint8)).cuda()
    dists = torch.empty(out, dtype=torch.float32, device="cuda")
    ws = api.pairwise_workspace(ds)
    _native.call("odba_dtw_pairlist_f32", ds.data.data_ptr(), ds.offsets.data_ptr(), ds.lens.data_ptr(),
                 d_tasks.data_ptr(), len(tasks), ds.max_len, dists.data_ptr(), ws.data_ptr(), ws.numel(),
                 torch.cuda.current_stream().cuda_stream)
    got = dists.cpu().numpy()
    assert np.array_equal(_bits(got), _bits(np.concatenate(want)))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_batched_jobs_equal_plain_and_oracle(api, dtype):
    rng = np.random.default_rng(11)
    jobs, flags = [], []
    for j, k in enumerate((2, 6, 1, 9, 4, 3)):
        jobs.append([(np.cumsum(rng.standard_normal(int(L))) + 30).astype(dtype)
                     for L in rng.integers(60, 700, size=k)])
        flags.append([0, 2, 0, 1, 3, 2][j])
    batched = api.dba_jobs(jobs, flags, norm=1, batched=True)
    plain = api.dba_jobs(jobs, flags, norm=1, batched=False)
    for j, (b, p) in enumerate(zip(batched, plain)):
        assert b["medoid"] == p["medoid"] and b["rounds"] == p["rounds"], j
        assert np.array_equal(_bits(b["centroid"]), _bits(p["centroid"])), j
        r = O.perform_dba(jobs[j], flags[j] & 1, (flags[j] >> 1) & 1, norm=1, fma_mode=1)
        assert r["order"][r["medoid"]] == b["medoid"], j
        assert np.array_equal(_bits(b["centroid"]), _bits(r["centroid"])), j
        if len(jobs[j]) > 1:
            assert b["rounds"] == r["rounds"], j


def test_batched_rounds_in_memory_bounded_waves(api, monkeypatch):
    # a tiny round budget forces one job per wave; results must not change
    rng = np.random.default_rng(77)
    jobs = [[(np.cumsum(rng.standard_normal(int(L))) + 30.0).astype(np.float32)
             for L in rng.integers(50, 900, size=int(k))] for k in (6, 2, 9, 4, 7)]
    flags = [0, 2, 2, 1, 0]
    whole = api.dba_jobs(jobs, flags, norm=1, batched=True)
    monkeypatch.setenv("ODBA_ROUND_BUDGET_BYTES", "1")
    waves = api.dba_jobs(jobs, flags, norm=1, batched=True)
    plain = api.dba_jobs(jobs, flags, norm=1, batched=False)
    for a, b, c in zip(whole, waves, plain):
        assert a["medoid"] == b["medoid"] == c["medoid"]
        assert a["rounds"] == b["rounds"] == c["rounds"]
        assert np.array_equal(_bits(a["centroid"]), _bits(b["centroid"]))
        assert np.array_equal(_bits(a["centroid"]), _bits(c["centroid"]))
