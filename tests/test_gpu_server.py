"""The serving loop on a B200: continuous batching of read-vs-centroid queries
and averaging jobs gives exactly the results of the direct paths, and the same
result for a request alone and in a mix."""
import threading
import time

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


def _workload(seed):
    rng = np.random.default_rng(seed)
    cents = [np.cumsum(rng.standard_normal(int(L))).astype(np.float32) for L in (300, 900, 1500)]
    queries = [[np.cumsum(rng.standard_normal(int(L))).astype(np.float32)
                for L in rng.integers(50, 2500, size=int(k))] for k in (1, 3, 5)]
    jobs = [[(np.cumsum(rng.standard_normal(int(L))) + 10).astype(np.float32)
             for L in rng.integers(80, 600, size=int(k))] for k in (4, 1, 7)]
    return cents, queries, jobs


def test_server_results_equal_direct_paths(api):
    cents, queries, jobs = _workload(1)
    srv = api.Server(np.float32, hbm_budget_bytes=4 << 30)
    try:
        ids = [srv.add_centroid(c) for c in cents]
        q_ids = [srv.submit_query(q, ids, open_end=(i % 2)) for i, q in enumerate(queries)]
        j_ids = [srv.submit_job(job, open_end=(i == 2), norm=1) for i, job in enumerate(jobs)]
        for i, rid in enumerate(q_ids):
            assert srv.wait(rid, 300) == 1
            got = srv.take(rid)["result"]
            oe = i % 2
            want = np.array([O.pairwise([r, c], 0, oe, fma_mode=1)[0]
                             for r in queries[i] for c in cents], dtype=np.float32)
            assert np.array_equal(_bits(got), _bits(want))
        plain = api.dba_jobs(jobs, [0, 0, 2], norm=1, batched=False)
        for i, rid in enumerate(j_ids):
            assert srv.wait(rid, 300) == 1
            r = srv.take(rid)
            assert r["medoid"] == plain[i]["medoid"]
            assert r["rounds"] == plain[i]["rounds"]
            assert np.array_equal(_bits(r["result"]), _bits(plain[i]["centroid"]))
        assert srv.stats()["iterations"] > 0
    finally:
        srv.close()


def test_server_alone_equals_in_mix(api):
    cents, queries, jobs = _workload(2)
    probe_q, probe_j = queries[1], jobs[2]
    alone = {}
    srv = api.Server(np.float32)
    try:
        ids = [srv.add_centroid(c) for c in cents]
        rq = srv.submit_query(probe_q, ids)
        assert srv.wait(rq, 300) == 1
        alone["q"] = srv.take(rq)["result"]
        rj = srv.submit_job(probe_j)
        assert srv.wait(rj, 300) == 1
        alone["j"] = srv.take(rj)["result"]
    finally:
        srv.close()
    # the same two requests submitted from two threads among many others
    srv = api.Server(np.float32, hbm_budget_bytes=256 << 20)
    try:
        ids = [srv.add_centroid(c) for c in cents]
        out = {}

        def noise(seed):
            rng = np.random.default_rng(seed)
            for _ in range(6):
                k = int(rng.integers(1, 4))
                rid = srv.submit_query([np.cumsum(rng.standard_normal(int(rng.integers(30, 3000))))
                                        .astype(np.float32) for _ in range(k)], ids)
                srv.wait(rid, 300)
                srv.take(rid)
                time.sleep(0.001)

        threads = [threading.Thread(target=noise, args=(s,)) for s in (10, 11)]
        for t in threads:
            t.start()
        rj = srv.submit_job(probe_j)
        rq = srv.submit_query(probe_q, ids)
        assert srv.wait(rq, 300) == 1 and srv.wait(rj, 300) == 1
        out["q"] = srv.take(rq)["result"]
        out["j"] = srv.take(rj)["result"]
        for t in threads:
            t.join()
    finally:
        srv.close()
    assert np.array_equal(_bits(out["q"]), _bits(alone["q"]))
    assert np.array_equal(_bits(out["j"]), _bits(alone["j"]))


def test_server_rejects_unknown_centroid(api):
    srv = api.Server(np.float32)
    try:
        from opendba_b200 import _native
        with pytest.raises(_native.OdbaError):
            srv.submit_query([np.ones(10, np.float32)], [7])
    finally:
        srv.close()
