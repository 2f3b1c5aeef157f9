"""Parity at the benchmark configurations themselves.

* The medoid configuration (2000 series of U[2000, 8000] samples, global,
  float32): the full distance triangle's SHA-256, a strided sample of its
  distances and the medoid against the reference's own run on the same input
  (its sources built for sm_100a; tests/golden/ref/c2_medoid_ref.json, made by
  tests/golden/make_reference_golden.py --configs-only), the pair_dists.txt
  that performDBA writes for it, byte for byte, and the error of a sample of
  distances against FP64.
* The plain-DBA configuration (64 random walks of U[512, 1024] samples,
  z-normalisation on, global, float32): performDBA run to convergence,
  avg.txt, pair_dists.txt and every member's last-round path against the
  reference's own run.
* One long pair of the stripe configuration's kind (step signals, 100k x 60k
  samples) per precision through the swath-pipeline plan, against the oracle.
"""
import ctypes
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C2_JSON = os.path.join(GOLDEN, "c2_medoid_ref.json")


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opendba_b200 import api, build
    build.build_library()
    return torch, api


def _sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def _c2_inputs():
    from opendba_b200 import synth
    raw = synth.medoid_workload(2000, 2000, 8000, synth.SEED_BASE + 2)
    normed, _, _ = O.znorm(raw)
    return raw, normed


def _child(code: str):
    p = subprocess.run([sys.executable, "-c", "import sys; sys.path.insert(0, %r)\n" % ROOT + code],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    return p


def test_medoid_configuration_matches_reference(env):
    torch, api = env
    with open(C2_JSON) as f:
        gold = json.load(f)
    raw, normed = _c2_inputs()
    assert _sha(np.concatenate(normed).tobytes()) == gold["input_sha256"]
    # the pipeline's own z-normalisation on the device, then the all-pairs pass
    ds = api.DeviceSeries.from_host(raw)
    api.znorm_(ds)
    flat = np.concatenate(normed)
    dev = ds.data[:len(flat)].cpu().numpy()
    assert np.array_equal(dev.view(np.uint32), flat.view(np.uint32))
    d = api.pairwise(ds, 0, 0)
    _, med = api.medoid(d, ds)
    dh = d.cpu().numpy()
    idx = np.arange(0, len(dh), gold["sample_stride"])
    assert np.array_equal(dh[idx].view(np.uint32), np.array(gold["sample_bits"], dtype=np.uint32))
    assert _sha(dh.tobytes()) == gold["dist_sha256"]
    assert med == gold["medoid"] == gold["medoid_from_dists"]
    # error against FP64 on 64 random pairs
    pairs = np.sort(np.random.default_rng(3).choice(len(dh), size=64, replace=False))
    err = O.rel_error(dh[pairs], O.pairwise_fp64ref(normed, 0, 0, pair_list=pairs)[pairs])
    assert err["max_rel"] < 1e-5, err


def test_medoid_configuration_pair_dists_file_matches_reference(env, tmp_path):
    # performDBA, clustering only, on the normalised inputs the reference ran on
    with open(C2_JSON) as f:
        gold = json.load(f)
    _, normed = _c2_inputs()
    src = str(tmp_path / "c2.odbs")
    O.write_bundle(src, normed)
    prefix = str(tmp_path / "c2")
    _child("from oracle import oracle as O\nfrom opendba_b200 import api\n"
           f"s = O.read_bundle({src!r})\n"
           f"api.perform_dba(s, ['s%d' % i for i in range(len(s))], {prefix!r}, 0, 0, norm=0, algo_mode=1)")
    with open(prefix + ".pair_dists.txt", "rb") as f:
        assert _sha(f.read()) == gold["pair_dists_txt_sha256"]


def test_plain_dba_configuration_converges_like_reference(env, tmp_path):
    src = os.path.join(GOLDEN, "perform_c1_f32.odbs")
    prefix = str(tmp_path / "c1")
    _child("from oracle import oracle as O\nfrom opendba_b200 import api\n"
           f"s = O.read_bundle({src!r})\n"
           f"api.perform_dba(s, ['s%d' % i for i in range(len(s))], {prefix!r}, 0, 0, norm=1)")
    for ext in (".avg.txt", ".pair_dists.txt"):
        with open(prefix + ext) as f, open(os.path.join(GOLDEN, "perform_c1_f32_global" + ext)) as g:
            assert f.read() == g.read(), ext
    gold = np.load(os.path.join(GOLDEN, "perform_c1_f32_global.paths.npz"))
    k = 0
    while f"ij{k}" in gold:
        with open(f"{prefix}.0.path{k}.txt") as f:
            rows = [ln.split("\t") for ln in f.read().splitlines()[1:]]
        ij = np.array([(int(r[0]), int(r[2])) for r in rows], dtype=np.int32)
        assert np.array_equal(ij, gold[f"ij{k}"]), f"path {k}"
        k += 1
    assert k == 64


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_long_pair_through_the_swath_pipeline_matches_oracle(env, dtype):
    torch, api = env
    from opendba_b200 import _native, synth
    rng = np.random.default_rng(0x0DBA0002 + 2)
    pair = synth.znorm_host(synth.step_signals(rng, [60_000, 100_000], 90.0, 12.0, 8.0, 1.5, dtype))
    ds = api.DeviceSeries.from_host(pair)
    lib = _native.lib()
    elem = np.dtype(dtype).itemsize
    ws = torch.empty(lib.odba_dtw_pairwise_workspace_bytes_n(elem, 2, ds.max_len), dtype=torch.uint8,
                     device="cuda")
    key = (elem, int(ds.max_len).bit_length() - 1, 0)  # (element size, log2 max_len, log2 pairs)
    assert lib.odba_tune_set(*key, 3) == 0  # pin the swath pipeline
    try:
        plan = ctypes.c_int(0)
        lib.odba_tune_query(elem, ds.max_len, 1, ws.numel(), ctypes.addressof(plan), None)
        assert plan.value == 3
        got = api.pairwise(ds, 0, 0, workspace=ws).cpu().numpy()
    finally:
        lib.odba_tune_set(*key, 0)
    want = O.pairwise_fast(pair, 0, 0)
    assert got.view(np.uint8).tobytes() == want.view(np.uint8).tobytes()
