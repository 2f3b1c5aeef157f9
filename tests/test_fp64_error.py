"""Error of the distances against an FP64 reference, per fixture family.

The distances this library computes are bit-identical to the reference's own
GPU results and to the oracle (the parity tests pin both), so the oracle's
float and double results stand for them here.  The FP64 reference is the same
recurrence, tie order and swath rules evaluated in double with a double
square root (oracle.pairwise_fp64ref).  Float results stay within 1e-5
relative.  Double results stay within 2e-7, a bound set by the reference's
epilogue, which works in float even for double (dtw.hpp:116-125, 242-257):
the cost cast to float, sqrtf, and the division by m with one open end are
three float roundings of at most 2^-24 each.

Run with -s to print the table (family, precision, mode, pairs, max and
median relative error).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O

BOUND = {np.dtype(np.float32): 1e-5, np.dtype(np.float64): 2e-7}
MODES = {"global": (0, 0), "open_start": (1, 0), "open_end": (0, 1), "open": (1, 1)}


def _report(family, series, mode, pair_list=None):
    os_, oe = MODES[mode]
    got = O.pairwise(series, os_, oe, pair_list=pair_list)
    ref = O.pairwise_fp64ref(series, os_, oe, pair_list=pair_list)
    sel = np.arange(len(got)) if pair_list is None else np.asarray(pair_list)
    err = O.rel_error(got[sel], ref[sel])
    dt = np.dtype(series[0].dtype)
    print(f"{family:28s} {dt.name:8s} {mode:10s} {err['pairs']:6d} "
          f"{err['max_rel']:.3e} {err['median_rel']:.3e}")
    assert err["max_rel"] < BOUND[dt], (family, mode, err)
    return err


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", list(MODES))
def test_edge_length_mix(sfx, mode):
    _report("edge lengths 2-3100", O.read_bundle(os.path.join(GOLDEN, f"pw_mix_{sfx}.odbs")), mode)


@pytest.mark.parametrize("mode", ["global", "open_end"])
def test_plain_dba_configuration(mode):
    # 64 z-normalised random walks of 512-1024 samples
    _report("plain DBA config (64 x 512-1024)", O.read_bundle(os.path.join(GOLDEN, "pw_c1_f32.odbs")),
            mode)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_medoid_configuration_sample(dtype):
    # 120 random pairs of the 2000-series medoid workload (z-normalised)
    from opendba_b200 import synth
    raw = synth.medoid_workload(2000, 2000, 8000, synth.SEED_BASE + 2)
    normed = [s.astype(dtype) for s in O.znorm([r.astype(dtype) for r in raw])[0]]
    n = len(normed)
    pairs = np.sort(np.random.default_rng(9).choice(n * (n - 1) // 2, size=120, replace=False))
    _report("medoid config sample", normed, "global", pair_list=pairs)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_long_pair_sample(dtype):
    # one pair of the stripe configuration's kind (step signals, dwell 8, noise 1.5)
    from opendba_b200 import synth
    rng = np.random.default_rng(0x0DBA0002 + 2)
    pair = synth.znorm_host(synth.step_signals(rng, [12_000, 20_000], 90.0, 12.0, 8.0, 1.5, dtype))
    _report("long pair 12k x 20k", pair, "global")
