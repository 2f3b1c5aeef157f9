"""The oracle's stripe-mode round and open-end shortcut, pinned against the
reference's own B200 runs (tests/golden/ref/stripe_ref.json, stripe_a_*,
sc_*; made by tests/golden/make_reference_golden.py --stripe-only /
--shortcut-only).

Stripe mode (dba.hpp:515-763) re-runs each stripe with the first sequence's
length set to the backtrack height, so with an open end its top-row rule and
shortcut act at that height; global and open-start rounds equal the
full-path round.  The shortcut's minimum is the partial one of the warp-0
lane whose shared store wins (dtw.hpp:97-105): lane 0 in the float build,
lane 16 in the double build.
"""
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle as O

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_reference_golden as G  # noqa: E402

REF = json.load(open(os.path.join(GOLDEN, "stripe_ref.json")))
DT = {"f32": np.float32, "f64": np.float64}


def _inputs(tag, sfx):
    return G.stripe_inputs(DT[sfx], tag)


def test_stripe_inputs_reproduce(tmp_path):
    for tag in REF["sets"]:
        assert tuple(REF["sets"][tag]) == (G.STRIPE_SETS[tag][0], G.STRIPE_SETS[tag][1],
                                           G.STRIPE_SETS[tag][2])
        for sfx in DT:
            c, m = _inputs(tag, sfx)
            O.write_bundle(str(tmp_path / "m.odbs"), m)
            O.write_bundle(str(tmp_path / "c.odbs"), [c])
            assert G._sha(open(tmp_path / "m.odbs", "rb").read()) == REF["inputs"][f"{tag}_{sfx}_members"]
            assert G._sha(open(tmp_path / "c.odbs", "rb").read()) == REF["inputs"][f"{tag}_{sfx}_centroid"]


def file_order(paths, centroid, members, oe):
    """(row, column) of the oriented matrix as the path files list them:
    (member, centroid) for members flipped under the open end."""
    out = []
    for k, p in enumerate(paths):
        p = np.asarray(p)
        ij = p[:, :2].astype(np.int32)
        if oe and len(centroid) < len(members[k]):
            ij = ij[:, ::-1]
        out.append((ij, p[:, 2].astype(np.uint8)))
    return out


@pytest.mark.parametrize("case", sorted(REF["cases"]))
def test_oracle_stripe_round_equals_reference(case):
    tag, sfx, mode = case.split("_", 2)
    os_, oe = G.MODES[mode]
    c, m = _inputs(tag, sfx)
    mean, _, delta, paths, hazards = O.dba_update_stripe(c, m, os_, oe)
    want = REF["cases"][case]
    assert G._sha(mean.tobytes()) == want["mean"]
    assert float(want["delta"]) == delta
    got = [G.path_digest(ij, mv) for ij, mv in file_order(paths, c, m, oe)]
    assert got == want["paths"]
    assert not hazards.any()
    if not oe:
        # global and open start: the stripe round is the full-path round
        full = O.dba_update(c, m, os_, oe)[0]
        assert np.array_equal(full.view(np.uint8), mean.view(np.uint8))


def test_oracle_stripe_raw_files_set_a():
    for sfx in DT:
        members = O.read_bundle(os.path.join(GOLDEN, f"stripe_a_{sfx}_members.odbs"))
        c = O.read_bundle(os.path.join(GOLDEN, f"stripe_a_{sfx}_centroid.odbs"))[0]
        for mode, (os_, oe) in G.MODES.items():
            ref_mean = O.read_bundle(os.path.join(GOLDEN, f"stripe_a_{sfx}_{mode}.mean.odbs"))[0]
            mean, _, _, paths, _ = O.dba_update_stripe(c, members, os_, oe)
            assert np.array_equal(mean.view(np.uint8), ref_mean.view(np.uint8)), (sfx, mode)
            gp = np.load(os.path.join(GOLDEN, f"stripe_a_{sfx}_{mode}.paths.npz"))
            for k, (ij, mv) in enumerate(file_order(paths, c, members, oe)):
                assert np.array_equal(ij, gp[f"ij{k}"]) and np.array_equal(mv, gp[f"mv{k}"]), (sfx, mode, k)


def test_shortcut_lane_is_what_distinguishes_the_reference():
    # the cases were chosen so that other lanes give other results: lane 0
    # (the full minimum) for double, and lane 31 for float, do not reproduce
    # the reference's double round d / float round e
    for case, lanes in (("d_f64_open_end", (0, 0)), ("e_f32_open_end", (31, 16))):
        tag, sfx, mode = case.split("_", 2)
        c, m = _inputs(tag, sfx)
        try:
            O.set_shortcut_lanes(*lanes)
            mean = O.dba_update_stripe(c, m, 0, 1, lane=lanes[0] if sfx == "f32" else lanes[1])[0]
        finally:
            O.set_shortcut_lanes()
        assert G._sha(mean.tobytes()) != REF["cases"][case]["mean"]


def undefined_single_row(m, n, sfx):
    """A one-row matrix whose last swath is not a multiple of 3 wide plus one:
    the reference reads the row-0 edge from a diagonal slot nothing wrote
    (dtw.hpp:155, costs[col-1] without the slot offset), unless its float
    build's shortcut fires first (n > 1024)."""
    if m != 1:
        return False
    if sfx == "f32" and n > 1024:
        return False
    return ((n - 1) % 1024) % 3 != 0


@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_open_end_pair_distances_shortcut_lanes(sfx):
    s = O.read_bundle(os.path.join(GOLDEN, f"sc_mix_{sfx}.odbs"))
    want = O.read_bundle(os.path.join(GOLDEN, f"sc_mix_{sfx}_open_end.dist.odbs"))[0]
    got = O.pairwise(s, 0, 1)
    p = checked = 0
    for i in range(len(s) - 1):
        for j in range(i + 1, len(s)):
            if not undefined_single_row(len(s[i]), len(s[j]), sfx):
                assert got[p].tobytes() == want[p].tobytes(), (i, j)
                checked += 1
            p += 1
    assert checked >= 80


@pytest.mark.parametrize("sfx", ["f32", "f64"])
def test_open_end_full_path_round_shortcut_lanes(sfx):
    members = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_members.odbs"))
    c = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_centroid.odbs"))[0]
    want = O.read_bundle(os.path.join(GOLDEN, f"sc_dba_{sfx}_open_end.mean.odbs"))[0]
    mean = O.dba_update(c, members, 0, 1)[0]
    assert np.array_equal(mean.view(np.uint8), want.view(np.uint8))
    if sfx == "f64":
        try:
            O.set_shortcut_lanes(0, 0)
            other = O.dba_update(c, members, 0, 1)[0]
        finally:
            O.set_shortcut_lanes()
        assert not np.array_equal(other.view(np.uint8), want.view(np.uint8))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_stripe_round_properties(dtype):
    # size-independent properties of the restatement on random ragged inputs:
    # global and open start equal the full-path round; with an open end a
    # centroid of one stripe (1024 columns or fewer) leaves the re-run's
    # height at the last row, so the full-path round again
    rng = np.random.default_rng(2024)
    for Lc in (1, 7, 1000, 1024, 1025, 2500):
        centroid = (np.cumsum(rng.standard_normal(Lc)) * 0.1).astype(dtype)
        for os_, oe in ((0, 0), (1, 0), (0, 1), (1, 1)):
            if oe and Lc > 1024:
                continue
            # with an open end keep every member within one stripe either way
            hi = 1025 if oe else 2600
            members = [(np.cumsum(rng.standard_normal(int(L))) * 0.1).astype(dtype)
                       for L in rng.integers(1, hi, size=5)]
            st = O.dba_update_stripe(centroid, members, os_, oe)
            full = O.dba_update(centroid, members, os_, oe)
            assert np.array_equal(st[0].view(np.uint8), full[0].view(np.uint8)), (Lc, os_, oe)
            assert np.array_equal(st[1], full[1]), (Lc, os_, oe)
