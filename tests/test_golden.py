"""The oracle and the binning order reproduce the committed golden fixtures
(tests/golden/*.npz, written by tests/golden/make_golden.py). Forward and
gradient walks are deterministic (per-tile partial sums merged in tile order),
so the comparison is to 1e-12 relative."""
import os
import sys

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402


def load(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def close(a, b, rel=1e-12):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= rel * np.maximum(1.0, np.abs(b)))


@pytest.mark.parametrize("name", [n for n in make_golden.CASES])
def test_oracle_reproduces_golden(name):
    want = load(name)
    got = make_golden.CASES[name]()
    assert set(got) == set(want)
    for k in want:
        if want[k].dtype.kind in "iu":
            assert np.array_equal(np.asarray(got[k]), want[k]), (name, k)
        else:
            assert close(got[k], want[k]), (name, k)


def test_golden_forward_covers_pixels():
    f = load("forward_s101_n20_d0_64")
    assert f["out_alpha"].max() > 0.5 and (f["out_ncontrib"] > 0).mean() > 0.2


def test_golden_binning_is_tile_then_depth_then_entry():
    b = load("binning_13x9")
    tiles_x = int(b["tiles_x"])
    items = b["entry_items"][b["sorted_entries"]]
    depth = b["depths"][items]
    # recover each sorted entry's tile from the ranges
    tile = np.zeros(items.size, np.int64)
    for t, (s, e) in enumerate(b["ranges"]):
        tile[s:e] = t
        if e > s:
            assert np.all(np.diff(depth[s:e].astype(np.int64)) >= 0)
            ties = np.diff(depth[s:e].astype(np.int64)) == 0
            assert np.all(np.diff(b["sorted_entries"][s:e].astype(np.int64))[ties] > 0)
    assert np.all(np.diff(tile) >= 0)
    r = b["rects"][items]
    tx, ty = tile % tiles_x, tile // tiles_x
    assert np.all((r[:, 0] <= tx) & (tx <= r[:, 2]) & (r[:, 1] <= ty) & (ty <= r[:, 3]))
