"""Host-side parts of the learned-closure evaluation."""
import numpy as np

from tests.golden_io import load
from zhenmode_b200.closure import mixed_layer_depth


def test_mixed_layer_depth_matches_the_reference():
    """diagnostics/mixed_layer.py:39-74 on thermocline columns with missing
    levels below the seafloor (tests/golden/mld_24x16x20.npz)."""
    g = load("mld_24x16x20")
    got = mixed_layer_depth(g["T"], g["S"], g["z"], g["wet3"])
    want = g["mld"]
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.nanmax(np.abs(got - want)) == 0.0
    assert np.nanmax(want) > np.nanmin(want)  # the columns differ
