"""The benchmark's reference arm on a small case, on CPU: the reference's own
Booster::train (oracle/_ref) stopped through its training callback after the
warm-up and timed trees, and the extrapolation of the full fit from the
measured set-up and per-tree times."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libtcref.so")),
                    reason="reference build oracle/_ref not present")
def test_reference_timed_stops_and_extrapolates():
    sys.path.insert(0, ROOT)
    import bench
    from datagen import imbalanced_c5

    X, y = imbalanced_c5(20_000, 12, seed=3, active=6)
    full, d = bench.reference_timed(X, y, warm_trees=2, timed_trees=3, max_seconds=120.0)
    assert d["trees_built"] == 5 and d["trees_timed"] == 3 and len(d["tree_ms"]) == 3
    assert 0 < d["setup_s"] < d["first_tree_end_s"]
    assert d["per_tree_s"] > 0
    assert np.isclose(np.mean(d["tree_ms"]) / 1e3, d["per_tree_s"])
    # the full 1000-tree fit: the measured part plus 995 more trees at the timed rate
    assert np.isclose(full, d["last_tree_end_s"] + (bench.TREES - 5) * d["per_tree_s"])
    assert np.isclose(d["last_tree_end_s"] - sum(d["tree_ms"]) / 1e3, d["first_tree_end_s"] +
                      (d["last_tree_end_s"] - d["first_tree_end_s"]) - sum(d["tree_ms"]) / 1e3)
