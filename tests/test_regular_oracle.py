"""The regular-tree oracle (models the reference trained with mode="small")
pinned to the reference: its FP32 predictions equal, bit for bit, the
reference's own predictions stored by tests/golden/make_golden.py."""
import numpy as np

import oracle as O
from datagen import regular_case, regular_pred_matrix


def test_regular_oracle_matches_reference_fixture():
    g = np.load(f"{O.HERE}/../tests/golden/regular_small.npz")
    m = O.parse_tcat_regular(g["tcat"].tobytes())
    X, _ = regular_case()
    P = regular_pred_matrix(X, m.edges)
    assert len(m.trees) == 40 and m.max_depth == 5
    # both binning rules of the reference occur: a feature of at most 16 edges
    # (edges <= x) and rows on an edge of a feature with more (edges < x)
    ne = np.array([len(e) for e in m.edges])
    assert (ne <= 16).any() and (ne > 16).any()
    on_edge = [(r, r % P.shape[1]) for r in range(200) if ne[r % P.shape[1]] > 16]
    assert on_edge
    p32 = O.predict_regular(m, P)
    assert np.array_equal(p32, g["pred_raw"])
    p64 = O.predict_regular(m, P, fp64=True)
    scale = abs(m.base) + sum(float(np.abs(t["value"]).max()) * float(w) for t, w in zip(m.trees, m.weights))
    assert np.max(np.abs(p64 - g["pred_raw"])) <= 1e-6 * scale
