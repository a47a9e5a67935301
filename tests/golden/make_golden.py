"""Generates the golden fixtures in this directory by running the reference
implementation itself (oracle/_ref/libtcref.so, built from the reference's
sources by oracle/ref.mk).  Run from the repository root in a container that
has the reference tree:

    make -f oracle/ref.mk && make -C oracle && python tests/golden/make_golden.py

Each case stores the seeded inputs' generator parameters (not the data: the
data is regenerated from the seed by tests/datagen.py), the reference's bins,
edges, TCAT model bytes and raw predictions.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from datagen import GOLDEN_CASES, make_case  # noqa: E402


def regular_golden():
    """A model of regular (depth-wise) trees trained by the reference
    (mode="small") and its raw predictions through the reference's own
    prediction path for such models."""
    from datagen import regular_case, regular_pred_matrix

    X, y = regular_case()
    hp = O.Hyper(loss="logloss", n_estimators=40, max_depth=5, learning_rate=0.2, regular_trees=True)
    _, model, _, _, _ = O.ref_fit(X, y, hp)
    m = O.parse_tcat_regular(model)
    P = regular_pred_matrix(X, m.edges)
    raw = O.ref_predict(model, P, proba=False)
    np.savez_compressed(os.path.join(HERE, "regular_small.npz"), tcat=np.frombuffer(model, np.uint8), pred_raw=raw)


def main():
    regular_golden()
    for name, spec in GOLDEN_CASES.items():
        X, y, hp = make_case(spec)
        if hp.loss == "softmax":
            depth, sf, sb, st, lv, tp = O.ref_fit_multiclass(X, y, hp)
            rb = O.ref_quantize(X, hp.max_bins)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), bins=rb.bins, edges=rb.edges,
                                n_edges=rb.n_edges, depth=depth, feature=sf, bin=sb, threshold=st, leaves=lv,
                                train_raw=tp)
        else:
            rb, model, gt, ht, tp = O.ref_fit(X, y, hp, trace=True)
            raw = O.ref_predict(model, X, proba=False)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), bins=rb.bins, edges=rb.edges,
                                n_edges=rb.n_edges, tcat=np.frombuffer(model, np.uint8), pred_raw=raw,
                                grad0=gt[0], hess0=ht[0], grad_last=gt[-1], hess_last=ht[-1])
        print("wrote", name)


if __name__ == "__main__":
    main()
