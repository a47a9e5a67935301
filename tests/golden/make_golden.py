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


def categorical_golden():
    """The reference's categorical target statistics on one dataset, for both
    methods: its per-row encodings, global tables, bins and edges, an order
    (ordered) / folds (cv) under which the oracle reproduces them (the
    reference draws its own from std::random_device), and for the ordered
    method the model it trains on those bins."""
    from datagen import CAT_HYPER, categorical_case

    X, y = categorical_case()
    hp = O.Hyper(**CAT_HYPER)
    out = {}
    for method in ("ordered", "cv"):
        enc, rb, tables, model = O.ref_cat_ts(X, y, [2], method, hp, fit=method == "ordered")
        e = enc[0]
        if method == "ordered":
            order = O.recover_order(X, y, 2, e)
            Xo, tab, _ = O.ordered_ts(X, y, [2], order)
            out["tcat"] = np.frombuffer(model, np.uint8)
        else:
            order = O.recover_folds(X, y, 2, e, 5)
            Xo, tab, _ = O.cv_ts(X, y, [2], order, 5)
        assert np.array_equal(Xo[:, 2].view(np.uint32), e.view(np.uint32)), method
        keys, vals = tables[2]
        out.update({f"{method}_enc": e, f"{method}_order": order, f"{method}_keys": keys, f"{method}_vals": vals,
                    f"{method}_bins": rb.bins, f"{method}_edges": rb.edges, f"{method}_n_edges": rb.n_edges})
    np.savez_compressed(os.path.join(HERE, "categorical_small.npz"), **out)


def regular_train_golden():
    """Regular (depth-wise) trees the reference trains, for the training
    oracle: depth 7, so that the 64-leaf cap binds in the recursion's order."""
    from datagen import REGULAR_TRAIN_HYPER, regular_train_case

    X, y = regular_train_case()
    hp = O.Hyper(**REGULAR_TRAIN_HYPER)
    _, model, _, _, tp = O.ref_fit(X, y, hp)
    np.savez_compressed(os.path.join(HERE, "regular_train_small.npz"), tcat=np.frombuffer(model, np.uint8),
                        train_raw=tp)


def leafwise_golden():
    """Leaf-wise regular trees of the reference's regression preset
    (mode="small" with MSE), for the leaf-wise training oracle."""
    from datagen import LEAFWISE_HYPER, leafwise_case

    X, y = leafwise_case()
    _, model, _, _, _ = O.ref_fit(X, y, O.Hyper(**LEAFWISE_HYPER))
    np.savez_compressed(os.path.join(HERE, "leafwise_small.npz"), tcat=np.frombuffer(model, np.uint8))


def multiclass_regular_golden():
    """The reference's multiclass loop (regular trees, one per class and
    iteration), for the multiclass regular-tree oracle."""
    from datagen import MULTICLASS_REGULAR_HYPER, multiclass_regular_case

    X, y = multiclass_regular_case()
    _, model, _, _, _ = O.ref_fit(X, y, O.Hyper(**MULTICLASS_REGULAR_HYPER), want_pred=False)
    np.savez_compressed(os.path.join(HERE, "multiclass_regular_small.npz"), tcat=np.frombuffer(model, np.uint8))


def main():
    regular_golden()
    regular_train_golden()
    leafwise_golden()
    multiclass_regular_golden()
    categorical_golden()
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
    if sys.argv[1:] == ["categorical"]:
        categorical_golden()
    elif sys.argv[1:] == ["regular_train"]:
        regular_train_golden()
    elif sys.argv[1:] == ["leafwise"]:
        leafwise_golden()
    elif sys.argv[1:] == ["multiclass_regular"]:
        multiclass_regular_golden()
    else:
        main()
