"""The reference-shaped Python surface on the device: multiclass and binary
predict_proba against the FP64 oracle, leaf solves with L1 and a
max_delta_step, and the regressor's tree_info / debug_predict diagnostics
(python/turbocat/__init__.py:779-800, python/bindings.cpp:804-964)."""
import numpy as np
import pytest

import oracle as O
from datagen import binary_c1, multiclass_c3, regression_c2

pytestmark = pytest.mark.gpu

REL = 1e-5


def _ensemble_from_dump(dump, base, K):
    """FP64-oracle ensemble of a facade model's get_booster_dump()."""
    T = len(dump)
    D = max([t["depth"] for t in dump] + [1])
    depth = np.array([t["depth"] for t in dump], np.int32)
    feat = np.zeros((T, D), np.uint16)
    thr = np.zeros((T, D), np.float32)
    leaves = np.zeros((T, 1 << D), np.float32)
    for i, t in enumerate(dump):
        for d, s in enumerate(t["splits"]):
            feat[i, d] = s["feature"]
            thr[i, d] = s["float_threshold"]
        leaves[i, :len(t["leaf_values"])] = t["leaf_values"]
    w = np.array([t["weight"] for t in dump], np.float32)
    return O.Ensemble(base, K, D, depth, feat, np.zeros((T, D), np.uint8), thr, leaves, w)


def test_multiclass_predict_proba_matches_oracle():
    import turbocat

    X, y = multiclass_c3(30_000, 12, 4, seed=91)
    clf = turbocat.TurboCatClassifier(n_estimators=12, learning_rate=0.2, max_depth=5, subsample=1.0,
                                      colsample_bytree=1.0, verbosity=0)
    clf.fit(X, y)
    assert clf.n_classes_ == 4
    proba = clf.predict_proba(X)
    assert proba.shape == (len(y), 4) and proba.dtype == np.float32
    ens = _ensemble_from_dump(clf._model.get_booster_dump(), clf._model.get_base_prediction(), 4)
    raw = O.predict(ens, X)
    z = np.exp(raw - raw.max(1, keepdims=True))
    want = z / z.sum(1, keepdims=True)
    assert np.max(np.abs(proba - want)) <= REL
    assert np.array_equal(clf.predict(X), np.argmax(proba, 1).astype(np.int32))


def test_binary_predict_proba_matches_oracle():
    import turbocat

    X, y = binary_c1(20_000, 10, seed=92)
    clf = turbocat.TurboCatClassifier(n_estimators=30, learning_rate=0.1, max_depth=6, subsample=1.0,
                                      colsample_bytree=1.0, verbosity=0)
    clf.fit(X, y)
    proba = clf.predict_proba(X)
    ens = _ensemble_from_dump(clf._model.get_booster_dump(), clf._model.get_base_prediction(), 1)
    p1 = 1.0 / (1.0 + np.exp(-O.predict(ens, X)[:, 0]))
    assert np.max(np.abs(proba[:, 1] - p1)) <= REL
    assert np.max(np.abs(proba[:, 0] - (1.0 - p1))) <= REL  # P0 = 1 - p (python/bindings.cpp:377-381)


@pytest.mark.parametrize("l1,mds", [(0.05, 0.0), (0.0, 0.15), (0.03, 0.1)])
def test_l1_and_max_delta_step_leaves(engine, capi, l1, mds):
    """Leaf values with the L1 soft threshold and the max_delta_step clamp
    (src/tree/symmetric_tree.cpp:753-775) against the FP64 oracle, on a tree
    built from given gradients and on a short fit."""
    X, y = binary_c1(40_000, 12, seed=93)
    hp = O.Hyper(loss="logloss", n_estimators=8, learning_rate=0.3, max_depth=6, lambda_l1=l1,
                 max_delta_step=mds)
    b = O.quantize(X)
    ds = engine.upload(X, y)
    ds.quantize(255)
    params = capi.params(loss="logloss", n_estimators=8, max_depth=6, learning_rate=0.3, lambda_l1=l1,
                         max_delta_step=mds)
    pred = np.full(len(y), O.init_prediction("logloss", y), np.float32)
    pred += 0.5 * np.random.default_rng(3).standard_normal(len(y)).astype(np.float32)
    g, h = O.gradients("logloss", y, pred)
    f64 = O.build_tree(b, g, h, hp, mode=1, want_rows=True)
    dev = engine.build_tree(ds, g, h, params)
    assert f64.margins().min() > 1e-6
    assert np.array_equal(dev["feature"], f64.feature) and np.array_equal(dev["bin"], f64.bin)
    L = 1 << f64.depth
    absg = np.bincount(f64.leaf_index, weights=np.abs(g.astype(np.float64)), minlength=L)
    H = np.bincount(f64.leaf_index, weights=h.astype(np.float64), minlength=L)
    tol = REL * absg / (H + hp.lambda_l2) + 1e-7
    assert np.all(np.abs(dev["leaves"][:L] - f64.leaves[:L]) <= tol)
    if mds > 0:
        assert np.max(np.abs(dev["leaves"])) <= mds
    # a short fit follows the FP64 oracle's trajectory (its margins permitting)
    ref = O.fit(b, y, hp, mode=1)
    tr = engine.trainer(ds, params)
    tr.step(hp.n_estimators)
    ex = tr.model().export()
    if ref.min_margin > 1e-6:
        assert np.array_equal(ex["feature"], ref.feature) and np.array_equal(ex["bin"], ref.bin)
        assert np.allclose(ex["leaves"], ref.leaves, rtol=REL, atol=1e-6)


def test_regressor_tree_info_and_debug_predict():
    import turbocat

    X, y = regression_c2(20_000, 14, seed=94)
    Xt = regression_c2(300, 14, seed=95)[0]
    Xt[0, 2] = np.nan
    reg = turbocat.TurboCatRegressor(n_estimators=15, learning_rate=0.1, max_depth=5, subsample=1.0,
                                     colsample_bytree=1.0, verbosity=0)
    reg.fit(X, y)
    info = reg.tree_info()
    dump = reg._model.get_booster_dump()
    assert len(info) == reg.n_trees == len(dump)
    for ti, t in zip(info, dump):
        nl = 1 << t["depth"]
        assert ti["n_leaves"] == nl and ti["n_nodes"] == 2 * nl - 1
        assert ti["is_single_leaf"] == (t["depth"] == 0)
        acc = np.float32(0.0)
        for v in np.asarray(t["leaf_values"], np.float32):  # FP32 in leaf order, as the binding sums
            acc = np.float32(acc + v)
        assert ti["leaf_sum"] == float(acc)
    dbg = reg.debug_predict(Xt)
    b = O.quantize(X)

    def bin_of(x, j):
        if np.isnan(x):
            return 255
        return int(np.searchsorted(b.edges[j, :b.n_edges[j]], x, side="right"))

    for fi in dbg["bin_variance"]:
        j = fi["feature"]
        assert fi["sample_bins"] == [bin_of(Xt[i, j], j) for i in range(10)]
        assert fi["unique_bins"] == len({bin_of(Xt[i, j], j) for i in range(100)})
    t0 = dump[0]
    for tr in dbg["sample_traces"]:
        i = tr["sample_idx"]
        idx = 0
        for k, step in enumerate(tr["path"]):
            s = t0["splits"][k]
            assert step["split_feature"] == s["feature"] and step["split_bin"] == s["threshold"]
            sb = bin_of(Xt[i, s["feature"]], s["feature"])
            assert step["sample_bin"] == sb and step["go_right"] == (sb != 255 and sb > s["threshold"])
            assert step["node_idx"] == (1 << k) - 1 + idx
            idx = 2 * idx + int(step["go_right"])
        assert tr["leaf_idx"] == idx and np.isclose(tr["leaf_value"], t0["leaf_values"][idx])
    for fi in dbg["train_bin_variance"]:
        j = fi["feature"]
        assert fi["unique_bins"] == len({int(b.bins[j, i]) for i in range(100)})
    for c in dbg["raw_value_comparison"]:
        j = c["feature"]
        assert c["train_min"] == np.nanmin(X[:, j]) and c["train_max"] == np.nanmax(X[:, j])
        assert c["test_min"] == np.nanmin(Xt[:, j]) and c["test_max"] == np.nanmax(Xt[:, j])
