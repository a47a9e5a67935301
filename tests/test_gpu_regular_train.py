"""Regular (depth-wise) trees trained on the device (tc_train_regular, the
reference's mode="small") against the regular-tree oracle.

The device sums exactly (fixed point) and scores in FP64, so its bar is the
oracle's FP64 mode: the same trees -- structure, numbering, the 64-leaf cap --
wherever the oracle's top gain beats the runner-up by more than 1e-6, leaf
values within 1e-5 relative.  Against the reference (FP32 sums, pinned to
the oracle's FP32 mode bit for bit on the CPU) the trees agree where FP32 and
FP64 choose alike."""
import numpy as np
import pytest

import oracle as O
from datagen import binary_c1

pytestmark = pytest.mark.gpu


def _params(capi, hp):
    return capi.params(loss=hp.loss, n_estimators=hp.n_estimators, max_depth=hp.max_depth, max_bins=hp.max_bins,
                       min_samples_leaf=hp.min_samples_leaf, learning_rate=hp.learning_rate,
                       lambda_l2=hp.lambda_l2, min_child_weight=hp.min_child_weight,
                       min_split_gain=hp.min_split_gain)


def _same_structure(t, r):
    return (len(t["value"]) == len(r["value"]) and all(np.array_equal(t[k], r[k]) for k in ("is_leaf", "left", "right"))
            and np.array_equal(t["feature"][~t["is_leaf"]], r["feature"][~r["is_leaf"]])
            and np.array_equal(t["split_bin"][~t["is_leaf"]], r["split_bin"][~r["is_leaf"]]))


@pytest.mark.parametrize("n,f,depth,msl,mcw,lam", [(3000, 10, 5, 1, 1.0, 1.0), (4000, 10, 7, 1, 1.0, 1.0),
                                                     (20_000, 8, 6, 20, 5.0, 3.0), (1, 3, 4, 1, 0.0, 1.0)])
def test_regular_fit_matches_fp64_oracle(engine, capi, n, f, depth, msl, mcw, lam):
    X, y = binary_c1(n, f, seed=n + depth)
    hp = O.Hyper(loss="logloss", n_estimators=10, max_depth=depth, learning_rate=0.2, min_samples_leaf=msl,
                 min_child_weight=mcw, lambda_l2=lam)
    ds = engine.upload(X, y)
    ds.quantize(255)
    m, st = engine.train_regular(ds, _params(capi, hp))
    dev = O.parse_tcat_regular(m.tcat())
    assert st.n_trees == hp.n_estimators and len(dev.trees) == hp.n_estimators
    b = O.quantize(X)
    base = O.init_prediction("logloss", y)
    assert np.float32(dev.base) == np.float32(base)
    p = np.full(n, base, np.float32)
    compared = 0
    for t_dev in dev.trees:
        g, h = O.gradients("logloss", y, p)
        t = O.build_regular_tree(b, g, h, hp, fp32=False)
        split = ~t["is_leaf"]
        if split.any() and t["margin"][split].min() <= 1e-6:
            break  # a near tie: the later trees follow from whichever side was taken
        assert _same_structure(t, t_dev)
        assert np.allclose(t_dev["value"], t["value"], rtol=1e-5, atol=1e-7)
        compared += 1
        leaf = t["value"][t["leaf_of"]].astype(np.longdouble)
        p = (p.astype(np.longdouble) + np.longdouble(np.float32(hp.learning_rate)) * leaf).astype(np.float32)
    assert compared >= 3
    # the model serves as the reference predicts regular trees (bit-exact to its oracle)
    pr = m.predict(X, "raw")[:, 0]
    assert np.array_equal(pr.view(np.uint32), O.predict_regular(dev, X).ravel().view(np.uint32))
    for hnd in (m, ds):
        hnd.close()


@pytest.mark.skipif(not O.ref_available(), reason="reference not built in this checkout")
def test_regular_fit_against_reference(engine, capi):
    X, y = binary_c1(3000, 10, seed=41)
    hp = O.Hyper(loss="logloss", n_estimators=8, max_depth=5, learning_rate=0.2, regular_trees=True)
    _, model, _, _, _ = O.ref_fit(X, y, hp)
    ref = O.parse_tcat_regular(model)
    ds = engine.upload(X, y)
    ds.quantize(255)
    m, _ = engine.train_regular(ds, _params(capi, hp))
    dev = O.parse_tcat_regular(m.tcat())
    for t_dev, t_ref in zip(dev.trees, ref.trees):
        assert _same_structure(t_dev, t_ref)
        # the reference's FP32 subtraction chains put its leaves ~1e-4 off exact sums
        assert np.allclose(t_dev["value"], t_ref["value"], rtol=2e-3, atol=2e-3)
    for hnd in (m, ds):
        hnd.close()


def test_regular_fit_rejects_what_it_does_not_build(engine, capi):
    X, y = binary_c1(500, 4, seed=2)
    ds = engine.upload(X, y)
    ds.quantize(255)
    for kw in (dict(loss="mse"), dict(loss="focal"), dict(subsample=0.5), dict(use_goss=True)):
        with pytest.raises(Exception):
            engine.train_regular(ds, capi.params(n_estimators=2, max_depth=3, **kw))
    ds.close()


def test_classifier_mode_small_trains_regular_trees(tmp_path):
    import turbocat
    from turbocat import _capi

    X, y = binary_c1(3000, 10, seed=41)
    clf = turbocat.TurboCatClassifier(n_estimators=10, max_depth=5, learning_rate=0.2, subsample=1.0,
                                      colsample_bytree=1.0, mode="small", verbosity=0)
    clf.fit(X, y)
    p = clf.predict_proba(X)
    clf.save(str(tmp_path / "r.tcat"))
    dev = O.parse_tcat_regular(open(tmp_path / "r.tcat", "rb").read())  # a regular-tree model
    assert len(dev.trees) == 10
    raw = O.predict_regular(dev, X).ravel().astype(np.float64)
    assert np.allclose(p[:, 1], 1.0 / (1.0 + np.exp(-raw)), rtol=1e-6, atol=1e-7)
    eng = _capi.Engine(0)
    m = eng.load_tcat(open(tmp_path / "r.tcat", "rb").read())
    assert np.array_equal(m.predict(X, "sigmoid")[:, 0], p[:, 1])
    m.close()
