"""Row sampling (subsample, colsample_bytree, seed) on the device against the
oracle's restatement of the reference's sampling, which
tests/test_oracle_pin.py pins bit for bit to the reference's own fit."""
import numpy as np
import pytest

import oracle as O
from datagen import binary_c1, multiclass_c3, noisy_binary_split, regression_c2

pytestmark = pytest.mark.gpu

MARGIN = 1e-6
REL = 1e-5


def _params(capi, hp, **kw):
    return capi.params(loss=hp.loss, n_classes=hp.n_classes, n_estimators=hp.n_estimators,
                       max_depth=hp.max_depth, max_bins=hp.max_bins, min_samples_leaf=hp.min_samples_leaf,
                       learning_rate=hp.learning_rate, lambda_l2=hp.lambda_l2, lambda_l1=hp.lambda_l1,
                       min_child_weight=hp.min_child_weight, min_split_gain=hp.min_split_gain,
                       max_delta_step=hp.max_delta_step, subsample=hp.subsample,
                       colsample_bytree=hp.colsample_bytree, seed=hp.seed, **kw)


def _check(engine, capi, X, y, hp, **kw):
    ds = engine.upload(X, y)
    ds.quantize(hp.max_bins)
    tr = engine.trainer(ds, _params(capi, hp, **kw))
    tr.step(hp.n_estimators)
    m = tr.model()
    ex = m.export()
    ob = O.quantize(X, hp.max_bins)
    f64 = O.fit(ob, y, hp, mode=1)
    assert f64.min_margin > MARGIN, "case too close to a tie for split identity"
    assert np.array_equal(ex["depth"], f64.depth)
    assert np.array_equal(ex["feature"], f64.feature) and np.array_equal(ex["bin"], f64.bin)
    assert np.allclose(ex["leaves"], f64.leaves, rtol=REL, atol=1e-6)
    # every row (sampled or not) carries every tree's prediction
    K = hp.n_classes if hp.loss == "softmax" else 1
    sc = tr.scores(len(y))
    assert np.allclose(sc, f64.train_pred.reshape(len(y), K), rtol=REL, atol=1e-5)
    return tr, ex, f64


@pytest.mark.parametrize("batched", [1, 0])
def test_binary_facade_defaults(engine, capi, batched):
    """subsample = colsample_bytree = 0.8, seed 42 (the Python facade's defaults)."""
    X, y = binary_c1(20_000, 12, seed=91)
    hp = O.Hyper(loss="logloss", n_estimators=6, learning_rate=0.1, max_depth=5, lambda_l2=1.0, subsample=0.8,
                 colsample_bytree=0.8, seed=42)
    _, ex, _ = _check(engine, capi, X, y, hp, batched=batched, hist_features_per_block=32)
    # and the reference's own trees (REF32 oracle == reference, pinned on the CPU)
    r32 = O.fit(O.quantize(X), y, hp, mode=0)
    if r32.min_margin > MARGIN:
        assert np.array_equal(ex["feature"], r32.feature) and np.array_equal(ex["bin"], r32.bin)


def test_regression_half_sample(engine, capi):
    X, y = regression_c2(30_000, 20, seed=92)
    hp = O.Hyper(loss="mse", n_estimators=8, learning_rate=0.1, max_depth=6, lambda_l2=0.0, subsample=0.5,
                 seed=7)
    _check(engine, capi, X, y, hp)


def test_multiclass_sampled(engine, capi):
    X, y = multiclass_c3(20_000, 10, K=3, seed=93)
    hp = O.Hyper(loss="softmax", n_classes=3, n_estimators=5, learning_rate=0.2, max_depth=4, lambda_l2=1.0,
                 subsample=0.7, colsample_bytree=0.5, seed=11)
    _check(engine, capi, X, y, hp, hist_features_per_block=32)


def test_sampling_with_validation_and_facade(engine, capi):
    """Sampling and early stopping together; the classifier's defaults
    (subsample 0.8, colsample_bytree 0.8, seed 42) fit the same ensemble as
    the C ABI with those parameters."""
    import turbocat

    Xt, yt, Xv, yv = noisy_binary_split()
    hp = O.Hyper(loss="logloss", n_estimators=150, learning_rate=0.3, max_depth=6, lambda_l2=1.0,
                 subsample=0.8, colsample_bytree=0.8, seed=42)
    ds = engine.upload(Xt, yt)
    ds.quantize(255)
    tr = engine.trainer(ds, _params(capi, hp, hist_features_per_block=32))
    tr.set_validation(engine.upload(Xv, yv), 10)
    tr.step(hp.n_estimators)
    st = tr.stats()
    ex = tr.model().export()
    f64 = O.fit(O.quantize(Xt), yt, hp, mode=1)
    n = st.iterations_done
    assert np.array_equal(ex["feature"], f64.feature[:n])
    clf = turbocat.TurboCatClassifier(n_estimators=150, learning_rate=0.3, max_depth=6, lambda_l2=1.0,
                                      early_stopping_rounds=10, mode="large", verbosity=0)
    clf.fit(Xt, yt, Xv, yv)
    assert clf.n_trees == n
