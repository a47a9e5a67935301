"""Row sampling (subsample, colsample_bytree, seed; GOSS) on the device
against the oracle's restatement of the reference's sampling, which
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
                       colsample_bytree=hp.colsample_bytree, seed=hp.seed, use_goss=hp.use_goss,
                       goss_top_rate=hp.goss_top_rate, goss_other_rate=hp.goss_other_rate, **kw)


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


def _goss_rows(g, hp, state):
    """The oracle's GOSS rows for gradients g [n] or [n][K] and the next draw of the stream."""
    a = np.abs(g) if g.ndim == 1 else np.max(np.abs(g), axis=1)
    state, seed = O.next_random(state)
    rows = O.goss_subsample(a, hp.goss_top_rate, hp.goss_other_rate, seed)
    if hp.colsample_bytree < 1.0:
        state, _ = O.next_random(state)
    return rows, state


@pytest.mark.parametrize("batched", [1, 0])
def test_goss_selection_every_iteration(engine, capi, batched):
    """GOSS on MSE: before every iteration the device's scores give the
    gradients 2 (pred - y) exactly (FP32), so the oracle's selection over
    them (std::nth_element, std::mt19937_64 draws from the xorshift64*
    stream) must be the device's sample bit for bit; the first tree (same
    gradients and sample as the FP64 oracle's fit) matches the oracle's."""
    X, y = regression_c2(30_000, 20, seed=94)
    n = len(y)
    hp = O.Hyper(loss="mse", n_estimators=6, learning_rate=0.1, max_depth=6, lambda_l2=0.0, use_goss=True,
                 goss_top_rate=0.2, goss_other_rate=0.1, colsample_bytree=0.8, seed=7)
    ds = engine.upload(X, y)
    ds.quantize(hp.max_bins)
    tr = engine.trainer(ds, _params(capi, hp, batched=batched))
    state = hp.seed
    for t in range(hp.n_estimators):
        s = tr.scores(n)[:, 0]
        g = np.float32(2.0) * (s - y)
        rows, state = _goss_rows(g, hp, state)
        tr.step(1)
        want = np.zeros(n, bool)
        want[rows] = True
        assert np.array_equal(tr.sample_mask(n), want), f"iteration {t}"
    ex = tr.model().export()
    f64 = O.fit(O.quantize(X), y, O.Hyper(**{**hp.__dict__, "n_estimators": 1}), mode=1)
    assert f64.min_margin > MARGIN
    assert ex["depth"][0] == f64.depth[0]
    assert np.array_equal(ex["feature"][0], f64.feature[0]) and np.array_equal(ex["bin"][0], f64.bin[0])
    assert np.allclose(ex["leaves"][0], f64.leaves[0], rtol=REL, atol=1e-6)
    # every row carries every tree (sampled or not): scores = the model's prediction
    m = tr.model()
    assert np.allclose(tr.scores(n)[:, 0], m.predict(X, "raw")[:, 0], rtol=1e-5, atol=1e-5)


def test_goss_multiclass_and_edges(engine, capi):
    """Softmax GOSS ranks rows by the largest |g| over the classes: the
    sample has (uint32)(n * top) + (uint32)(n * other) rows, the same seed
    gives the same ensemble and another seed another one; rates 0 / 0 build
    single-leaf trees of 0, rate 1 uses every row (the trees of no sampling)."""
    X, y = multiclass_c3(12_000, 10, K=3, seed=95)
    n = len(y)
    hp = O.Hyper(loss="softmax", n_classes=3, n_estimators=4, learning_rate=0.2, max_depth=4, lambda_l2=1.0,
                 use_goss=True, goss_top_rate=0.3, goss_other_rate=0.2, seed=3)
    ds = engine.upload(X, y)
    ds.quantize(255)

    def run(**kw):
        h = O.Hyper(**{**hp.__dict__, **kw})
        tr = engine.trainer(ds, _params(capi, h, hist_features_per_block=32))
        tr.step(h.n_estimators)
        return tr, tr.model().export()

    tr, a = run()
    top, other = int(np.float32(n) * np.float32(0.3)), int(np.float32(n) * np.float32(0.2))
    assert tr.sample_mask(n).sum() == top + other
    _, b = run()
    assert np.array_equal(a["leaves"], b["leaves"]) and np.array_equal(a["feature"], b["feature"])
    _, c = run(seed=4)
    assert not np.array_equal(a["leaves"], c["leaves"])
    tr0, z = run(goss_top_rate=0.0, goss_other_rate=0.0)
    assert not tr0.sample_mask(n).any()
    assert np.all(z["depth"] == 0) and np.all(z["leaves"] == 0.0)
    tr1, full = run(goss_top_rate=1.0, goss_other_rate=0.0)
    assert tr1.sample_mask(n).all()
    _, plain = run(use_goss=False)
    assert np.array_equal(full["feature"], plain["feature"]) and np.array_equal(full["bin"], plain["bin"])
    assert np.allclose(full["leaves"], plain["leaves"], rtol=1e-5, atol=1e-6)
    with pytest.raises(capi.TCError):
        engine.trainer(ds, _params(capi, O.Hyper(**{**hp.__dict__, "goss_top_rate": 1.5})))


def test_goss_facade(engine, capi):
    """TurboCatClassifier(use_goss=True) and TurboCatRegressor(use_goss=True)
    train on the device (no warning, no fallback) and reproduce the C ABI's
    ensemble with the same parameters."""
    import warnings

    import turbocat

    X, y = binary_c1(20_000, 12, seed=96)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        clf = turbocat.TurboCatClassifier(n_estimators=12, learning_rate=0.1, max_depth=5, lambda_l2=1.0,
                                          use_goss=True, goss_top_rate=0.2, goss_other_rate=0.1, subsample=1.0,
                                          colsample_bytree=0.8, mode="large", verbosity=0, seed=42)
        clf.fit(X, y)
    hp = O.Hyper(loss="logloss", n_estimators=12, learning_rate=0.1, max_depth=5, lambda_l2=1.0,
                 colsample_bytree=0.8, seed=42, use_goss=True)
    ds = engine.upload(X, y)
    ds.quantize(255)
    tr = engine.trainer(ds, _params(capi, hp))
    tr.step(hp.n_estimators)
    p_capi = tr.model().predict(X, "sigmoid")[:, 0]
    assert np.allclose(clf.predict_proba(X)[:, 1], p_capi, rtol=1e-5, atol=1e-6)
    Xr, yr = regression_c2(20_000, 16, seed=97)
    reg = turbocat.TurboCatRegressor(n_estimators=10, learning_rate=0.1, max_depth=5, use_goss=True, verbosity=0)
    reg.fit(Xr, yr)
    assert reg.n_trees == 10 and np.isfinite(reg.predict(Xr)).all()
