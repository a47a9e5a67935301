"""Validation set and early stopping on the device (tc_trainer_set_validation)
against the oracle's replay of the reference's rule (Booster::train's
valid_data branch), which tests/test_oracle_pin.py pins to the reference's
own early-stopped fit."""
import numpy as np
import pytest

import oracle as O
from datagen import multiclass_c3, noisy_binary_split, regression_c2

pytestmark = pytest.mark.gpu

MARGIN = 1e-6


def _params(capi, hp, **kw):
    return capi.params(loss=hp.loss, n_classes=hp.n_classes, n_estimators=hp.n_estimators,
                       max_depth=hp.max_depth, max_bins=hp.max_bins, min_samples_leaf=hp.min_samples_leaf,
                       learning_rate=hp.learning_rate, lambda_l2=hp.lambda_l2, lambda_l1=hp.lambda_l1,
                       min_child_weight=hp.min_child_weight, min_split_gain=hp.min_split_gain,
                       max_delta_step=hp.max_delta_step, hist_features_per_block=32, **kw)


def _fit(engine, capi, Xt, yt, Xv, yv, hp, rounds, batched=1):
    ds = engine.upload(Xt, yt)
    ds.quantize(hp.max_bins)
    vds = engine.upload(Xv, yv)
    tr = engine.trainer(ds, _params(capi, hp, batched=batched))
    tr.set_validation(vds, rounds)
    tr.step(hp.n_estimators)
    m = tr.model()
    return tr, tr.stats(), tr.valid_loss(), m.export(), m


def _replay(m, ex, Xv, yv, hp, rounds):
    e = O.Ensemble(m.info.base_prediction, m.info.n_classes, ex["leaves"].shape[1].bit_length() - 1,
                   ex["depth"], ex["feature"], ex["bin"], ex["threshold"], ex["leaves"], ex["weights"])
    return O.early_stopping(e, Xv, yv, hp.loss, hp.n_estimators, rounds, hp.learning_rate)


@pytest.mark.parametrize("batched", [1, 0])
def test_binary_stops_where_the_rule_fires(engine, capi, batched):
    Xt, yt, Xv, yv = noisy_binary_split()
    hp = O.Hyper(loss="logloss", n_estimators=200, learning_rate=0.3, max_depth=6, lambda_l2=1.0)
    tr, st, losses, ex, m = _fit(engine, capi, Xt, yt, Xv, yv, hp, 10, batched)
    assert st.stopped_early == 1 and 50 < st.iterations_done < 200
    assert m.info.n_trees == st.iterations_done
    # the oracle's replay over the device's own trees: same losses, stops at the last one
    lo, stop, best = _replay(m, ex, Xv, yv, hp, 10)
    assert np.allclose(losses, lo, rtol=1e-5, atol=1e-7)
    assert stop == st.iterations_done - 1 and st.best_iteration == best
    # the reference-identical oracle's trees and stopping iteration (pinned to
    # the reference in tests/test_oracle_pin.py)
    e32 = O.fit(O.quantize(Xt), yt, hp, mode=0)
    _, stop32, _ = O.early_stopping(e32, Xv, yv, "logloss", 200, 10, 0.3)
    if e32.min_margin > MARGIN and np.array_equal(e32.feature[: st.iterations_done], ex["feature"]):
        assert st.iterations_done == stop32 + 1
    # more steps after the stop grow nothing
    tr.step(5)
    assert tr.stats().iterations_done == st.iterations_done
    # train scores equal the model's prediction of the training rows
    sc = tr.scores(len(yt))[:, 0]
    assert np.allclose(sc, m.predict(Xt, "raw")[:, 0], rtol=1e-5, atol=1e-5)


def test_regression_and_never_stop(engine, capi):
    X, y = regression_c2(12_000, 16, seed=83)
    Xt, yt, Xv, yv = X[:8000], y[:8000], X[8000:], y[8000:]
    hp = O.Hyper(loss="mse", n_estimators=80, learning_rate=0.2, max_depth=6, lambda_l2=0.0)
    tr, st, losses, ex, m = _fit(engine, capi, Xt, yt, Xv, yv, hp, -1)
    assert st.stopped_early == 0 and st.iterations_done == 80 and len(losses) == 80
    lo, stop, best = _replay(m, ex, Xv, yv, hp, -1)
    assert stop == -1 and st.best_iteration == best
    assert np.allclose(losses, lo, rtol=1e-5, atol=1e-7)
    assert losses[-1] < losses[0]


def test_multiclass_validation(engine, capi):
    X, y = multiclass_c3(9000, 12, K=4, seed=84)
    Xt, yt, Xv, yv = X[:6000], y[:6000], X[6000:], y[6000:]
    hp = O.Hyper(loss="softmax", n_classes=4, n_estimators=120, learning_rate=0.5, max_depth=5, lambda_l2=1.0)
    for batched in (1, 0):
        tr, st, losses, ex, m = _fit(engine, capi, Xt, yt, Xv, yv, hp, 5, batched)
        lo, stop, best = _replay(m, ex, Xv, yv, hp, 5)
        assert np.allclose(losses, lo, rtol=1e-5, atol=1e-7)
        assert st.best_iteration == best
        if st.stopped_early:
            assert stop == st.iterations_done - 1
        else:
            assert stop == -1 and st.iterations_done == 120


def test_validation_set_is_checked(engine, capi):
    Xt, yt, Xv, yv = noisy_binary_split(n=500, nv=200)
    ds = engine.upload(Xt, yt)
    ds.quantize(255)
    tr = engine.trainer(ds, capi.params(loss="logloss", n_estimators=10, max_depth=4,
                                        hist_features_per_block=32))
    with pytest.raises(capi.TCError) as ei:
        tr.set_validation(engine.upload(Xv[:, :5], yv), 10)  # wrong feature count
    assert ei.value.status == 1
    tr.step(1)
    with pytest.raises(capi.TCError):
        tr.set_validation(engine.upload(Xv, yv), 10)  # after the first iteration


def test_facade_fit_with_validation(engine, capi):
    """TurboCatClassifier.fit(X, y, X_val, y_val) early-stops like the C ABI run."""
    import turbocat

    Xt, yt, Xv, yv = noisy_binary_split()
    hp = O.Hyper(loss="logloss", n_estimators=200, learning_rate=0.3, max_depth=6, lambda_l2=1.0)
    _, st, _, _, _ = _fit(engine, capi, Xt, yt, Xv, yv, hp, 10)
    clf = turbocat.TurboCatClassifier(n_estimators=200, learning_rate=0.3, max_depth=6, lambda_l2=1.0,
                                      min_child_weight=1.0, early_stopping_rounds=10, mode="large",
                                      subsample=1.0, colsample_bytree=1.0, verbosity=0)
    clf.fit(Xt, yt, Xv, yv)
    assert clf.n_trees == st.iterations_done
