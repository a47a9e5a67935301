"""Categorical target statistics on the device, through the C ABI, against the
reference's stored run (tests/golden/categorical_small.npz) and the oracle.

Bars: encodings, global tables, bins and edges bit-exact (integer and float
work in the reference's order of additions); the model trained on them equal
to the reference's split for split where the reference's margins exceed 1e-6,
leaves within 1e-5 relative."""
import numpy as np
import pytest

import oracle as O
from datagen import CAT_HYPER, categorical_case

pytestmark = pytest.mark.gpu


def _u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _fixture():
    return np.load(f"{O.HERE}/../tests/golden/categorical_small.npz")


@pytest.mark.parametrize("method", ["ordered", "cv"])
def test_encode_matches_reference_run(engine, method):
    """Given the order / folds of the reference's stored run, the device
    reproduces its encodings, table, bins and edges bit for bit."""
    g = _fixture()
    X, y = categorical_case()
    ds = engine.upload(X, y)
    ds.encode_categorical([2], method, order=g[f"{method}_order"])
    F = ds.features()
    assert np.array_equal(_u32(F[:, 2]), _u32(g[f"{method}_enc"]))
    assert np.array_equal(_u32(np.delete(F, 2, 1)), _u32(np.delete(X, 2, 1)))
    keys, vals = ds.category_table(2)
    assert np.array_equal(keys, g[f"{method}_keys"]) and np.array_equal(_u32(vals), _u32(g[f"{method}_vals"]))
    edges, ne = ds.quantize(255)
    assert np.array_equal(ds.bins(), g[f"{method}_bins"])
    assert np.array_equal(_u32(edges), _u32(g[f"{method}_edges"])) and np.array_equal(ne, g[f"{method}_n_edges"])
    ds.close()


def _odd_case(n, seed, labels="float"):
    """Three categorical columns: small ids, wide ids (category 0xFFFFFFFF from
    -1.0 next to NaN rows, 2^32 folding onto 0, fractions truncated) and a
    high-cardinality one.  Float labels make the order of the additions show
    (the device's sequential walk); class ids add exactly in any order (its
    parallel prefix / fold-total path)."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 7)).astype(np.float32)
    X[:, 1] = rng.integers(0, 9, n)
    X[:, 3] = rng.choice(np.array([-1.0, 0.0, 1.5, 2.0, 4294967296.0, 7e6], np.float32), n)
    X[:, 5] = rng.integers(0, max(2, n // 3), n)
    for j in (1, 3, 5):
        X[rng.random(n) < 0.04, j] = np.nan
    y = rng.random(n).astype(np.float32) if labels == "float" else rng.integers(0, 3, n).astype(np.float32)
    return X, y


@pytest.mark.parametrize("method,n,pw,labels", [
    ("ordered", 1, 1.0, "float"), ("ordered", 5000, 1.0, "float"), ("ordered", 40_000, 2.5, "float"),
    ("cv", 5000, 1.0, "float"), ("cv", 40_000, 0.5, "float"),
    ("ordered", 1, 1.0, "class"), ("ordered", 70_000, 1.0, "class"), ("ordered", 70_000, 2.5, "class"),
    ("cv", 70_000, 1.0, "class"), ("cv", 9000, 0.5, "class")])
def test_encode_matches_oracle(engine, method, n, pw, labels):
    X, y = _odd_case(n, seed=n + int(pw * 10), labels=labels)
    rng = np.random.default_rng(7)
    feats = [1, 3, 5]
    if method == "ordered":
        order = rng.permutation(n).astype(np.uint32)
        Xo, tab, _ = O.ordered_ts(X, y, feats, order, pw)
    else:
        order = rng.integers(0, 5, n).astype(np.uint32)
        Xo, tab, _ = O.cv_ts(X, y, feats, order, 5, pw)
    ds = engine.upload(X, y)
    ds.encode_categorical(feats, method, prior_weight=pw, order=order)
    F = ds.features()
    assert np.array_equal(_u32(F), _u32(Xo))
    for j in feats:
        keys, vals = ds.category_table(j)
        assert np.array_equal(keys, tab[j][0]) and np.array_equal(_u32(vals), _u32(tab[j][1]))
    edges, ne = ds.quantize(255)
    b = O.quantize_ts(Xo, feats)
    assert np.array_equal(ds.bins(), b.bins)
    assert np.array_equal(_u32(edges), _u32(b.edges)) and np.array_equal(ne, b.n_edges)
    ds.close()


@pytest.mark.parametrize("method", ["ordered", "cv"])
def test_seeded_order_is_a_valid_draw(engine, method):
    """Without a given order the device draws one from the seed: the result is
    reproducible, differs between seeds, and is what the reference could have
    drawn (the oracle recovers an order / folds that reproduce it)."""
    X, y = categorical_case(n=60_000, f=6, seed=12, cardinality=300)
    runs = []
    for seed in (1, 1, 2):
        ds = engine.upload(X, y)
        ds.encode_categorical([2], method, seed=seed)
        runs.append((ds.features()[:, 2].copy(), ds.category_table(2)))
        ds.close()
    assert np.array_equal(_u32(runs[0][0]), _u32(runs[1][0]))
    assert not np.array_equal(_u32(runs[0][0]), _u32(runs[2][0]))
    e = runs[0][0]
    if method == "ordered":
        order = O.recover_order(X, y, 2, e)
        Xo, tab, _ = O.ordered_ts(X, y, [2], order)
    else:
        folds = O.recover_folds(X, y, 2, e, 5)
        Xo, tab, _ = O.cv_ts(X, y, [2], folds, 5)
    assert np.array_equal(_u32(Xo[:, 2]), _u32(e))
    keys, vals = runs[0][1]
    assert np.array_equal(keys, tab[2][0]) and np.array_equal(_u32(vals), _u32(tab[2][1]))
    # class-id labels: the global table does not depend on the draw
    assert np.array_equal(_u32(runs[2][1][1]), _u32(vals))


def test_apply_bins_encodes_test_rows(engine):
    X, y = categorical_case(n=20_000, f=6, seed=21, n_cat=2, cardinality=50)
    order = np.random.default_rng(3).permutation(len(y)).astype(np.uint32)
    Xo, tab, _ = O.ordered_ts(X, y, [2, 4], order)
    ds = engine.upload(X, y)
    ds.encode_categorical([2, 4], "ordered", order=order)
    edges, ne = ds.quantize(255)
    Xt, _ = categorical_case(n=5000, f=6, seed=22, n_cat=2, cardinality=60)  # ids 50..59 unseen
    Xt[:3, 2] = [np.nan, 59.0, 0.0]
    vt = engine.upload(Xt, None)
    vt.apply_bins(ds)
    Et = O.encode_test(Xt, tab)
    assert np.array_equal(_u32(vt.features()), _u32(Et))
    assert Et[1, 2] == np.float32(0.5) and np.isnan(Et[0, 2])
    exp = np.zeros((6, len(Xt)), np.uint8)
    for j in range(6):
        v = Et[:, j]
        b = np.searchsorted(edges[j, :ne[j]], v, side="right")
        b[np.isnan(v)] = 255
        exp[j] = b
    assert np.array_equal(vt.bins(), exp)
    vt.apply_bins(ds)  # a second call bins again but encodes once
    assert np.array_equal(_u32(vt.features()), _u32(Et))
    for h in (vt, ds):
        h.close()


def test_fit_on_target_statistics_matches_reference(engine, capi):
    """The device's fit on its own encoding of the stored run equals the
    reference's model trained on the reference's encoding."""
    g = _fixture()
    X, y = categorical_case()
    hp = O.Hyper(**CAT_HYPER)
    ds = engine.upload(X, y)
    ds.encode_categorical([2], "ordered", order=g["ordered_order"])
    ds.quantize(255)
    tr = engine.trainer(ds, capi.params(loss=hp.loss, n_classes=hp.n_classes, n_estimators=hp.n_estimators,
                                        max_depth=hp.max_depth, max_bins=hp.max_bins,
                                        min_samples_leaf=hp.min_samples_leaf, learning_rate=hp.learning_rate,
                                        lambda_l2=hp.lambda_l2, lambda_l1=hp.lambda_l1,
                                        min_child_weight=hp.min_child_weight, min_split_gain=hp.min_split_gain,
                                        max_delta_step=hp.max_delta_step))
    tr.step(hp.n_estimators)
    m = tr.model()
    ex = m.export()
    ref = O.parse_tcat(g["tcat"].tobytes())
    assert np.array_equal(ex["feature"], ref.feature) and np.array_equal(ex["bin"], ref.bin)
    assert np.array_equal(_u32(ex["threshold"]), _u32(ref.threshold))
    assert np.allclose(ex["leaves"], ref.leaves, rtol=1e-5, atol=1e-6)
    # predictions on encoded rows through tc_predict_dataset = tc_predict on those rows
    vt = engine.upload(X, None)
    vt.apply_bins(ds)
    pd = m.predict_dataset(vt, "sigmoid")
    pe = m.predict(vt.features(), "sigmoid")
    assert np.array_equal(pd, pe)
    for h in (m, tr, vt, ds):
        h.close()


def test_validation_set_encoded_by_training_table(engine, capi):
    """The binding's fit with cat_features and a validation set: the
    validation rows are encoded by tc_apply_bins against the training set
    (valid_data->apply_bins(*train_data_)), and the device's validation loss
    is the logloss of the model's predictions on those encoded rows."""
    X, y = categorical_case(n=8000, f=6, seed=41)
    Xv, yv = categorical_case(n=3000, f=6, seed=42)
    ds = engine.upload(X, y)
    ds.encode_categorical([2], "ordered", seed=3)
    ds.quantize(255)
    vds = engine.upload(Xv, yv)
    vds.apply_bins(ds)
    tr = engine.trainer(ds, capi.params(loss="logloss", n_estimators=15, max_depth=4, learning_rate=0.3))
    tr.set_validation(vds, 1000)
    tr.step(15)
    vl = tr.valid_loss()
    m = tr.model()
    keys, vals = ds.category_table(2)
    Ev = O.encode_test(Xv, {2: (keys, vals)})
    assert np.array_equal(_u32(vds.features()), _u32(Ev))
    p = m.predict(Ev, "sigmoid")[:, 0].astype(np.float64)
    p = np.clip(p, 1e-7, 1 - 1e-7)
    ll = -np.mean(yv * np.log(p) + (1 - yv) * np.log(1 - p))
    assert len(vl) == 15 and abs(vl[-1] - ll) <= 1e-5 * ll
    for h in (m, tr, vds, ds):
        h.close()


def test_encode_rejects_bad_input(engine, capi):
    X, y = categorical_case(n=100, f=4, seed=1)
    ds = engine.upload(X, y)
    for kw in (dict(features=[9]), dict(features=[2, 2]), dict(features=[2], cv_folds=0, method="cv"),
               dict(features=[2], order=np.zeros(100, np.uint32)),
               dict(features=[2], method="cv", order=np.full(100, 5, np.uint32))):
        with pytest.raises(Exception):
            ds.encode_categorical(**kw)
    ds.quantize(255)
    with pytest.raises(Exception):
        ds.encode_categorical([2])  # after binning
    nolab = engine.upload(X, None)
    with pytest.raises(Exception):
        nolab.encode_categorical([2])
    for h in (nolab, ds):
        h.close()


def test_classifier_cat_features(tmp_path):
    """The facade: binary prediction is the reference's no-binning path on the
    raw rows; multiclass prediction encodes the rows with the training set's
    global table first (the binned path)."""
    import turbocat
    from turbocat import _capi, _turbocat

    X, y = categorical_case(n=6000, f=6, seed=31)
    clf = turbocat.TurboCatClassifier(n_estimators=30, max_depth=4, learning_rate=0.2)
    clf.fit(X, y, cat_features=[2])
    p = clf.predict_proba(X)
    clf.save(str(tmp_path / "b.tcat"))
    eng = _capi.Engine(0)
    m = eng.load_tcat(open(tmp_path / "b.tcat", "rb").read())
    assert np.array_equal(p[:, 1], m.predict(X, "sigmoid")[:, 0])
    m.close()

    X3, y3 = categorical_case(n=6000, f=6, n_classes=3, seed=32)
    # the extension class itself: the facade leaves cat_encoding at its default ("ordered")
    c3 = _turbocat.TurboCatClassifier(n_estimators=10, max_depth=4, learning_rate=0.2, cat_encoding="cv",
                                      verbosity=0)
    c3.fit(X3, y3, cat_features=[2])
    p3 = c3.predict_proba(X3)
    c3.save(str(tmp_path / "m.tcat"))
    m3 = eng.load_tcat(open(tmp_path / "m.tcat", "rb").read())
    _, tab, _ = O.cv_ts(X3, y3, [2], np.zeros(len(y3), np.uint32), 5)  # class-id labels: any folds give the table
    assert np.array_equal(p3, m3.predict(O.encode_test(X3, tab), "softmax"))
    m3.close()
    with pytest.raises(ValueError):
        _turbocat.TurboCatClassifier(n_estimators=2, cat_encoding="onehot").fit(X, y, cat_features=[2])
    with pytest.raises(ValueError):
        turbocat.TurboCatClassifier(n_estimators=2).fit(X, y, cat_features=[6])
