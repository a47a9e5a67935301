"""Device path vs the oracle, through the C ABI.

Bars (from the task statement):
  * bin indices, per-row leaf indices and chosen (feature, bin) splits are
    bit-exact wherever the reference's top gain beats the runner-up by more
    than 1e-6 relative (the REF32 oracle is bit-identical to the reference);
  * float histograms, leaf values and predictions are within 1e-5 relative.
    "Relative" is taken against the natural scale of each sum, so that sums
    that cancel to ~0 are measured against the magnitude of their terms:
      histogram bin:  |dev - fp64| <= 1e-5 * sum|g_i| over the bin's rows
      leaf value:     |dev - ref|  <= 1e-5 * sum|g_i| / (H + lambda)
      prediction:     |dev - fp64| <= 1e-5 * (|base| + sum_t |w_t * leaf_t(x)|)
"""
import numpy as np
import pytest

import oracle as O
from datagen import GOLDEN_CASES, binary_c1, imbalanced_c5, make_case, multiclass_c3, regression_c2

pytestmark = pytest.mark.gpu

MARGIN = 1e-6
REL = 1e-5


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _params(capi, hp, **kw):
    return capi.params(loss=hp.loss, n_classes=hp.n_classes, n_estimators=hp.n_estimators,
                       max_depth=hp.max_depth, max_bins=hp.max_bins, min_samples_leaf=hp.min_samples_leaf,
                       learning_rate=hp.learning_rate, lambda_l2=hp.lambda_l2, lambda_l1=hp.lambda_l1,
                       min_child_weight=hp.min_child_weight, min_split_gain=hp.min_split_gain,
                       max_delta_step=hp.max_delta_step, **kw)


# ------------------------------------------------------------------ binning --

@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_quantize_matches_reference_fixture(engine, name):
    X, y, hp = make_case(GOLDEN_CASES[name])
    g = np.load(f"{O.HERE}/../tests/golden/{name}.npz")
    ds = engine.upload(X, y)
    edges, ne = ds.quantize(hp.max_bins)
    assert np.array_equal(ne, g["n_edges"])
    assert np.array_equal(edges, g["edges"])  # == on floats: -0.0 / +0.0 edges compare equal
    assert np.array_equal(ds.bins(), g["bins"])


@pytest.mark.parametrize("n,f", [(1, 3), (7, 5), (33, 2), (1000, 17), (4097, 3), (70_000, 9)])
def test_quantize_shapes_and_edge_values(engine, n, f):
    rng = np.random.default_rng(n * 31 + f)
    X = rng.standard_normal((n, f)).astype(np.float32)
    if f > 2:
        X[:, 1] = np.round(X[:, 1] * 3) / 3          # duplicates
        X[rng.random(n) < 0.2, 2] = np.nan           # NaN rows
    if n > 8:
        X[:4, 0] = [-0.0, 0.0, np.inf, -np.inf]
    ds = engine.upload(X)
    for compat in (True, False):
        for mb in (255, 64, 2):
            edges, ne = ds.quantize(mb, compat)
            ob = O.quantize(X, mb, compat)
            assert np.array_equal(ne, ob.n_edges), (mb, compat)
            assert np.array_equal(edges, ob.edges), (mb, compat)
            assert np.array_equal(ds.bins(), ob.bins), (mb, compat)


def test_quantize_all_nan_and_constant(engine):
    X = np.zeros((500, 4), np.float32)
    X[:, 0] = np.nan
    X[:, 1] = 7.0
    X[:, 2] = np.arange(500) % 2
    X[:, 3] = np.arange(300, 800)  # 500 distinct -> 500 mod 256 = 244 bins in compat mode
    ds = engine.upload(X)
    edges, ne = ds.quantize(255)
    ob = O.quantize(X)
    assert np.array_equal(ne, ob.n_edges) and list(ne[:3]) == [1, 0, 1] and ne[3] == 243
    assert np.array_equal(edges, ob.edges)
    assert np.array_equal(ds.bins(), ob.bins)


@pytest.mark.parametrize("n,f", [(1, 3), (1000, 17), (70_000, 40)])
def test_apply_bins_with_training_edges(engine, n, f):
    """A second matrix binned with the first one's edges
    (Dataset::apply_bins, src/core/dataset.cpp:346-379): bin = number of edges
    <= x (upper_bound), NaN -> 255, values outside the training range, +-0
    and +-inf included; bit-exact against the oracle's edges."""
    rng = np.random.default_rng(n + f)
    Xtr = rng.standard_normal((5000, f)).astype(np.float32)
    Xtr[:, 1] = np.round(Xtr[:, 1] * 2) / 2
    ob = O.quantize(Xtr)
    tr = engine.upload(Xtr)
    tr.quantize(255)
    X = (3.0 * rng.standard_normal((n, f))).astype(np.float32)
    X[rng.random(X.shape) < 0.1] = np.nan
    X[0, :] = ob.edges[np.arange(f), np.maximum(ob.n_edges.astype(np.int64) - 1, 0)]  # on an edge
    if n > 4:
        X[1:5, 0] = [-0.0, 0.0, np.inf, -np.inf]
    ds = engine.upload(X)
    ds.apply_bins(tr)
    want = np.zeros((f, n), np.uint8)
    for j in range(f):
        e = ob.edges[j, :ob.n_edges[j]]
        col = X[:, j]
        b = np.searchsorted(e, col, side="right")
        want[j] = np.where(np.isnan(col), 255, b).astype(np.uint8)
    assert np.array_equal(ds.bins(), want)


def test_quantize_full_size_c2_bins(engine):
    X, y = regression_c2()
    ds = engine.upload(X, y)
    edges, ne = ds.quantize(255)
    ob = O.quantize(X)
    assert np.array_equal(ne, ob.n_edges)
    assert np.array_equal(edges, ob.edges)
    assert np.array_equal(ds.bins(), ob.bins)


# --------------------------------------------------------- one tree, forced --

def _check_tree(dev, ref, f64, g, h, hp, lam):
    """Level-by-level split parity under the margin rule; returns the number
    of levels compared.  Leaf values: within 1e-5 of the FP64 oracle, and no
    farther from the reference than the reference's own FP32 summation error
    plus 1e-5 (the reference sums gradients sequentially in FP32, which is off
    by up to ~3e-4 relative on 60k-row nodes)."""
    m = ref.margins()
    checked = 0
    for d in range(ref.depth):
        if m[d] <= MARGIN:
            return checked, False
        assert dev["depth"] > d, d
        assert (int(dev["feature"][d]), int(dev["bin"][d])) == (int(ref.feature[d]), int(ref.bin[d])), d
        assert dev["threshold"][d] == ref.threshold[d]
        checked += 1
    assert dev["depth"] == ref.depth
    # leaf indices
    assert np.array_equal(dev["leaf_index"], ref.leaf_index)
    # leaf values within 1e-5 of the natural scale
    L = 1 << ref.depth
    absg = np.bincount(ref.leaf_index, weights=np.abs(g.astype(np.float64)), minlength=L)
    H = np.bincount(ref.leaf_index, weights=h.astype(np.float64), minlength=L)
    tol = REL * absg / (H + lam) + 1e-7
    dv = dev["leaves"].astype(np.float64)
    assert np.all(np.abs(dv - f64.leaves) <= tol)
    ref_err = np.abs(ref.leaves.astype(np.float64) - f64.leaves)
    assert np.all(np.abs(dv - ref.leaves) <= ref_err + tol)
    return checked, True


@pytest.mark.parametrize("case", ["logloss", "mse", "focal", "deep"])
def test_tree_parity_teacher_forced(engine, capi, case):
    if case == "logloss":
        X, y = binary_c1(50_000, 20, seed=41)
        hp = O.Hyper(loss="logloss", max_depth=6)
    elif case == "mse":
        X, y = regression_c2(60_000, 40, seed=42)
        hp = O.Hyper(loss="mse", max_depth=8, lambda_l2=0.0)
    elif case == "focal":
        # focal hessians are tiny: a small min_child_weight lets the root split
        X, y = imbalanced_c5(60_000, 24, seed=43)
        hp = O.Hyper(loss="focal", max_depth=8, min_child_weight=1e-3)
    else:
        X, y = binary_c1(30_000, 9, seed=44)
        hp = O.Hyper(loss="logloss", max_depth=10, min_child_weight=0.1)
    b = O.quantize(X)
    ds = engine.upload(X, y)
    ds.quantize(255)
    base = O.init_prediction(hp.loss, y)
    rng = np.random.default_rng(7)
    pred = (base + 0.3 * rng.standard_normal(len(y))).astype(np.float32)
    g, h = O.gradients(hp.loss, y, pred)
    ref = O.build_tree(b, g, h, hp, mode=0, want_rows=True)
    f64 = O.build_tree(b, g, h, hp, mode=1, want_rows=True, want_hist=True)
    dev = engine.build_tree(ds, g, h, _params(capi, hp), want_hist=True)
    # root histogram vs FP64 within 1e-5 of sum|g| per bin
    node0 = np.zeros(len(y), np.uint32)
    scale = O.histogram(b, np.abs(g), h, node0, 1)[0]
    diff = np.abs(dev["root_hist"] - f64.root_hist)
    assert np.all(diff[..., 0] <= REL * scale[..., 0] + 1e-9)
    assert np.all(diff[..., 1] <= REL * scale[..., 1] + 1e-9)
    if np.array_equal(ref.feature, f64.feature) and np.array_equal(ref.bin, f64.bin):
        checked, full = _check_tree(dev, ref, f64, g, h, hp, hp.lambda_l2)
    else:
        # the reference's FP32 gains flipped a decision that FP64 makes the
        # other way: the device follows the FP64 arithmetic
        checked, full = _check_tree(dev, f64, f64, g, h, hp, hp.lambda_l2)
    assert checked >= 1
    # device FP64 gains vs the FP64 oracle
    for d in range(checked):
        # gains are differences of larger terms: checked at 1e-4 relative (their
        # role is the argmax, checked above)
        assert abs(dev["gain"][d] - f64.gain_top[d]) <= 1e-4 * abs(f64.gain_top[d]) + 1e-9


def test_partition_skewed_levels(engine, capi):
    """Levels where one node holds more than 1/8 of the rows: the partition
    sums that node's two children in registers and every other child with
    per-warp shared atomics.  The data is checked to have such a level at
    depth >= 3 in the device's own tree; the device's leaf values are checked
    against FP64 sums over the device's own row leaf indices, whatever the
    splits, and the tree against the FP64 oracle under the margin rule."""
    rng = np.random.default_rng(48)
    n, f = 80_000, 12
    X = rng.standard_normal((n, f)).astype(np.float32)
    # the label lives in rare tails: most rows stay in one node, level after level
    y = (((X[:, 0] > 1.8) ^ (X[:, 1] > 2.0)) | (X[:, 2] > 2.2)).astype(np.float32)
    hp = O.Hyper(loss="logloss", max_depth=7, min_child_weight=1e-3)
    b = O.quantize(X)
    pred = np.full(n, O.init_prediction(hp.loss, y), np.float32)
    g, h = O.gradients(hp.loss, y, pred)
    ds = engine.upload(X, y)
    ds.quantize(255)
    dev = engine.build_tree(ds, g, h, _params(capi, hp))
    D = int(dev["depth"])
    li = np.asarray(dev["leaf_index"]).astype(np.int64)
    assert D >= 4
    assert max(np.bincount(li >> (D - d)).max() / n for d in range(3, D)) > 1 / 8
    L = 1 << D
    lam = float(hp.lambda_l2)
    G = np.bincount(li, weights=g.astype(np.float64), minlength=L)
    H = np.bincount(li, weights=h.astype(np.float64), minlength=L)
    absg = np.bincount(li, weights=np.abs(g.astype(np.float64)), minlength=L)
    want = np.where(H >= 1e-10, -G / (H + lam), 0.0)
    tol = REL * absg / (H + lam) + 1e-7
    assert np.all(np.abs(dev["leaves"][:L].astype(np.float64) - want) <= tol)
    ref = O.build_tree(b, g, h, hp, mode=0, want_rows=True)
    f64 = O.build_tree(b, g, h, hp, mode=1, want_rows=True)
    teacher = ref if np.array_equal(ref.feature, f64.feature) and np.array_equal(ref.bin, f64.bin) else f64
    checked, _ = _check_tree(dev, teacher, f64, g, h, hp, lam)
    assert checked >= 3


# ----------------------------------------------------------------- full fit --

def _fit_compare(engine, capi, X, y, hp, batched=1):
    ob = O.quantize(X, hp.max_bins)
    ref = O.fit(ob, y, hp, mode=0)
    ds = engine.upload(X, y)
    ds.quantize(hp.max_bins)
    tr = engine.trainer(ds, _params(capi, hp, batched=batched))
    tr.step(hp.n_estimators)
    m = tr.model()
    ex = m.export()
    return ob, ref, ds, tr, m, ex


@pytest.mark.parametrize("batched", [1, 0])
def test_fit_c1_all_trees_match(engine, capi, batched):
    """Config 1 in full: 50k x 20 binary, 100 trees, depth 6.  Its smallest
    top-vs-runner-up margin is > 1e-6, so every split of every tree must
    match the reference bit for bit."""
    X, y = binary_c1()
    hp = O.Hyper(loss="logloss", n_estimators=100, learning_rate=0.1, max_depth=6, lambda_l2=1.0)
    ob, ref, ds, tr, m, ex = _fit_compare(engine, capi, X, y, hp, batched)
    assert ref.min_margin > MARGIN
    assert np.array_equal(ex["depth"], ref.depth)
    assert np.array_equal(ex["feature"], ref.feature)
    assert np.array_equal(ex["bin"], ref.bin)
    assert np.array_equal(_u32(ex["threshold"]), _u32(ref.threshold))
    # leaves: within 1e-5 of the FP64-arithmetic fit (same splits), and close
    # to the reference up to its own FP32 summation error
    f64 = O.fit(ob, y, hp, mode=1)
    assert np.array_equal(f64.feature, ref.feature)
    assert np.allclose(ex["leaves"], f64.leaves, rtol=REL, atol=1e-6)
    assert np.all(np.abs(ex["leaves"] - ref.leaves) <= np.abs(ref.leaves - f64.leaves) + REL * np.abs(f64.leaves) + 1e-6)
    # predictions: device model vs FP64 oracle on the device's own trees
    dev_e = O.Ensemble(m.info.base_prediction, 1, ex["leaves"].shape[1].bit_length() - 1, ex["depth"],
                       ex["feature"], ex["bin"], ex["threshold"], ex["leaves"], ex["weights"])
    p64 = O.predict(dev_e, X)[:, 0]
    pd = m.predict(X)[:, 0]
    scale = np.abs(m.info.base_prediction) + np.abs(ex["leaves"]).max(1).sum() * 0.1
    assert np.all(np.abs(pd - p64) <= REL * scale)
    # and vs the reference's raw prediction of its own model
    pr = O.predict(ref, X)[:, 0]
    assert np.max(np.abs(pd - pr)) <= 1e-4 * scale
    # train scores
    ts = tr.scores(len(y))[:, 0]
    assert np.allclose(ts, ref.train_pred[:, 0], rtol=1e-5, atol=1e-5 * scale)


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_fit_golden_cases(engine, capi, name):
    """Every tree against the oracle.  Where the reference's FP32 arithmetic
    and FP64 arithmetic choose the same splits (all cases except the focal
    one, whose tiny gradients make the reference's FP32 histogram
    subtraction flip a deep-level choice), the device must match the
    reference bit for bit; everywhere it must match the FP64 oracle's
    trajectory wherever that oracle's margin exceeds 1e-6."""
    X, y, hp = make_case(GOLDEN_CASES[name])
    ob, ref, ds, tr, m, ex = _fit_compare(engine, capi, X, y, hp)
    f64 = O.fit(ob, y, hp, mode=1)
    if f64.min_margin > MARGIN:
        assert np.array_equal(ex["depth"], f64.depth)
        assert np.array_equal(ex["feature"], f64.feature)
        assert np.array_equal(ex["bin"], f64.bin)
        assert np.allclose(ex["leaves"], f64.leaves, rtol=REL, atol=1e-6)
    if ref.min_margin > MARGIN and np.array_equal(f64.feature, ref.feature) and np.array_equal(f64.bin, ref.bin):
        assert np.array_equal(ex["feature"], ref.feature)
        assert np.array_equal(ex["bin"], ref.bin)
        assert np.array_equal(_u32(ex["threshold"]), _u32(ref.threshold))
    K = ref.n_classes
    p = m.predict(X, "raw")
    dev_e = O.Ensemble(m.info.base_prediction, K, m.info.max_depth, ex["depth"], ex["feature"], ex["bin"],
                       ex["threshold"], ex["leaves"], ex["weights"])
    p64 = O.predict(dev_e, X)
    scale = abs(m.info.base_prediction) + (np.abs(ex["leaves"]).max(1) * ex["weights"]).sum() / K
    assert np.max(np.abs(p - p64)) <= REL * scale


def test_multiclass_batched_equals_plain(engine, capi):
    X, y = multiclass_c3(40_000, 12, 5, seed=51)
    hp = O.Hyper(loss="softmax", n_classes=5, n_estimators=6, learning_rate=0.1, max_depth=6)
    outs = []
    for batched in (1, 0):
        ds = engine.upload(X, y)
        ds.quantize(255)
        tr = engine.trainer(ds, _params(capi, hp, batched=batched))
        tr.step(hp.n_estimators)
        outs.append(tr.model().export())
    a, b = outs
    assert np.array_equal(a["feature"], b["feature"]) and np.array_equal(a["bin"], b["bin"])
    assert np.allclose(a["leaves"], b["leaves"], rtol=1e-6, atol=1e-7)


# --------------------------------------------------------- predict and TCAT --

def test_predict_reference_model_from_tcat(engine):
    g = np.load(f"{O.HERE}/../tests/golden/c1_small.npz")
    X, y, hp = make_case(GOLDEN_CASES["c1_small"])
    m = engine.load_tcat(g["tcat"].tobytes())
    p = m.predict(X)[:, 0]
    r = O.parse_tcat(g["tcat"].tobytes())
    p64 = O.predict(r, X)[:, 0]
    scale = abs(r.base) + (np.abs(r.leaves).max(1) * r.weights).sum()
    assert np.max(np.abs(p - p64)) <= REL * scale
    assert np.max(np.abs(p - g["pred_raw"])) <= REL * scale
    # round trip: the device writer emits the same stream the reference wrote
    assert m.tcat() == g["tcat"].tobytes()


def test_predict_nan_and_edges(engine):
    rng = np.random.default_rng(3)
    T, D, F = 37, 7, 11
    info_arrays = dict(depth=rng.integers(0, D + 1, T).astype(np.int32),
                       feature=rng.integers(0, F, (T, D)).astype(np.uint16),
                       threshold=rng.standard_normal((T, D)).astype(np.float32),
                       leaves=rng.standard_normal((T, 1 << D)).astype(np.float32),
                       weights=np.full(T, 0.1, np.float32))
    from turbocat import _capi
    info = _capi.ModelInfo(T, 1, D, F, 0, 0.25, 0.1, 1.0)
    m = engine.import_model(info, info_arrays)
    X = rng.standard_normal((1000, F)).astype(np.float32)
    X[rng.random(X.shape) < 0.1] = np.nan
    X[0, :] = info_arrays["threshold"][0, 0]  # exactly on a threshold: goes right
    e = O.Ensemble(0.25, 1, D, info_arrays["depth"], info_arrays["feature"], np.zeros((T, D), np.uint8),
                   info_arrays["threshold"], info_arrays["leaves"], info_arrays["weights"])
    p64 = O.predict(e, X)[:, 0]
    for tr_, fn in (("raw", lambda v: v), ("sigmoid", lambda v: 1 / (1 + np.exp(-v)))):
        p = m.predict(X, tr_)[:, 0]
        assert np.max(np.abs(p - fn(p64))) <= 1e-5 * (0.25 + np.abs(info_arrays["leaves"]).max(1).sum() * 0.1)


@pytest.mark.parametrize("D,K,F", [(1, 1, 1), (4, 1, 9), (6, 1, 100), (7, 1, 1), (8, 3, 20), (10, 1, 13),
                                   (11, 1, 7), (13, 2, 5)])
def test_predict_tile_shapes(engine, D, K, F):
    """Every walk of the predict kernels against FP64: trees of every depth up
    to D (padded on the device), NaN inputs and thresholds, values on
    thresholds, a feature with more than 127 distinct thresholds (two virtual
    features of the binned form), request sizes around the tile (128 rows)
    boundary, and the small-request path (at most 64 rows)."""
    rng = np.random.default_rng(100 + D)
    T = K * (3 if D >= 11 else 29)
    depth = rng.integers(0, D + 1, T).astype(np.int32)
    depth[0] = D
    arrays = dict(depth=depth, feature=rng.integers(0, F, (T, D)).astype(np.uint16),
                  threshold=rng.standard_normal((T, D)).astype(np.float32),
                  leaves=rng.standard_normal((T, 1 << D)).astype(np.float32),
                  weights=rng.uniform(0.05, 0.2, T).astype(np.float32))
    arrays["threshold"][rng.random((T, D)) < 0.03] = np.nan  # x >= NaN is false
    arrays["threshold"][0, 0] = 0.25
    from turbocat import _capi
    m = engine.import_model(_capi.ModelInfo(T, K, D, F, 1 if K > 1 else 0, -0.5, 0.1, 1.0), arrays)
    e = O.Ensemble(-0.5, K, D, depth, arrays["feature"], np.zeros((T, D), np.uint8), arrays["threshold"],
                   arrays["leaves"], arrays["weights"])
    scale = 0.5 + (np.abs(arrays["leaves"]).max(1) * arrays["weights"]).sum() / K
    X = rng.standard_normal((1000, F)).astype(np.float32)
    X[rng.random(X.shape) < 0.08] = np.nan
    X[1, arrays["feature"][0, 0]] = 0.25  # on a threshold: goes right
    X[2, :] = -0.0
    p64_all = O.predict(e, X)
    for n in (1, 5, 32, 33, 64, 65, 127, 128, 129, 300, 1000):
        p = m.predict(X[:n], "raw")
        assert p.shape == (n, K)
        assert np.max(np.abs(p - p64_all[:n])) <= 1e-5 * scale, n


def test_bad_tcat_is_rejected(engine, capi):
    g = np.load(f"{O.HERE}/../tests/golden/c1_small.npz")
    data = g["tcat"].tobytes()
    for bad in (b"XCAT" + data[4:], data[: len(data) // 2], data[:20]):
        with pytest.raises(capi.TCError) as ei:
            engine.load_tcat(bad)
        assert ei.value.status == 6


# ---------------------------------------------- tile shapes and the tuner --

@pytest.mark.parametrize("width,rows", [(32, 0), (64, 0), (32, 700), (64, 700), (32, 5000)])
def test_fit_identical_across_histogram_tilings(engine, capi, width, rows):
    """Every histogram tiling (rows per chunk; the group width is fixed at 32)
    must grow the same trees: a tiling changes only the fixed-point scale of
    each work item (the sums themselves are exact)."""
    X, y = regression_c2(40_000, 70, seed=61)
    hp = O.Hyper(loss="mse", n_estimators=6, learning_rate=0.1, max_depth=7, lambda_l2=0.0)
    ob = O.quantize(X)
    f64 = O.fit(ob, y, hp, mode=1)
    ds = engine.upload(X, y)
    ds.quantize(255)
    tr = engine.trainer(ds, _params(capi, hp, hist_features_per_block=width, hist_rows_per_chunk=rows))
    tr.step(hp.n_estimators)
    st = tr.stats()
    assert st.hist_features_per_block == 32  # the only group width (64 is accepted and means 32)
    ex = tr.model().export()
    assert f64.min_margin > MARGIN
    assert np.array_equal(ex["feature"], f64.feature) and np.array_equal(ex["bin"], f64.bin)
    assert np.allclose(ex["leaves"], f64.leaves, rtol=REL, atol=1e-6)


def test_autotuner_and_profile(engine, capi):
    X, y = binary_c1(30_000, 40, seed=62)
    ds = engine.upload(X, y)
    ds.quantize(255)
    tr = engine.trainer(ds, capi.params(loss="logloss", n_estimators=12, max_depth=6))
    st = tr.stats()
    assert st.hist_features_per_block in (32, 64) and st.iterations_done == 0 and st.kernel_launches == 0
    tr.step(4)
    prof = tr.profile(3)
    levels = prof.pop("_hist_levels")
    part_levels = prof.pop("_part_levels")
    # timed inside the replayed graph: the kernels fill most of the iteration
    assert prof.pop("_in_graph")
    it_ms = prof.pop("_iteration_ms")
    kern_ms = sum(v[1] for v in prof.values())
    assert 0.5 * it_ms <= kern_ms <= it_ms * 1.001 + 1e-3
    assert all(part_levels[d] > 0 for d in range(6))  # depth 6: a partition launch per level
    assert prof["hist"][0] == 3 * 6 and prof["hist"][1] > 0 and prof["hist"][2] > 0
    assert levels[0][1] == 3 * 30_000  # root rows histogrammed per profiled iteration
    assert tr.stats().iterations_done == 7
    # the tuned model equals an untuned one on the same data
    ref = O.fit(O.quantize(X), y, O.Hyper(loss="logloss", n_estimators=7, max_depth=6), mode=1)
    ex = tr.model().export()
    if ref.min_margin > MARGIN:
        assert np.array_equal(ex["feature"], ref.feature)


def test_predict_regular_model_from_reference(engine, capi, tmp_path):
    """A model of regular (depth-wise) trees trained by the reference
    (mode="small", tests/golden/make_golden.py) served on the device: the
    reference's own predictions (stored in the fixture) bit for bit (the same
    binning, node walk and FP32 fused multiply-adds in tree order), through
    tc_predict (tile and small requests) and the facade; the stream saves
    back byte for byte; the model has no symmetric export and the server
    refuses it."""
    from datagen import regular_case, regular_pred_matrix

    g = np.load(f"{O.HERE}/../tests/golden/regular_small.npz")
    data = g["tcat"].tobytes()
    rm = O.parse_tcat_regular(data)
    X, _ = regular_case()
    P = regular_pred_matrix(X, rm.edges)
    want = g["pred_raw"]
    scale = abs(rm.base) + sum(float(np.abs(t["value"]).max()) * float(w) for t, w in zip(rm.trees, rm.weights))
    m = engine.load_tcat(data)
    assert m.info.n_trees == 40 and m.info.n_features == P.shape[1]
    raw = m.predict(P, "raw")[:, 0]
    assert np.array_equal(raw, want)
    for n in (1, 5, 64, 65):
        assert np.array_equal(m.predict(P[:n], "raw")[:, 0], want[:n]), n
    p64 = O.predict_regular(rm, P, fp64=True)
    assert np.max(np.abs(raw - p64)) <= 1e-6 * scale
    prob = m.predict(P, "sigmoid")[:, 0]
    assert np.max(np.abs(prob - 1.0 / (1.0 + np.exp(-want.astype(np.float64))))) <= 1e-6
    assert m.tcat() == data
    with pytest.raises(capi.TCError):
        m.export()
    srv = capi.Server(engine)
    with pytest.raises(capi.TCError):
        srv.add_model(m)
    srv.close()
    import turbocat

    path = str(tmp_path / "regular.tcat")
    with open(path, "wb") as fh:
        fh.write(data)
    clf = turbocat.TurboCatClassifier(verbosity=0).load(path)
    p1 = clf.predict_proba(P)[:, 1]
    assert np.max(np.abs(p1 - 1.0 / (1.0 + np.exp(-want.astype(np.float64))))) <= 1e-6
