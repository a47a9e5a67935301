"""Device training at the benchmark configurations' full sizes against the
oracle, tree by tree, with the error of every result against FP64.

Each device iteration is replayed on the CPU from the device's own training
scores before it: the oracle computes that iteration's gradients (the
reference's formulas) and builds the tree twice, in the reference's FP32
arithmetic (REF32, bit-identical to the reference) and in FP64.  Checked:

  * splits: the device's tree equals the FP64 tree level by level wherever
    the FP64 top gain beats the runner-up by more than 1e-6 relative (up to
    the first level where it does not); the levels where it also equals
    REF32 are counted;
  * the device's tree builder given the same gradients (tc_build_tree)
    chooses the same splits as the trainer's tree;
  * root histograms within 1e-5 of each bin's sum |g| of the FP64 histogram;
  * gains of the matched levels within 1e-4 relative of FP64 (they are
    differences of larger terms; the argmax is checked above);
  * leaf values of fully matched trees within 1e-5 of sum |g| / (H + lambda);
  * predictions of the device's ensemble within 1e-5 of the FP64 oracle's
    prediction of the same ensemble (relative to |base| + sum |w * leaf|).

The measured maxima (and where REF32 and FP64 choose differently) are written
to the JSON file named by $TURBOCAT_PARITY_REPORT when it is set.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from datagen import imbalanced_c5, multiclass_c3, regression_c2

pytestmark = pytest.mark.gpu

MARGIN = 1e-6
REL = 1e-5
GAIN_REL = 1e-4


def _params(capi, hp, **kw):
    return capi.params(loss=hp.loss, n_classes=hp.n_classes, n_estimators=hp.n_estimators,
                       max_depth=hp.max_depth, max_bins=hp.max_bins, min_samples_leaf=hp.min_samples_leaf,
                       learning_rate=hp.learning_rate, lambda_l2=hp.lambda_l2, lambda_l1=hp.lambda_l1,
                       min_child_weight=hp.min_child_weight, min_split_gain=hp.min_split_gain,
                       max_delta_step=hp.max_delta_step, **kw)


def _report(name, rec):
    path = os.environ.get("TURBOCAT_PARITY_REPORT")
    if not path:
        return
    data = {}
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[name] = rec
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1)


class Errors:
    def __init__(self):
        self.hist = 0.0
        self.gain = 0.0
        self.leaf = 0.0
        self.pred = 0.0
        self.levels_checked = 0
        self.trees_full = 0
        self.trees = 0
        self.ref_fp64_split_diff = []   # (iteration, class, level): first level where REF32 and FP64 differ
        self.below_margin = []          # (iteration, class, level): comparison stops (FP64 margin <= 1e-6)
        self.dev_eq_ref32_levels = 0    # compared levels where the device also equals REF32


def _hist_err(dev, f64, absg, absh):
    dg = np.abs(dev[..., 0] - f64[..., 0])
    dh = np.abs(dev[..., 1] - f64[..., 1])
    eg = np.where(absg > 0, dg / np.where(absg > 0, absg, 1.0), np.where(dg > 0, np.inf, 0.0))
    eh = np.where(absh > 0, dh / np.where(absh > 0, absh, 1.0), np.where(dh > 0, np.inf, 0.0))
    return float(max(eg.max(), eh.max()))


def _check_one_tree(E, key, engine, capi, ds, b, g, h, hp, dev_tree, want_hist):
    """One device tree (from the trainer) against the oracle's trees built
    from the same gradients; updates the error maxima."""
    lam = float(hp.lambda_l2)
    one = O.Hyper(**{**hp.__dict__, "loss": "mse" if hp.loss == "softmax" else hp.loss, "n_classes": 1})
    ref = O.build_tree(b, g, h, one, mode=0, want_rows=False)
    f64 = O.build_tree(b, g, h, one, mode=1, want_rows=True, want_hist=want_hist)
    E.trees += 1
    rm = ref.margins()
    for d in range(min(ref.depth, f64.depth)):
        if (int(ref.feature[d]), int(ref.bin[d])) != (int(f64.feature[d]), int(f64.bin[d])):
            # the reference's own margin at that level: above 1e-6, its FP32
            # arithmetic (not a near tie) decides differently from FP64
            E.ref_fp64_split_diff.append((*key, d, float(rm[d])))
            break
    # the device's builder on the same gradients: same splits as the trainer's tree
    bt = engine.build_tree(ds, g, h, _params(capi, one), want_hist=want_hist)
    m = f64.margins()
    full = True
    for d in range(f64.depth):
        if m[d] <= MARGIN:
            E.below_margin.append((*key, d))
            full = False
            break
        assert dev_tree["depth"] > d, (key, d)
        got = (int(dev_tree["feature"][d]), int(dev_tree["bin"][d]))
        assert got == (int(f64.feature[d]), int(f64.bin[d])), (key, d, got, f64.feature[d], f64.bin[d])
        assert (int(bt["feature"][d]), int(bt["bin"][d])) == got, (key, d)
        assert dev_tree["threshold"][d] == f64.threshold[d]
        if d < ref.depth and (int(ref.feature[d]), int(ref.bin[d])) == got:
            E.dev_eq_ref32_levels += 1
        top = float(f64.gain_top[d])
        e = abs(float(bt["gain"][d]) - top) / max(abs(top), 1e-300)
        E.gain = max(E.gain, e)
        assert e <= GAIN_REL, (key, d, e)
        E.levels_checked += 1
    if full:
        assert dev_tree["depth"] == f64.depth, key
        L = 1 << f64.depth
        absg = np.bincount(f64.leaf_index, weights=np.abs(g.astype(np.float64)), minlength=L)
        H = np.bincount(f64.leaf_index, weights=h.astype(np.float64), minlength=L)
        unit = absg / (H + lam) + 1e-7 / REL
        dv = dev_tree["leaves"][:L].astype(np.float64)
        err = float(np.max(np.abs(dv - f64.leaves[:L]) / unit))
        E.leaf = max(E.leaf, err)
        assert err <= REL, (key, err)
        assert np.array_equal(bt["leaf_index"], f64.leaf_index), key
        E.trees_full += 1
    if want_hist:
        node0 = np.zeros(len(g), np.uint32)
        sc = O.histogram(b, np.abs(g), h, node0, 1)[0]
        e = _hist_err(bt["root_hist"], f64.root_hist, sc[..., 0], sc[..., 1])
        E.hist = max(E.hist, e)
        assert e <= REL, (key, e)


def _run(engine, capi, name, X, y, hp, hist_every=1, check=None):
    """Trains hp.n_estimators iterations; the iterations in `check` (default:
    all) are compared with the oracle."""
    check = set(range(hp.n_estimators) if check is None else check)
    b = O.quantize(X, hp.max_bins)
    ds = engine.upload(X, y)
    ds.quantize(hp.max_bins)
    assert np.array_equal(ds.bins(), b.bins), "bins differ from the oracle"
    K = hp.n_classes if hp.loss == "softmax" else 1
    tr = engine.trainer(ds, _params(capi, hp))
    n = len(y)
    E = Errors()
    for it in range(hp.n_estimators):
        if it not in check:
            tr.step(1)
            continue
        pred = tr.scores(n)       # the scores this iteration's gradients come from [n][K]
        tr.step(1)
        ex = tr.model().export()
        if hp.loss == "softmax":
            g_all, h_all = O.gradients("softmax", y, pred, K)
        else:
            g_all, h_all = O.gradients(hp.loss, y, pred[:, 0])
            g_all, h_all = g_all[:, None], h_all[:, None]
        for k in range(K):
            t = it * K + k
            dev_tree = dict(depth=int(ex["depth"][t]), feature=ex["feature"][t], bin=ex["bin"][t],
                            threshold=ex["threshold"][t], leaves=ex["leaves"][t])
            g = np.ascontiguousarray(g_all[:, k])
            h = np.ascontiguousarray(h_all[:, k])
            _check_one_tree(E, (it, k), engine, capi, ds, b, g, h, hp, dev_tree, want_hist=(it % hist_every == 0))
    # predictions of the device's ensemble vs the FP64 oracle's prediction of it
    m = tr.model()
    ex = m.export()
    p = m.predict(X, "raw")
    ens = O.Ensemble(m.info.base_prediction, K, m.info.max_depth, ex["depth"], ex["feature"], ex["bin"],
                     ex["threshold"], ex["leaves"], ex["weights"])
    p64 = O.predict(ens, X)
    scale = abs(m.info.base_prediction) + (np.abs(ex["leaves"]).max(1) * ex["weights"]).sum() / K
    E.pred = float(np.max(np.abs(p - p64)) / scale)
    rec = {"rows": int(n), "features": int(X.shape[1]), "classes": K, "iterations_checked": sorted(check),
           "trees": E.trees,
           "levels_compared": E.levels_checked, "levels_device_equals_ref32": E.dev_eq_ref32_levels,
           "trees_fully_matched": E.trees_full,
           "max_rel_err": {"histogram_root": E.hist, "gain": E.gain, "leaf": E.leaf, "prediction": E.pred},
           "ref32_vs_fp64_first_split_difference": E.ref_fp64_split_diff,
           "ref32_vs_fp64_differences_above_ref_margin": sum(1 for v in E.ref_fp64_split_diff if v[-1] > MARGIN),
           "comparison_stopped_below_margin": E.below_margin}
    _report(name, rec)
    print(name, json.dumps(rec))
    assert E.pred <= REL
    assert E.levels_checked >= E.trees  # on average at least one compared level per tree
    return rec


def test_scale_parity_regression_c2(engine, capi):
    """1M x 100 regression, MSE, depth 8: the first 20 trees."""
    X, y = regression_c2()
    hp = O.Hyper(loss="mse", n_estimators=20, learning_rate=0.05, max_depth=8, lambda_l2=0.0)
    _run(engine, capi, "c2_regression_1M_x_100", X, y, hp, hist_every=5)


def test_scale_parity_multiclass_c3(engine, capi):
    """2M x 50 softmax with 10 classes, depth 6: the first 3 iterations (30 trees)."""
    X, y = multiclass_c3()
    hp = O.Hyper(loss="softmax", n_classes=10, n_estimators=3, learning_rate=0.1, max_depth=6, lambda_l2=1.0)
    _run(engine, capi, "c3_multiclass_2M_x_50_K10", X, y, hp, hist_every=3)


def test_scale_parity_focal_c5(engine, capi):
    """10M x 200 focal loss, depth 8: the first 3 trees and trees 200-202
    (the first trees stop early: focal hessians are tiny, and the
    min_child_weight rule ends them after a level or two)."""
    X, y = imbalanced_c5()
    hp = O.Hyper(loss="focal", n_estimators=203, learning_rate=0.1, max_depth=8, lambda_l2=1.0)
    _run(engine, capi, "c5_focal_10M_x_200", X, y, hp, hist_every=1, check=[0, 1, 2, 200, 201, 202])
