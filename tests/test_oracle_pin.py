"""The oracle against the reference: golden fixtures generated by running the
reference build (tests/golden/make_golden.py), and -- where the reference
build is present -- direct runs of the reference on fresh seeds."""
import numpy as np
import pytest

import oracle as O
from datagen import GOLDEN_CASES, binary_c1, make_case, noisy_binary_split, regression_c2


def _u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference_fixture(name):
    X, y, hp = make_case(GOLDEN_CASES[name])
    g = np.load(f"{O.HERE}/../tests/golden/{name}.npz")
    b = O.quantize(X, hp.max_bins)
    assert np.array_equal(b.bins, g["bins"])
    assert np.array_equal(b.n_edges, g["n_edges"])
    assert np.array_equal(_u32(b.edges), _u32(g["edges"]))
    e = O.fit(b, y, hp, mode=O.__dict__.get("REF32", 0), trace=True)
    if hp.loss == "softmax":
        assert np.array_equal(e.depth, g["depth"])
        assert np.array_equal(e.feature, g["feature"])
        assert np.array_equal(e.bin, g["bin"])
        assert np.array_equal(_u32(e.threshold), _u32(g["threshold"]))
        assert np.array_equal(_u32(e.leaves), _u32(g["leaves"]))
        assert np.array_equal(_u32(e.train_pred), _u32(g["train_raw"]))
    else:
        r = O.parse_tcat(g["tcat"].tobytes())
        assert r.base == e.base
        assert np.array_equal(r.depth, e.depth)
        assert np.array_equal(r.feature, e.feature)
        assert np.array_equal(r.bin, e.bin)
        assert np.array_equal(_u32(r.threshold), _u32(e.threshold))
        assert np.array_equal(_u32(r.gain), _u32(e.gain))
        assert np.array_equal(_u32(r.leaves), _u32(e.leaves))
        # gradients of the first and last iteration, bit for bit
        assert np.array_equal(_u32(e.grad_trace[0, :, 0]), _u32(g["grad0"]))
        assert np.array_equal(_u32(e.hess_trace[0, :, 0]), _u32(g["hess0"]))
        assert np.array_equal(_u32(e.grad_trace[-1, :, 0]), _u32(g["grad_last"]))
        assert np.array_equal(_u32(e.hess_trace[-1, :, 0]), _u32(g["hess_last"]))
        # FP64 prediction of the reference's own model vs its FP32 predictor
        p64 = O.predict(r, X)[:, 0]
        assert np.allclose(p64, g["pred_raw"], rtol=1e-5, atol=1e-5)


def test_fp64_mode_agrees_with_ref32():
    X, y = binary_c1(6000, 10, seed=21)
    hp = O.Hyper(loss="logloss", n_estimators=1, max_depth=6)
    b = O.quantize(X)
    g, h = O.gradients("logloss", y, np.full(len(y), O.init_prediction("logloss", y), np.float32))
    t32 = O.build_tree(b, g, h, hp, mode=0)
    t64 = O.build_tree(b, g, h, hp, mode=1)
    m = t32.margins()
    for d in range(t32.depth):
        if m[d] <= 1e-6:
            break
        assert (t32.feature[d], t32.bin[d]) == (t64.feature[d], t64.bin[d])
    assert np.allclose(t32.leaves, t64.leaves, rtol=1e-4, atol=1e-6)


def test_quantize_edge_cases():
    rng = np.random.default_rng(5)
    X = rng.standard_normal((600, 8)).astype(np.float32)
    X[:, 1] = 3.0                       # constant column: no edges
    X[:, 2] = np.where(rng.random(600) < 0.3, np.nan, X[:, 2])  # NaN rows -> bin 255
    X[:, 3] = np.nan                    # all NaN: one edge {0}, every bin 255
    X[:, 4] = np.round(X[:, 4] * 2) / 2  # heavy duplicates
    X[:5, 5] = [-0.0, 0.0, np.inf, -np.inf, 0.0]
    X[:, 6] = rng.integers(0, 2, 600)   # boolean column
    b = O.quantize(X)
    assert b.n_edges[1] == 0 and np.all(b.bins[1] == 0)
    assert np.all(b.bins[2][np.isnan(X[:, 2])] == 255)
    assert b.n_edges[3] == 1 and b.edges[3, 0] == 0.0 and np.all(b.bins[3] == 255)
    assert list(b.edge_list(6)) == [1.0]
    if O.ref_available():
        r = O.ref_quantize(X)
        for j in range(8):
            if j in (2, 3):  # NaN bins: the reference writes max_bins (=255) too
                pass
            assert np.array_equal(b.bins[j], r.bins[j]), j
            assert np.array_equal(b.edge_list(j), r.edge_list(j)), j


def test_uint8_truncation_of_unique_count():
    # 300 distinct values: the reference keeps min(255, 300 mod 256) = 44 bins
    X = np.arange(300, dtype=np.float32).reshape(-1, 1)
    b = O.quantize(X)
    assert b.n_edges[0] == 43
    b2 = O.quantize(X, compat_u8=False)
    assert b2.n_edges[0] == 254
    X2 = np.arange(257, dtype=np.float32).reshape(-1, 1)  # 257 mod 256 = 1 -> no edges
    assert O.quantize(X2).n_edges[0] == 0


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", [31, 32])
def test_oracle_matches_reference_live(seed):
    X, y = regression_c2(5000, 12, seed=seed)
    hp = O.Hyper(loss="mse", n_estimators=8, learning_rate=0.05, max_depth=8, lambda_l2=0.0)
    rb, model, gt, ht, _ = O.ref_fit(X, y, hp, trace=True)
    b = O.quantize(X)
    e = O.fit(b, y, hp, mode=0, trace=True)
    r = O.parse_tcat(model)
    assert np.array_equal(rb.bins, b.bins)
    assert np.array_equal(r.feature, e.feature) and np.array_equal(r.bin, e.bin)
    assert np.array_equal(_u32(r.leaves), _u32(e.leaves))
    assert np.array_equal(_u32(gt), _u32(e.grad_trace[:, :, 0]))


_ES_SCRIPT = r"""
import sys
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import numpy as np
import _turbocat as ref
from datagen import noisy_binary_split
Xt, yt, Xv, yv = noisy_binary_split()
m = ref.TurboCatClassifier(n_estimators=200, learning_rate=0.3, max_depth=6, max_bins=255, subsample=1.0,
                           colsample_bytree=1.0, min_child_weight=1.0, lambda_l2=1.0, loss="logloss",
                           mode="large", early_stopping_rounds=10, verbosity=0)
m.fit(Xt, yt, Xv, yv)
print(m.n_trees)
"""


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_early_stopping_replay_matches_reference():
    """The oracle's replay of the validation/early-stopping rule over its own
    (reference-identical) trees stops where the reference's fit with a
    validation set stops.  The reference runs in a process of its own (one
    fit per process)."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    out = subprocess.run([sys.executable, "-c", _ES_SCRIPT, here, os.path.join(O.HERE, "_ref")],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    ref_trees = int(out.stdout.strip().splitlines()[-1])
    Xt, yt, Xv, yv = noisy_binary_split()
    hp = O.Hyper(loss="logloss", n_estimators=200, learning_rate=0.3, max_depth=6, lambda_l2=1.0)
    e = O.fit(O.quantize(Xt), yt, hp, mode=0)
    losses, stop, best = O.early_stopping(e, Xv, yv, "logloss", 200, 10, 0.3)
    assert stop >= 50 and best < stop  # the rule fired after the minimum iterations
    assert ref_trees == stop + 1


_SS_SCRIPT = r"""
import sys, os, tempfile
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import _turbocat as ref
from datagen import binary_c1
X, y = binary_c1(20000, 12, seed=91)
m = ref.TurboCatClassifier(n_estimators=6, learning_rate=0.1, max_depth=5, max_bins=255, subsample=0.8,
                           colsample_bytree=0.8, min_child_weight=1.0, lambda_l2=1.0, loss="logloss",
                           mode="large", verbosity=0, seed=42)
m.fit(X, y)
path = os.path.join(tempfile.mkdtemp(), "m.tcat")
m.save(path)
sys.stdout.write(path)
"""


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_row_sampling_matches_reference():
    """subsample = colsample_bytree = 0.8 (the facade's defaults), seed 42:
    the oracle's row sampling (xorshift64* draws, std::shuffle with
    std::mt19937_64, trees built over the sampled rows in their shuffled
    order) reproduces the reference's fit bit for bit."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    out = subprocess.run([sys.executable, "-c", _SS_SCRIPT, here, os.path.join(O.HERE, "_ref")],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    r = O.parse_tcat(open(out.stdout.strip().splitlines()[-1], "rb").read())
    X, y = binary_c1(20000, 12, seed=91)
    hp = O.Hyper(loss="logloss", n_estimators=6, learning_rate=0.1, max_depth=5, lambda_l2=1.0, subsample=0.8,
                 colsample_bytree=0.8, seed=42)
    e = O.fit(O.quantize(X), y, hp, mode=0)
    assert np.array_equal(r.feature, e.feature) and np.array_equal(r.bin, e.bin)
    assert np.array_equal(_u32(r.leaves), _u32(e.leaves))
    full = O.fit(O.quantize(X), y, O.Hyper(loss="logloss", n_estimators=6, learning_rate=0.1, max_depth=5,
                                           lambda_l2=1.0), mode=0)
    assert not np.array_equal(full.leaves, e.leaves)  # sampling changed the trees


_GOSS_SCRIPT = r"""
import sys, os, tempfile
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import _turbocat as ref
from datagen import binary_c1
X, y = binary_c1(20000, 12, seed=91)
m = ref.TurboCatClassifier(n_estimators=6, learning_rate=0.1, max_depth=5, max_bins=255, subsample=1.0,
                           colsample_bytree=0.8, min_child_weight=1.0, lambda_l2=1.0, loss="logloss",
                           mode="large", verbosity=0, seed=42, use_goss=True, goss_top_rate=0.2,
                           goss_other_rate=0.1)
m.fit(X, y)
path = os.path.join(tempfile.mkdtemp(), "m.tcat")
m.save(path)
sys.stdout.write(path)
"""


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_goss_matches_reference():
    """use_goss with the facade's rates (top 0.2, other 0.1), colsample_bytree
    0.8, seed 42: the oracle's GOSS (std::nth_element over (|g|, row), a
    partial Fisher-Yates shuffle of the rest with std::mt19937_64, trees
    built over the sampled rows in that order) reproduces the reference's
    fit bit for bit."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    out = subprocess.run([sys.executable, "-c", _GOSS_SCRIPT, here, os.path.join(O.HERE, "_ref")],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    r = O.parse_tcat(open(out.stdout.strip().splitlines()[-1], "rb").read())
    X, y = binary_c1(20000, 12, seed=91)
    hp = O.Hyper(loss="logloss", n_estimators=6, learning_rate=0.1, max_depth=5, lambda_l2=1.0,
                 colsample_bytree=0.8, seed=42, use_goss=True, goss_top_rate=0.2, goss_other_rate=0.1)
    e = O.fit(O.quantize(X), y, hp, mode=0)
    assert np.array_equal(r.feature, e.feature) and np.array_equal(r.bin, e.bin)
    assert np.array_equal(_u32(r.leaves), _u32(e.leaves))
    full = O.fit(O.quantize(X), y, O.Hyper(loss="logloss", n_estimators=6, learning_rate=0.1, max_depth=5,
                                           lambda_l2=1.0), mode=0)
    assert not np.array_equal(full.leaves, e.leaves)  # the sample changed the trees


def test_goss_selection_properties():
    """The oracle's GOSS selection: the top rows are the largest |g| (ties
    aside), the other rows come from the rest, counts as the reference
    computes them (uint32)(n * rate), and the same seed gives the same rows."""
    rng = np.random.default_rng(5)
    n = 10_007
    absg = np.abs(rng.standard_normal(n)).astype(np.float32)
    rows = O.goss_subsample(absg, 0.2, 0.1, 1234)
    top_n, other_n = int(np.float32(n) * np.float32(0.2)), int(np.float32(n) * np.float32(0.1))
    assert len(rows) == top_n + other_n and len(np.unique(rows)) == len(rows)
    thr = np.sort(absg)[::-1][top_n - 1]
    assert np.all(absg[rows[:top_n]] >= thr) and np.all(absg[rows[top_n:]] <= thr)
    assert np.array_equal(rows, O.goss_subsample(absg, 0.2, 0.1, 1234))
    assert not np.array_equal(rows[top_n:], O.goss_subsample(absg, 0.2, 0.1, 1235)[top_n:])
    assert len(O.goss_subsample(absg, 0.0, 0.0, 1)) == 0
    assert len(O.goss_subsample(absg, 1.0, 0.5, 1)) == n  # all rows on top, nothing else to draw
    assert len(O.goss_subsample(absg, 0.0, 0.3, 1)) == int(np.float32(n) * np.float32(0.3))
