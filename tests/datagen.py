"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no public dataset is involved), plus the small
cases the golden fixtures and the parity tests use."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def binary_c1(n=50_000, f=20, seed=1):
    """Binary: X ~ N(0,1); y ~ Bernoulli(sigmoid(w.x + 0.5*x0*x1))."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    w = rng.standard_normal(f)
    s = X.astype(np.float64) @ w + 0.5 * X[:, 0].astype(np.float64) * X[:, 1]
    y = (rng.random(n) < 1.0 / (1.0 + np.exp(-s))).astype(np.float32)
    return X, y


def regression_c2(n=1_000_000, f=100, seed=2):
    """Regression: 60% N(0,1), 30% U(-3,3), 10% Student-t(3) columns;
    y = sum of sin over 10 random features + x2*x3 + N(0, 0.1)."""
    rng = np.random.default_rng(seed)
    a, b = int(round(f * 0.6)), int(round(f * 0.3))
    c = f - a - b
    X = np.concatenate([rng.standard_normal((n, a)), rng.uniform(-3, 3, (n, b)),
                        rng.standard_t(3, (n, c))], axis=1).astype(np.float32)
    S = rng.choice(f, min(10, f), replace=False)
    y = (np.sin(X[:, S].astype(np.float64)).sum(1) + X[:, 2].astype(np.float64) * X[:, 3]
         + rng.normal(0, 0.1, n)).astype(np.float32)
    return X, y


def multiclass_c3(n=2_000_000, f=50, K=10, seed=3):
    """Multiclass: y = argmax of K random projections plus Gumbel noise."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    W = rng.standard_normal((f, K))
    y = np.argmax(X.astype(np.float64) @ W + rng.gumbel(size=(n, K)), axis=1).astype(np.float32)
    return X, y


def imbalanced_c5(n=10_000_000, f=200, seed=5, active=20):
    """Imbalanced: half N(0,1), half LogNormal(0,1); ~1% positives from a
    sparse linear score (20 active features) + N(0, 0.5), thresholded at the
    99th percentile."""
    rng = np.random.default_rng(seed)
    h = f // 2
    X = np.empty((n, f), np.float32)
    X[:, :h] = rng.standard_normal((n, h), dtype=np.float32)
    X[:, h:] = np.exp(rng.standard_normal((n, f - h), dtype=np.float32))
    A = rng.choice(f, min(active, f), replace=False)
    beta = rng.standard_normal(len(A)).astype(np.float32)
    s = X[:, A] @ beta + rng.normal(0, 0.5, n).astype(np.float32)
    y = (s > np.quantile(s, 0.99)).astype(np.float32)
    return X, y


def serving_rows(n, f=100, seed=4):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, f)).astype(np.float32)


# small cases for golden fixtures / CPU-speed parity: name -> spec
GOLDEN_CASES = {
    "c1_small": dict(kind="binary", n=8_000, f=20, seed=11, hyper=dict(loss="logloss", n_estimators=30,
                                                                          learning_rate=0.1, max_depth=6)),
    "c1_odd": dict(kind="binary", n=1003, f=7, seed=12, hyper=dict(loss="logloss", n_estimators=20,
                                                                   learning_rate=0.3, max_depth=4)),
    "c2_small": dict(kind="regression", n=10_000, f=30, seed=13, hyper=dict(loss="mse", n_estimators=20,
                                                                            learning_rate=0.05, max_depth=8,
                                                                            lambda_l2=0.0)),
    "c3_small": dict(kind="multiclass", n=8_000, f=12, K=4, seed=14, hyper=dict(loss="softmax", n_classes=4,
                                                                                n_estimators=5,
                                                                                learning_rate=0.1,
                                                                                max_depth=5)),
    "c5_small": dict(kind="imbalanced", n=15_000, f=16, seed=15, hyper=dict(loss="focal", n_estimators=20,
                                                                            learning_rate=0.1, max_depth=8)),
}


def make_case(spec):
    """(X, y, oracle.Hyper) of a small parity case (imports the oracle: tests only)."""
    if os.path.join(ROOT, "oracle") not in sys.path:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Hyper

    kind = spec["kind"]
    if kind == "binary":
        X, y = binary_c1(spec["n"], spec["f"], spec["seed"])
    elif kind == "regression":
        X, y = regression_c2(spec["n"], spec["f"], spec["seed"])
    elif kind == "multiclass":
        X, y = multiclass_c3(spec["n"], spec["f"], spec["K"], spec["seed"])
    else:
        X, y = imbalanced_c5(spec["n"], spec["f"], spec["seed"], active=min(20, spec["f"]))
    return X, y, Hyper(**spec["hyper"])


def noisy_binary_split(n=3000, nv=2000, f=10, seed=81, noise=2.0):
    """A small noisy binary problem with a held-out validation split: training
    overfits within a few dozen iterations at a high learning rate, so the
    validation loss turns and early stopping fires."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n + nv, f)).astype(np.float32)
    w = rng.standard_normal(f)
    y = ((X @ w + rng.normal(0, noise, n + nv)) > 0).astype(np.float32)
    return X[:n], y[:n], X[n:], y[n:]


def regular_case():
    """Data of the regular-tree golden model: the binary generator with a
    discrete feature (at most 16 bin edges, the reference's linear-scan
    binning at prediction) and NaN values."""
    X, y = binary_c1(3000, 12, seed=41)
    X[:, 5] = np.round(X[:, 5] * 2) / 2
    X[::13, 2] = np.nan
    return X, y


def regular_pred_matrix(X, edges):
    """Prediction rows for the regular-tree golden model: the first 400
    training rows, 200 of them with one feature set exactly to one of its bin
    edges (where the two binning rules of the reference differ)."""
    P = np.array(X[:400], np.float32)
    for r in range(200):
        j = r % P.shape[1]
        e = edges[j]
        if len(e):
            P[r, j] = e[(7 * r) % len(e)]
    return P


def categorical_case(n=3000, f=6, n_classes=2, seed=5, n_cat=1, cardinality=25, nan_rate=0.03):
    """Rows with categorical columns 2, 4, ... (integer category ids, some NaN)
    whose category shifts the label's log-odds, plus standard-normal numeric
    columns; labels are class ids."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, f)).astype(np.float32)
    logit = X[:, 0].astype(np.float64)
    for c in range(n_cat):
        j = 2 + 2 * c
        cat = rng.integers(0, cardinality, n)
        X[:, j] = cat.astype(np.float32)
        X[rng.random(n) < nan_rate, j] = np.nan
        logit = logit + (cat % 7 - 3) * 0.5
    if n_classes == 2:
        y = (rng.random(n) < 1.0 / (1.0 + np.exp(-logit))).astype(np.float32)
    else:
        y = np.clip(np.floor((logit + 4.0) / 8.0 * n_classes + rng.random(n) - 0.5), 0, n_classes - 1)
        y = y.astype(np.float32)
    return X, y


CAT_HYPER = dict(loss="logloss", n_estimators=20, max_depth=4, learning_rate=0.2)


def regular_train_case():
    """Data of the regular-tree training fixture: the binary generator, no NaN
    (the reference's NaN rows spill into the next feature's histogram from
    parallel threads, which makes its own runs differ)."""
    return binary_c1(4000, 10, seed=43)


REGULAR_TRAIN_HYPER = dict(loss="logloss", n_estimators=12, max_depth=7, learning_rate=0.2, regular_trees=True)


def leafwise_case():
    """Data of the leaf-wise (regression preset) fixture: the regression generator."""
    return regression_c2(8000, 12, seed=8000)


LEAFWISE_HYPER = dict(loss="mse", n_estimators=10, max_depth=8, learning_rate=0.1, min_samples_leaf=5,
                      lambda_l2=0.0, regular_trees=True)


def multiclass_regular_case():
    """Data of the multiclass regular-tree fixture: the multiclass generator."""
    return multiclass_c3(4000, 10, 4, seed=7)


MULTICLASS_REGULAR_HYPER = dict(loss="softmax", n_classes=4, n_estimators=5, max_depth=5, learning_rate=0.2,
                                regular_trees=True)
