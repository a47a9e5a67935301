"""The categorical target-statistics oracle pinned to the reference.

The reference draws its processing order (ordered method) and its folds
(cross-validated method) from std::random_device, so no two of its runs agree.
tests/golden/make_golden.py stores one run's per-row encodings, global tables,
bins and edges together with an order / folds under which the oracle
reproduces that run; here the oracle must reproduce it bit for bit, and (when
the reference is built in this checkout) so must fresh runs of the reference
with orders recovered from their own encodings."""
import numpy as np
import pytest

import oracle as O
from datagen import CAT_HYPER, categorical_case


def _u32(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _fixture():
    return np.load(f"{O.HERE}/../tests/golden/categorical_small.npz")


@pytest.mark.parametrize("method", ["ordered", "cv"])
def test_oracle_matches_reference_fixture(method):
    g = _fixture()
    X, y = categorical_case()
    order = g[f"{method}_order"]
    if method == "ordered":
        Xo, tab, prior = O.ordered_ts(X, y, [2], order)
    else:
        Xo, tab, prior = O.cv_ts(X, y, [2], order, 5)
    assert np.array_equal(_u32(Xo[:, 2]), _u32(g[f"{method}_enc"]))
    assert np.array_equal(tab[2][0], g[f"{method}_keys"])
    assert np.array_equal(_u32(tab[2][1]), _u32(g[f"{method}_vals"]))
    # numeric columns untouched; NaN rows got the prior
    assert np.array_equal(_u32(np.delete(Xo, 2, 1)), _u32(np.delete(X, 2, 1)))
    assert np.all(Xo[np.isnan(X[:, 2]), 2] == prior)
    b = O.quantize_ts(Xo, [2])
    assert np.array_equal(b.bins, g[f"{method}_bins"])
    assert np.array_equal(_u32(b.edges), _u32(g[f"{method}_edges"]))
    assert np.array_equal(b.n_edges, g[f"{method}_n_edges"])
    assert b.n_edges[2] > 16  # the quantile rule, not the per-category fallback


def test_reference_model_trained_on_target_statistics():
    """The REF32 oracle fit on the oracle's TS bins is the reference's model."""
    g = _fixture()
    X, y = categorical_case()
    Xo, _, _ = O.ordered_ts(X, y, [2], g["ordered_order"])
    b = O.quantize_ts(Xo, [2])
    hp = O.Hyper(**CAT_HYPER)
    fit = O.fit(b, y, hp, mode=0)
    ref = O.parse_tcat(g["tcat"].tobytes())
    assert fit.min_margin > 1e-6
    assert np.array_equal(fit.feature, ref.feature) and np.array_equal(fit.bin, ref.bin)
    assert np.array_equal(_u32(fit.threshold), _u32(ref.threshold))
    assert (ref.feature == 2).any()  # the encoded column is split on
    assert np.allclose(fit.leaves, ref.leaves, rtol=1e-6, atol=1e-7)


@pytest.mark.skipif(not O.ref_available(), reason="reference not built in this checkout")
@pytest.mark.parametrize("method", ["ordered", "cv"])
def test_oracle_matches_live_reference(method):
    """Fresh reference runs (each with its own random order) on a dataset with
    two categorical columns: per column, the oracle under the order / folds
    recovered from that run's encodings reproduces the run bit for bit."""
    X, y = categorical_case(n=2000, f=7, seed=8, n_cat=2, cardinality=40)
    for _ in range(2):
        enc, rb, tables, _ = O.ref_cat_ts(X, y, [2, 4], method)
        Xall = np.array(X)
        for c, j in enumerate((2, 4)):
            if method == "ordered":
                order = O.recover_order(X, y, j, enc[c])
                Xo, tab, _ = O.ordered_ts(X, y, [j], order)
            else:
                order = O.recover_folds(X, y, j, enc[c], 5)
                Xo, tab, _ = O.cv_ts(X, y, [j], order, 5)
            assert np.array_equal(_u32(Xo[:, j]), _u32(enc[c]))
            assert np.array_equal(tab[j][0], tables[j][0])
            assert np.array_equal(_u32(tab[j][1]), _u32(tables[j][1]))
            Xall[:, j] = Xo[:, j]
        b = O.quantize_ts(Xall, [2, 4])
        assert np.array_equal(b.bins, rb.bins)
        assert np.array_equal(_u32(b.edges), _u32(rb.edges)) and np.array_equal(b.n_edges, rb.n_edges)


def test_oracle_properties():
    X, y = categorical_case(n=800, f=5, seed=3, cardinality=12, nan_rate=0.05)
    rng = np.random.default_rng(0)
    o1 = rng.permutation(len(y))
    o2 = rng.permutation(len(y))
    A, ta, prior = O.ordered_ts(X, y, [2], o1)
    B, tb, _ = O.ordered_ts(X, y, [2], o2)
    # class-id labels sum exactly in float: the global table does not depend on the order
    assert np.array_equal(ta[2][0], tb[2][0]) and np.array_equal(_u32(ta[2][1]), _u32(tb[2][1]))
    # the first row of each category in the order is encoded with the prior
    seen = set()
    for r in o1:
        if np.isnan(X[r, 2]):
            assert A[r, 2] == prior
            continue
        c = O.category_of(X[r, 2])
        if c not in seen:
            assert A[r, 2] == prior
            seen.add(c)
    # cross-validated with one fold: every row sees no other fold -> (0 + a*prior) / (0 + a)
    C1, _, _ = O.cv_ts(X, y, [2], np.zeros(len(y), np.uint32), 1)
    assert np.all(C1[:, 2] == prior)
    # test rows: known categories -> table, unseen -> 0.5, NaN stays NaN
    T = np.array([[0, 0, 3.0, 0, 0], [0, 0, 999.0, 0, 0], [0, 0, np.nan, 0, 0]], np.float32)
    E = O.encode_test(T, ta)
    k = int(np.searchsorted(ta[2][0], 3))
    assert E[0, 2] == ta[2][1][k] and E[1, 2] == np.float32(0.5) and np.isnan(E[2, 2])
    # category ids as x86-64 truncates them
    assert O.category_of(np.float32(-1.0)) == 0xFFFFFFFF and O.category_of(np.float32(2.9)) == 2
