"""The regular-tree (mode="small", depth-wise) training oracle pinned to the
reference: `oracle.fit_regular` in its FP32 mode rebuilds, bit for bit, the
trees the reference trained (structure, node numbering, leaf values), from
the fixture tests/golden/make_golden.py stored and, where the reference is
built in this checkout, from fresh fits."""
import numpy as np
import pytest

import oracle as O
from datagen import REGULAR_TRAIN_HYPER, binary_c1, regular_train_case


def _same_tree(t, r):
    return (len(t["value"]) == len(r["value"]) and all(np.array_equal(t[k], r[k]) for k in ("is_leaf", "left", "right"))
            and np.array_equal(t["feature"][~t["is_leaf"]], r["feature"][~r["is_leaf"]])
            and np.array_equal(t["split_bin"][~t["is_leaf"]], r["split_bin"][~r["is_leaf"]])
            and np.array_equal(t["value"].view(np.uint32), r["value"].view(np.uint32)))


def test_regular_training_oracle_matches_reference_fixture():
    g = np.load(f"{O.HERE}/../tests/golden/regular_train_small.npz")
    m = O.parse_tcat_regular(g["tcat"].tobytes())
    X, y = regular_train_case()
    hp = O.Hyper(**REGULAR_TRAIN_HYPER)
    trees, pred, base = O.fit_regular(O.quantize(X), y, hp)
    assert np.float32(base) == np.float32(m.base) and len(trees) == len(m.trees) == hp.n_estimators
    for t, r in zip(trees, m.trees):
        assert _same_tree(t, r)
    # depth 7 would allow 128 leaves: the 64-leaf cap, applied in the
    # recursion's order (smaller child first), shapes every tree
    assert all(64 <= int(t["is_leaf"].sum()) <= 70 for t in trees)
    # the FP64 mode (the bar for a device build) takes the same top splits
    # (root and its children) from the same gradients; deeper down, the
    # reference's FP32 subtraction chains move node sums across the
    # min_child_weight bound, so whole trees agree only up to that
    b = O.quantize(X)
    p = np.full(len(y), base, np.float32)
    for t in trees:
        g, h = O.gradients("logloss", y, p)
        t64 = O.build_regular_tree(b, g, h, hp, fp32=False)
        for i in (0, 1, 2):
            if not t["is_leaf"][i] and t64["margin"][i] > 1e-5:
                assert (t64["feature"][i], t64["split_bin"][i]) == (t["feature"][i], t["split_bin"][i])
        leaf = t["value"][t["leaf_of"]].astype(np.longdouble)
        p = (p.astype(np.longdouble) + np.longdouble(np.float32(hp.learning_rate)) * leaf).astype(np.float32)


@pytest.mark.skipif(not O.ref_available(), reason="reference not built in this checkout")
@pytest.mark.parametrize("n,f,depth,msl,mcw,lam", [(3000, 10, 5, 1, 1.0, 1.0), (30_000, 6, 6, 20, 5.0, 3.0),
                                                     (5000, 12, 8, 1, 0.5, 0.0)])
def test_regular_training_oracle_matches_live_reference(n, f, depth, msl, mcw, lam):
    X, y = binary_c1(n, f, seed=n + depth)
    hp = O.Hyper(loss="logloss", n_estimators=8, max_depth=depth, learning_rate=0.2, min_samples_leaf=msl,
                 min_child_weight=mcw, lambda_l2=lam, regular_trees=True)
    b, model, _, _, _ = O.ref_fit(X, y, hp)
    m = O.parse_tcat_regular(model)
    trees, _, _ = O.fit_regular(b, y, hp)
    for t, r in zip(trees, m.trees):
        assert _same_tree(t, r)


@pytest.mark.parametrize("n,f,depth,msl,mcw,lam", [(3000, 10, 5, 1, 1.0, 1.0), (4000, 10, 7, 1, 1.0, 1.0),
                                                     (5000, 8, 6, 20, 5.0, 3.0)])
def test_level_wise_growth_with_replay_is_the_recursion(n, f, depth, msl, mcw, lam):
    """The device grows a tree level by level and replays the reference's
    recursion afterwards (the leaf cap, the numbering); in FP64 that gives
    the recursion's tree exactly, the 64-leaf cap included (depth 7)."""
    X, y = binary_c1(n, f, seed=n + depth)
    hp = O.Hyper(loss="logloss", max_depth=depth, min_samples_leaf=msl, min_child_weight=mcw, lambda_l2=lam)
    b = O.quantize(X)
    p = np.full(n, O.init_prediction("logloss", y), np.float32)
    for _ in range(3):
        g, h = O.gradients("logloss", y, p)
        t = O.build_regular_tree(b, g, h, hp, fp32=False)
        lw = O.build_regular_tree_levelwise(b, g, h, hp)
        for k in ("is_leaf", "left", "right"):
            assert np.array_equal(t[k], lw[k])
        assert np.array_equal(t["feature"][~t["is_leaf"]], lw["feature"][~lw["is_leaf"]])
        assert np.array_equal(t["split_bin"][~t["is_leaf"]], lw["split_bin"][~lw["is_leaf"]])
        assert np.array_equal(t["value"].view(np.uint32), lw["value"].astype(np.float32).view(np.uint32))
        leaf = t["value"][t["leaf_of"]].astype(np.longdouble)
        p = (p.astype(np.longdouble) + np.longdouble(np.float32(0.2)) * leaf).astype(np.float32)


def test_leafwise_oracle_matches_reference_fixture():
    """The regression preset grows leaf-wise trees in mode="small"
    (GrowPolicy::Lossguide): the oracle's FP32 mode rebuilds the reference's,
    bit for bit, from the stored fit."""
    from datagen import LEAFWISE_HYPER, leafwise_case

    g = np.load(f"{O.HERE}/../tests/golden/leafwise_small.npz")
    m = O.parse_tcat_regular(g["tcat"].tobytes())
    X, y = leafwise_case()
    trees, _, base = O.fit_leafwise(O.quantize(X), y, O.Hyper(**LEAFWISE_HYPER))
    assert np.float32(base) == np.float32(m.base)
    for t, r in zip(trees, m.trees):
        assert _same_tree(t, r)
    # the 64-leaf bound only stops new candidates: open ones still end as leaves
    assert max(int(t["is_leaf"].sum()) for t in trees) > 64


@pytest.mark.skipif(not O.ref_available(), reason="reference not built in this checkout")
@pytest.mark.parametrize("n,f,depth,msl,lam", [(3000, 10, 6, 1, 1.0), (6000, 8, 5, 20, 3.0)])
def test_leafwise_oracle_matches_live_reference(n, f, depth, msl, lam):
    from datagen import regression_c2

    X, y = regression_c2(n, f, seed=n + depth)
    hp = O.Hyper(loss="mse", n_estimators=6, max_depth=depth, learning_rate=0.1, min_samples_leaf=msl,
                 lambda_l2=lam, regular_trees=True)
    b, model, _, _, _ = O.ref_fit(X, y, hp)
    m = O.parse_tcat_regular(model)
    trees, _, _ = O.fit_leafwise(b, y, hp)
    for t, r in zip(trees, m.trees):
        assert _same_tree(t, r)


def test_multiclass_regular_oracle_matches_reference_fixture():
    """The reference's multiclass loop builds one regular tree per class and
    iteration on that class's softmax gradients (in every mode); the oracle
    rebuilds every tree bit for bit."""
    from datagen import MULTICLASS_REGULAR_HYPER, multiclass_regular_case

    g = np.load(f"{O.HERE}/../tests/golden/multiclass_regular_small.npz")
    m = O.parse_tcat_regular(g["tcat"].tobytes())
    assert m.task == 1 and m.n_classes == 4
    X, y = multiclass_regular_case()
    hp = O.Hyper(**MULTICLASS_REGULAR_HYPER)
    trees, _ = O.fit_regular_multiclass(O.quantize(X), y, hp, 4)
    assert len(trees) == len(m.trees) == hp.n_estimators * 4
    for t, r in zip(trees, m.trees):
        assert _same_tree(t, r)
