"""Several host threads on one context: training calls are serialised by the
context, predict calls share its staging buffer under a lock, and every
thread gets the result it would get alone."""
import threading

import numpy as np
import pytest

from datagen import binary_c1

pytestmark = pytest.mark.gpu


def test_threads_share_a_context(engine, capi):
    X, y = binary_c1(20_000, 20, seed=71)
    ds = engine.upload(X, y)
    ds.quantize(255)
    p = capi.params(loss="logloss", n_estimators=15, max_depth=6, learning_rate=0.1, hist_features_per_block=32)
    alone_tr = engine.trainer(ds, p)
    alone_tr.step(15)
    alone = alone_tr.model().export()
    ref_model = alone_tr.model()
    Xq = np.ascontiguousarray(X[:3000])
    ref_pred = ref_model.predict(Xq, "sigmoid")

    results, errors = {}, []

    def train(i):
        try:
            tr = engine.trainer(ds, p)
            tr.step(15)
            results[("train", i)] = tr.model().export()
        except Exception as e:  # surfaced below
            errors.append(e)

    def predict(i):
        try:
            for _ in range(20):
                out = ref_model.predict(Xq, "sigmoid")  # same request, so the same row tiles
                if not np.array_equal(out, ref_pred):
                    raise AssertionError("predict result changed under concurrency")
            results[("pred", i)] = True
        except Exception as e:
            errors.append(e)

    ts = [threading.Thread(target=train, args=(i,)) for i in range(3)]
    ts += [threading.Thread(target=predict, args=(i,)) for i in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for i in range(3):
        ex = results[("train", i)]
        assert np.array_equal(ex["feature"], alone["feature"]) and np.array_equal(ex["bin"], alone["bin"])
        assert np.allclose(ex["leaves"], alone["leaves"], rtol=1e-5, atol=1e-6)
        assert results[("pred", i)]


def test_threads_small_requests_two_models(engine, capi):
    """Small requests (at most 64 rows: the latency worker) from several
    threads at once, alternating between two models (the worker restarts for
    the other model under the context's lock) while another thread trains:
    every result equals the one predicted alone, bit for bit."""
    X, y = binary_c1(20_000, 16, seed=72)
    ds = engine.upload(X, y)
    ds.quantize(255)
    p1 = capi.params(loss="logloss", n_estimators=40, max_depth=6, learning_rate=0.1)
    p2 = capi.params(loss="logloss", n_estimators=12, max_depth=4, learning_rate=0.3)
    m1, _ = engine.train(ds, p1)
    m2, _ = engine.train(ds, p2)
    sizes = (1, 7, 64)
    want = {(k, n): m.predict(X[:n], "sigmoid") for k, m in ((1, m1), (2, m2)) for n in sizes}
    errors = []

    def serve(i):
        try:
            for r in range(30):
                k, m = ((1, m1), (2, m2))[(i + r) % 2]
                n = sizes[(i + r) % 3]
                if not np.array_equal(m.predict(X[:n], "sigmoid"), want[(k, n)]):
                    raise AssertionError(f"small request changed under concurrency ({k}, {n})")
        except Exception as e:  # surfaced below
            errors.append(e)

    def train():
        try:
            tr = engine.trainer(ds, p2)
            tr.step(12)
        except Exception as e:
            errors.append(e)

    ts = [threading.Thread(target=serve, args=(i,)) for i in range(4)] + [threading.Thread(target=train)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
