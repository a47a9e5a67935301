"""Serving loop through the C ABI: every request's result is the same when
served alone (tc_predict) and when coalesced with others (continuous
batching) -- bit for bit for requests of more than 64 rows, within the
stated tolerance for smaller ones (served alone they take the small-request
path) -- in both the coalescing and the plain per-request modes, with pinned
and pageable buffers, and under a tight staging-memory budget."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _random_model(engine, capi, seed, T, D, F, K=1):
    rng = np.random.default_rng(seed)
    arrays = dict(depth=rng.integers(max(0, D - 2), D + 1, T).astype(np.int32),
                  feature=rng.integers(0, F, (T, D)).astype(np.uint16),
                  threshold=rng.standard_normal((T, D)).astype(np.float32),
                  leaves=(0.1 * rng.standard_normal((T, 1 << D))).astype(np.float32),
                  weights=np.full(T, 0.1, np.float32))
    info = capi.ModelInfo(T, K, D, F, 1 if K > 1 else 0, 0.3, 0.1, 1.0)
    return engine.import_model(info, arrays), arrays


def _same_as_alone(o, X, m, arrays, transform="raw"):
    """A served result against the request predicted alone: bit for bit above
    64 rows; within the stated tolerance at most 64 rows, where tc_predict
    takes the small-request path (trees split over blocks: FP32 sums in
    another order)."""
    alone = m.predict(X, transform)
    if X.shape[0] > 64:
        return np.array_equal(o, alone)
    scale = 0.3 + (np.abs(arrays["leaves"]).max(1) * arrays["weights"]).sum()
    return np.max(np.abs(o - alone)) <= 1e-5 * (scale if transform == "raw" else 1.0)


def _requests(F, sizes, seed, pinned):
    import torch

    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        X = rng.standard_normal((n, F)).astype(np.float32)
        if pinned:
            t = torch.empty((n, F), dtype=torch.float32, pin_memory=True)
            t.numpy()[:] = X
            X = t.numpy()
        out.append(X)
    return out


@pytest.mark.parametrize("coalesce,pinned", [(True, True), (True, False), (False, True)])
def test_results_same_alone_and_in_the_mix(engine, capi, coalesce, pinned):
    import torch

    F = 24
    m1, a1 = _random_model(engine, capi, 1, 300, 6, F)
    m2, a2 = _random_model(engine, capi, 2, 40, 10, F)
    m3, a3 = _random_model(engine, capi, 3, 50, 5, F, K=4)
    sizes = [1, 7, 128, 129, 1000, 4096, 33, 5000, 2, 700, 16384, 64, 3, 900]
    reqs = _requests(F, sizes, 11, pinned)
    models = [m1, m2, m3]
    transforms = ["sigmoid", "raw", "softmax"]
    alone = []
    for i, X in enumerate(reqs):
        m = models[i % 3]
        alone.append(m.predict(X, transforms[i % 3]))
    srv = capi.Server(engine, staging_bytes=0, max_batch_rows=65536, coalesce=coalesce, max_inflight=4)
    ids = [srv.add_model(m) for m in models]
    outs = []
    tickets = []
    for i, X in enumerate(reqs):
        K = models[i % 3].info.n_classes
        if pinned:
            o = torch.empty((X.shape[0], K), dtype=torch.float32, pin_memory=True).numpy()
        else:
            o = np.zeros((X.shape[0], K), np.float32)
        outs.append(o)
        tickets.append(srv.submit(ids[i % 3], X, o, transforms[i % 3]))
    for t in tickets:
        done, lat = srv.poll(t, 10_000_000)
        assert done and lat is not None and lat >= 0
    for i in range(len(reqs)):
        if reqs[i].shape[0] > 64:
            assert np.array_equal(outs[i], alone[i]), i
        else:
            # alone, a request of at most 64 rows takes the small-request
            # path (trees split over blocks): FP32 sums in another order,
            # equal within the stated tolerance
            a = (a1, a2, a3)[i % 3]
            scale = 0.3 + (np.abs(a["leaves"]).max(1) * a["weights"]).sum()
            tol = 1e-5 * (scale if transforms[i % 3] == "raw" else 1.0)
            assert np.max(np.abs(outs[i] - alone[i])) <= tol, i
    done_n, launches, rows = srv.stats()
    assert done_n == len(reqs) and rows == sum(sizes)
    if not coalesce:
        assert launches == len(reqs)
    srv.close()
    # every request's result (served in the mix, equal to alone above) against
    # the FP64 oracle's prediction of its model with the request's transform
    ens = []
    for (T, D, K), a in zip(((300, 6, 1), (40, 10, 1), (50, 5, 4)), (a1, a2, a3)):
        ens.append(O.Ensemble(0.3, K, D, a["depth"], a["feature"], np.zeros((T, D), np.uint8), a["threshold"],
                              a["leaves"], a["weights"]))
    for i, X in enumerate(reqs):
        raw = O.predict(ens[i % 3], X)
        if transforms[i % 3] == "sigmoid":
            want = 1.0 / (1.0 + np.exp(-raw))
        elif transforms[i % 3] == "softmax":
            z = np.exp(raw - raw.max(1, keepdims=True))
            want = z / z.sum(1, keepdims=True)
        else:
            want = raw
        a = (a1, a2, a3)[i % 3]
        scale = 0.3 + (np.abs(a["leaves"]).max(1) * a["weights"]).sum()  # |base| + sum |w * leaf|
        tol = 1e-5 * (scale if transforms[i % 3] == "raw" else 1.0)
        assert np.max(np.abs(outs[i] - want)) <= tol, (i, transforms[i % 3])


def test_coalescing_happens_under_a_burst(engine, capi):
    import torch

    F = 16
    m, arr = _random_model(engine, capi, 5, 200, 6, F)
    reqs = _requests(F, [256] * 64, 3, True)
    srv = capi.Server(engine, staging_bytes=0, max_batch_rows=65536, coalesce=True, max_inflight=2)
    mid = srv.add_model(m)
    outs = [torch.empty((256, 1), dtype=torch.float32, pin_memory=True).numpy() for _ in reqs]
    tickets = [srv.submit(mid, X, o, "raw") for X, o in zip(reqs, outs)]
    for t in tickets:
        assert srv.poll(t, 10_000_000)[0]
    _, launches, _ = srv.stats()
    assert launches < len(reqs)  # requests that arrived while a batch ran shared a launch
    for X, o in zip(reqs, outs):
        assert _same_as_alone(o, X, m, arr)
    srv.close()


def test_admission_by_staging_memory(engine, capi):
    F = 32
    m, arr = _random_model(engine, capi, 7, 100, 6, F)
    # room for ~3000 rows per slot: requests queue until a slot frees
    budget = 2 * 3000 * (F + 16) * 4
    srv = capi.Server(engine, staging_bytes=budget, max_batch_rows=65536, coalesce=True, max_inflight=2)
    mid = srv.add_model(m)
    reqs = _requests(F, [1000, 2500, 3000, 10, 2999, 1500, 700, 3000], 9, False)
    outs = [np.zeros((X.shape[0], 1), np.float32) for X in reqs]
    tickets = [srv.submit(mid, X, o, "raw") for X, o in zip(reqs, outs)]
    for t in tickets:
        assert srv.poll(t, 10_000_000)[0]
    for X, o in zip(reqs, outs):
        assert _same_as_alone(o, X, m, arr)
    # a request larger than a slot is refused up front
    big = np.zeros((3001, F), np.float32)
    with pytest.raises(capi.TCError) as ei:
        srv.submit(mid, big, np.zeros((3001, 1), np.float32), "raw")
    assert ei.value.status == 1
    with pytest.raises(capi.TCError):
        srv.submit(mid, np.zeros((5, F + 1), np.float32), np.zeros((5, 1), np.float32), "raw")
    srv.close()


def test_replay_open_loop(engine, capi):
    import torch

    F = 20
    m, arr = _random_model(engine, capi, 8, 120, 6, F)
    srv = capi.Server(engine, staging_bytes=0, max_batch_rows=65536, coalesce=True, max_inflight=4)
    mid = srv.add_model(m)
    rng = np.random.default_rng(4)
    sizes = np.floor(np.exp(rng.uniform(0, np.log(4097), 200))).astype(int)
    reqs = _requests(F, sizes, 12, True)
    outs = [torch.empty((X.shape[0], 1), dtype=torch.float32, pin_memory=True).numpy() for X in reqs]
    arrivals = np.cumsum(rng.exponential(1 / 5000.0, len(reqs)))
    lat, wall = srv.replay([(float(t), mid, X, o, "raw") for t, X, o in zip(arrivals, reqs, outs)])
    assert np.all(lat > 0) and wall >= arrivals[-1]
    for X, o in zip(reqs, outs):
        assert _same_as_alone(o, X, m, arr)
    srv.close()


@pytest.mark.parametrize("K,T,D", [(1, 1000, 6), (4, 120, 5), (1, 20, 8)])
def test_small_requests_match_oracle(engine, capi, K, T, D):
    """Requests of 1..64 rows through tc_predict take the small-request path
    (trees split over blocks, inputs and outputs through pinned mapped
    staging): every size against the FP64 oracle, NaN features included, and
    two calls in a row give the same bits."""
    F = 37
    m, a = _random_model(engine, capi, 20 + K + T, T, D, F, K=K)
    ens = O.Ensemble(0.3, K, D, a["depth"], a["feature"], np.zeros((T, D), np.uint8), a["threshold"],
                     a["leaves"], a["weights"])
    rng = np.random.default_rng(T + D)
    scale = 0.3 + (np.abs(a["leaves"]).max(1) * a["weights"]).sum()
    for n in list(range(1, 17)) + [31, 32, 33, 63, 64]:
        X = rng.standard_normal((n, F)).astype(np.float32)
        X[rng.random((n, F)) < 0.05] = np.nan
        raw = O.predict(ens, X)
        tr = "softmax" if K > 1 else "sigmoid"
        got = m.predict(X, tr)
        again = m.predict(X, tr)
        assert np.array_equal(got, again), n
        if K > 1:
            z = np.exp(raw - raw.max(1, keepdims=True))
            want = z / z.sum(1, keepdims=True)
        else:
            want = 1.0 / (1.0 + np.exp(-raw))
        assert np.max(np.abs(got - want)) <= 1e-5, n
        assert np.max(np.abs(m.predict(X, "raw") - raw)) <= 1e-5 * scale, n


def test_latency_worker_lifecycle(engine, capi):
    """Small requests go through the persistent latency worker: results stay
    equal (bits) across the worker ending on its own after an idle gap and
    being relaunched, across switches between two models (the worker is
    restarted for the other model), and after the model it serves is
    destroyed (it is stopped first)."""
    import time

    F = 21
    m1, a1 = _random_model(engine, capi, 501, 300, 6, F)
    m2, a2 = _random_model(engine, capi, 502, 50, 4, F)
    rng = np.random.default_rng(503)
    X = rng.standard_normal((64, F)).astype(np.float32)
    X[rng.random(X.shape) < 0.05] = np.nan
    want1 = {n: m1.predict(X[:n], "sigmoid") for n in (1, 7, 64)}
    want2 = {n: m2.predict(X[:n], "raw") for n in (1, 7, 64)}
    for n in (1, 7, 64):
        e1 = O.Ensemble(0.3, 1, 6, a1["depth"], a1["feature"], np.zeros((300, 6), np.uint8), a1["threshold"],
                        a1["leaves"], a1["weights"])
        p = 1.0 / (1.0 + np.exp(-O.predict(e1, X[:n])))
        assert np.max(np.abs(want1[n] - p)) <= 1e-5
    for rnd in range(3):
        for n in (1, 7, 64):
            assert np.array_equal(m1.predict(X[:n], "sigmoid"), want1[n]), (rnd, n)
            assert np.array_equal(m2.predict(X[:n], "raw"), want2[n]), (rnd, n)
        time.sleep(0.05)  # longer than the worker's idle limit: it ends and is relaunched
        assert np.array_equal(m1.predict(X[:1], "sigmoid"), want1[1])
    # one launch per request instead of the worker: the same values within
    # the stated tolerance (the trees are split over blocks differently)
    engine.set_latency_worker(False)
    scale = 0.3 + (np.abs(a1["leaves"]).max(1) * a1["weights"]).sum()
    for n in (1, 7, 64):
        assert np.max(np.abs(m1.predict(X[:n], "raw") - engine_raw(m1, X[:n], a1))) <= 1e-5 * scale
        assert np.max(np.abs(m1.predict(X[:n], "sigmoid") - want1[n])) <= 1e-5
    engine.set_latency_worker(True)
    m1.close()  # stops the worker serving m1
    assert np.array_equal(m2.predict(X[:7], "raw"), want2[7])


def engine_raw(m, X, a):
    """FP64 oracle raw scores of a model built by _random_model (depth 6)."""
    T = a["depth"].shape[0]
    e = O.Ensemble(0.3, 1, 6, a["depth"], a["feature"], np.zeros((T, 6), np.uint8), a["threshold"], a["leaves"],
                   a["weights"])
    return O.predict(e, X)
