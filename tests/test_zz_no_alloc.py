"""The allocation-free root histogram (tc_histogram_root_noalloc) against the
allocating path (tc_build_tree's root histogram), through the C ABI.

Callers that cannot call cudaMalloc -- a process whose device memory is
owned by another framework's allocator, or a latency-critical request path
that must not allocate -- pass their own device buffers; the entry point's
scratch is a fixed array inside the library.  Two calls in a row must both
agree with the allocating path within the histogram tolerance the other
tests use: 1e-5 of the sum of |grad| (or hess) over the bin's rows.
This file is collected last on purpose."""
import ctypes as C
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-5


def _fp64_hist(bins_rm, f, g, h):
    """FP64 histogram [f][256][2] of row-major bins and the per-bin sums of
    |g| and h (the tolerance scale)."""
    n = bins_rm.shape[0]
    idx = (np.arange(f, dtype=np.int64)[None, :] * 256 + bins_rm[:, :f].astype(np.int64)).ravel()
    gg = np.repeat(g.astype(np.float64), f)
    hh = np.repeat(h.astype(np.float64), f)
    out = np.zeros((f, 256, 2))
    out[..., 0] = np.bincount(idx, gg, f * 256).reshape(f, 256)
    out[..., 1] = np.bincount(idx, hh, f * 256).reshape(f, 256)
    sg = np.bincount(idx, np.abs(gg), f * 256).reshape(f, 256)
    sh = np.bincount(idx, np.abs(hh), f * 256).reshape(f, 256)
    assert n * f == idx.size
    return out, sg, sh


def _noalloc(lib, engine, d_bins, n, f, stride, d_g, d_h, out, stream=None):
    return lib.tc_histogram_root_noalloc(engine.ctx, C.c_void_p(d_bins.data_ptr()), C.c_uint32(n), C.c_uint16(f),
                                         C.c_uint32(stride), C.c_void_p(d_g.data_ptr()), C.c_void_p(d_h.data_ptr()),
                                         C.c_void_p(out.data_ptr()), stream)


def test_noalloc_root_histogram_matches_allocating_path(engine, capi):
    import torch

    rng = np.random.default_rng(2024)
    n, f = 40_000, 77
    X = rng.standard_normal((n, f)).astype(np.float32)
    X[rng.random((n, f)) < 0.02] = np.nan   # exercise the NaN slot
    g = rng.standard_normal(n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    ds = engine.upload(X, np.zeros(n, np.float32))
    ds.quantize(255)
    ref = engine.build_tree(ds, g, h, capi.params(loss="mse", max_depth=1), want_hist=True)["root_hist"]

    bins_cm = ds.bins()                                   # [f][n]
    stride = (f + 15) // 16 * 16
    bins_rm = np.zeros((n, stride), np.uint8)
    bins_rm[:, :f] = bins_cm.T
    dev = torch.device("cuda", 0)
    d_bins = torch.from_numpy(bins_rm).to(dev)
    d_g = torch.from_numpy(g).to(dev)
    d_h = torch.from_numpy(h).to(dev)
    scale_g = np.zeros((f, 256))
    scale_h = np.zeros((f, 256))
    for j in range(f):
        np.add.at(scale_g[j], bins_cm[j], np.abs(g.astype(np.float64)))
        np.add.at(scale_h[j], bins_cm[j], h.astype(np.float64))
    lib = capi.lib()
    for call in range(2):
        out = torch.full((f, 256, 2), -1.0, dtype=torch.float64, device=dev)
        st = lib.tc_histogram_root_noalloc(engine.ctx, C.c_void_p(d_bins.data_ptr()), C.c_uint32(n), C.c_uint16(f),
                                           C.c_uint32(stride), C.c_void_p(d_g.data_ptr()),
                                           C.c_void_p(d_h.data_ptr()), C.c_void_p(out.data_ptr()), None)
        assert st == 0, lib.tc_last_error(engine.ctx)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got[..., 0] - ref[..., 0]) <= REL * scale_g + 1e-9), call
        assert np.all(np.abs(got[..., 1] - ref[..., 1]) <= REL * scale_h + 1e-9), call


def test_noalloc_rejects_oversized_feature_count(engine, capi):
    lib = capi.lib()
    dummy = C.c_void_p(1)
    st = lib.tc_histogram_root_noalloc(engine.ctx, dummy, C.c_uint32(10), C.c_uint16(8193), C.c_uint32(8208),
                                       dummy, dummy, dummy, None)
    assert st == 1
    assert b"8192" in lib.tc_last_error(engine.ctx)


@pytest.mark.parametrize("n,f", [(3_000, 8_000), (2_500_000, 6)])
def test_noalloc_wide_and_long_inputs(engine, capi, n, f):
    """Near the feature limit (one row chunk per pass) and with many rows
    (several passes of capped row chunks, merged in FP64): both within the
    tolerance of an FP64 histogram, on two calls in a row."""
    import torch

    rng = np.random.default_rng(n + f)
    stride = (f + 15) // 16 * 16
    bins_rm = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    g = rng.standard_normal(n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    ref, sg, sh = _fp64_hist(bins_rm, f, g, h)
    dev = torch.device("cuda", 0)
    d_bins = torch.from_numpy(bins_rm).to(dev)
    d_g = torch.from_numpy(g).to(dev)
    d_h = torch.from_numpy(h).to(dev)
    lib = capi.lib()
    for call in range(2):
        out = torch.full((f, 256, 2), -1.0, dtype=torch.float64, device=dev)
        st = _noalloc(lib, engine, d_bins, n, f, stride, d_g, d_h, out)
        assert st == 0, lib.tc_last_error(engine.ctx)
        engine.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got[..., 0] - ref[..., 0]) <= REL * sg + 1e-9), call
        assert np.all(np.abs(got[..., 1] - ref[..., 1]) <= REL * sh + 1e-9), call


def test_noalloc_on_the_context_stream_while_training(engine, capi):
    """With no stream given, calls made while another thread trains on the
    same context wait for the training call instead of joining its graph
    capture: the trainer's result equals a fit made alone, every call's
    histogram is right, and no later graph replay writes into a call's
    output buffer."""
    import torch

    from datagen import binary_c1

    X, y = binary_c1(30_000, 16, seed=5)
    ds = engine.upload(X, y)
    ds.quantize(255)
    p = capi.params(loss="logloss", n_estimators=24, max_depth=6, learning_rate=0.1)
    alone = engine.trainer(ds, p)
    alone.step(24)
    ref_model = alone.model().export()

    rng = np.random.default_rng(11)
    n, f = 50_000, 40
    stride = 48
    bins_rm = rng.integers(0, 256, (n, stride), dtype=np.uint8)
    g = rng.standard_normal(n).astype(np.float32)
    h = rng.uniform(0.05, 1.0, n).astype(np.float32)
    ref, sg, sh = _fp64_hist(bins_rm, f, g, h)
    dev = torch.device("cuda", 0)
    d_bins = torch.from_numpy(bins_rm).to(dev)
    d_g = torch.from_numpy(g).to(dev)
    d_h = torch.from_numpy(h).to(dev)
    out = torch.empty((f, 256, 2), dtype=torch.float64, device=dev)
    lib = capi.lib()
    errors, trained = [], {}

    def train():
        try:
            tr = engine.trainer(ds, p)
            for _ in range(6):
                tr.step(4)
            trained["m"] = tr.model().export()
        except Exception as e:  # surfaced below
            errors.append(e)

    t = threading.Thread(target=train)
    t.start()
    for call in range(12):
        st = _noalloc(lib, engine, d_bins, n, f, stride, d_g, d_h, out)
        assert st == 0, lib.tc_last_error(engine.ctx)
        engine.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.abs(got[..., 0] - ref[..., 0]) <= REL * sg + 1e-9), call
        assert np.all(np.abs(got[..., 1] - ref[..., 1]) <= REL * sh + 1e-9), call
        out.fill_(-1.0)
        # torch's stream only: a device-wide synchronise would reach into the
        # other thread's graph capture
        torch.cuda.current_stream().synchronize()
    t.join()
    assert not errors, errors
    engine.synchronize()
    assert bool((out == -1.0).all()), "a training graph replay wrote into the no-alloc output"
    m = trained["m"]
    assert np.array_equal(m["feature"], ref_model["feature"]) and np.array_equal(m["bin"], ref_model["bin"])
    assert np.allclose(m["leaves"], ref_model["leaves"], rtol=1e-5, atol=1e-6)
