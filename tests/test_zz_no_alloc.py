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

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-5


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
