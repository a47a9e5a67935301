"""ctypes view of the C ABI in include/tcgpu.h (libtcgpu.so next to this file).

This is the binding a Python host would add for the device engine; the
pybind11 module `_turbocat` is the reference-shaped surface, this module is
the thin layer the tests, the benchmark and smoke checks use to call the
C ABI directly.  Loading fails loudly when the library is missing: there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtcgpu.so")

TC_OK = 0
STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "TIMEOUT", 4: "CUDA_ERROR", 5: "NOT_FITTED",
          6: "FORMAT", 7: "BUSY"}
LOSS = {"logloss": 0, "mse": 1, "focal": 2, "softmax": 3}
TRANSFORM = {"raw": 0, "sigmoid": 1, "softmax": 2}

# every symbol include/tcgpu.h declares
SYMBOLS = [
    "tc_ctx_create", "tc_ctx_destroy", "tc_last_error", "tc_ctx_memory", "tc_ctx_fail_next_allocs",
    "tc_ctx_synchronize", "tc_ctx_set_latency_worker", "tc_dataset_upload", "tc_dataset_destroy", "tc_quantize",
    "tc_apply_bins", "tc_dataset_bins", "tc_dataset_features", "tc_encode_categorical", "tc_category_table",
    "tc_trainer_create", "tc_trainer_step", "tc_trainer_reset", "tc_trainer_stats", "tc_trainer_profile",
    "tc_trainer_train_scores", "tc_trainer_sample_mask", "tc_trainer_set_validation", "tc_trainer_valid_loss",
    "tc_trainer_model", "tc_trainer_destroy", "tc_train", "tc_train_regular", "tc_build_tree", "tc_histogram_root_noalloc",
    "tc_model_info_get", "tc_model_export",
    "tc_model_import", "tc_model_save_tcat", "tc_model_load_tcat", "tc_model_destroy", "tc_predict",
    "tc_predict_device", "tc_predict_dataset", "tc_server_create", "tc_server_add_model", "tc_server_submit", "tc_server_poll",
    "tc_server_replay", "tc_server_stats", "tc_server_destroy",
]


class TrainParams(C.Structure):
    _fields_ = [
        ("loss", C.c_int32), ("n_classes", C.c_int32), ("n_estimators", C.c_int32), ("max_depth", C.c_int32),
        ("max_bins", C.c_int32), ("min_samples_leaf", C.c_int32), ("learning_rate", C.c_float),
        ("lambda_l2", C.c_float), ("lambda_l1", C.c_float), ("min_child_weight", C.c_float),
        ("min_split_gain", C.c_float), ("max_delta_step", C.c_float), ("focal_gamma", C.c_float),
        ("focal_alpha", C.c_float), ("batched", C.c_int32), ("hist_features_per_block", C.c_int32),
        ("hist_rows_per_chunk", C.c_int32), ("subsample", C.c_float), ("colsample_bytree", C.c_float),
        ("seed", C.c_uint64), ("use_goss", C.c_int32), ("goss_top_rate", C.c_float),
        ("goss_other_rate", C.c_float),
    ]


class CatParams(C.Structure):
    _fields_ = [("method", C.c_int32), ("prior_weight", C.c_float), ("cv_folds", C.c_int32), ("seed", C.c_uint64)]


CAT_METHOD = {"ordered": 0, "cv": 1}


class TrainStats(C.Structure):
    _fields_ = [("n_trees", C.c_int32), ("iterations_done", C.c_int32), ("base_prediction", C.c_float),
                ("seconds", C.c_double), ("hist_features_per_block", C.c_int32),
                ("hist_rows_per_chunk", C.c_int32), ("kernel_launches", C.c_int64),
                ("best_iteration", C.c_int32), ("stopped_early", C.c_int32)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 16), ("launches", C.c_int64), ("ms", C.c_double), ("alg_bytes", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("n_kernels", C.c_int32), ("k", KernelTime * 12), ("hist_level_ms", C.c_double * 16),
                ("hist_level_rows", C.c_double * 16), ("part_level_ms", C.c_double * 16),
                ("in_graph", C.c_int32), ("iteration_ms", C.c_double)]


class ModelInfo(C.Structure):
    _fields_ = [("n_trees", C.c_int32), ("n_classes", C.c_int32), ("max_depth", C.c_int32),
                ("n_features", C.c_int32), ("task", C.c_int32), ("base_prediction", C.c_float),
                ("learning_rate", C.c_float), ("lambda_l2", C.c_float)]


class ServerParams(C.Structure):
    _fields_ = [("staging_bytes", C.c_size_t), ("max_batch_rows", C.c_int32), ("coalesce", C.c_int32),
                ("max_inflight", C.c_int32)]


class ReplayRequest(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("model_id", C.c_int32), ("transform", C.c_int32),
                ("X", C.c_void_p), ("out", C.c_void_p), ("n", C.c_uint32), ("f", C.c_uint16),
                ("pad", C.c_uint16)]


class TCError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run turbo-cat_b200/build.py "
                               "(the device engine has no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _lib.tc_last_error.restype = C.c_char_p
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def params(loss="logloss", n_classes=1, n_estimators=10, max_depth=6, max_bins=255, min_samples_leaf=1,
           learning_rate=0.1, lambda_l2=1.0, lambda_l1=0.0, min_child_weight=1.0, min_split_gain=0.0,
           max_delta_step=0.0, focal_gamma=2.0, focal_alpha=0.25, batched=1, hist_features_per_block=0,
           hist_rows_per_chunk=0, subsample=1.0, colsample_bytree=1.0, seed=42, use_goss=False,
           goss_top_rate=0.2, goss_other_rate=0.1) -> TrainParams:
    return TrainParams(LOSS[loss] if isinstance(loss, str) else loss, n_classes, n_estimators, max_depth, max_bins,
                       min_samples_leaf, learning_rate, lambda_l2, lambda_l1, min_child_weight, min_split_gain,
                       max_delta_step, focal_gamma, focal_alpha, batched, hist_features_per_block,
                       hist_rows_per_chunk, subsample, colsample_bytree, seed, 1 if use_goss else 0,
                       goss_top_rate, goss_other_rate)


class Model:
    def __init__(self, eng, handle):
        self.eng, self.h = eng, handle
        info = ModelInfo()
        eng._chk(lib().tc_model_info_get(handle, C.byref(info)))
        self.info = info

    def export(self):
        i = self.info
        T, D, F = i.n_trees, i.max_depth, i.n_features
        out = dict(depth=np.zeros(T, np.int32), feature=np.zeros((T, D), np.uint16),
                   bin=np.zeros((T, D), np.uint8), threshold=np.zeros((T, D), np.float32),
                   gain=np.zeros((T, D), np.float32), leaves=np.zeros((T, 1 << D), np.float32),
                   weights=np.zeros(T, np.float32), edges=np.zeros((F, 255), np.float32),
                   n_edges=np.zeros(F, np.uint16))
        self.eng._chk(lib().tc_model_export(self.h, *[_p(out[k]) for k in (
            "depth", "feature", "bin", "threshold", "gain", "leaves", "weights", "edges", "n_edges")]))
        return out

    def tcat(self) -> bytes:
        n = C.c_size_t(0)
        self.eng._chk(lib().tc_model_save_tcat(self.h, None, C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        self.eng._chk(lib().tc_model_save_tcat(self.h, buf, C.byref(n)))
        return bytes(buf)

    def predict(self, X, transform="raw"):
        X = np.ascontiguousarray(X, np.float32)
        n, f = X.shape
        out = np.zeros((n, self.info.n_classes), np.float32)
        self.eng._chk(lib().tc_predict(self.eng.ctx, self.h, _p(X), C.c_uint32(n), C.c_uint16(f),
                                       C.c_int32(TRANSFORM[transform]), _p(out)))
        return out

    def predict_device(self, x_ptr, n, f, out_ptr, transform="raw", stream=0):
        """tc_predict_device: inputs and outputs already in device memory
        (raw pointers), launched on `stream` (0: the engine's stream); no
        synchronisation."""
        self.eng._chk(lib().tc_predict_device(self.eng.ctx, self.h, C.c_void_p(x_ptr), C.c_uint32(n),
                                              C.c_uint16(f), C.c_int32(TRANSFORM[transform]),
                                              C.c_void_p(out_ptr), C.c_void_p(stream)))

    def predict_dataset(self, ds: "Dataset", transform="raw"):
        """tc_predict_dataset: the dataset's rows as the device holds them."""
        out = np.zeros((ds.n, self.info.n_classes), np.float32)
        self.eng._chk(lib().tc_predict_dataset(self.eng.ctx, self.h, ds.h, C.c_int32(TRANSFORM[transform]),
                                               _p(out)))
        return out

    def close(self):
        if self.h and lib is not None:  # at interpreter exit the module globals may be gone
            lib().tc_model_destroy(self.h)
            self.h = None

    __del__ = close


class Dataset:
    def __init__(self, eng, handle, n, f):
        self.eng, self.h, self.n, self.f = eng, handle, n, f

    def quantize(self, max_bins=255, compat_u8=True):
        edges = np.zeros((self.f, 255), np.float32)
        ne = np.zeros(self.f, np.uint16)
        self.eng._chk(lib().tc_quantize(self.h, C.c_uint16(max_bins), C.c_int(1 if compat_u8 else 0), _p(edges),
                                        _p(ne)))
        return edges, ne

    def apply_bins(self, ref: "Dataset"):
        """Bins this dataset with ref's edges (Dataset::apply_bins)."""
        self.eng._chk(lib().tc_apply_bins(self.h, ref.h))

    def bins(self):
        out = np.zeros((self.f, self.n), np.uint8)
        self.eng._chk(lib().tc_dataset_bins(self.h, _p(out)))
        return out

    def features(self):
        """The feature matrix as the device holds it (encoded categorical columns)."""
        out = np.zeros((self.n, self.f), np.float32)
        self.eng._chk(lib().tc_dataset_features(self.h, _p(out)))
        return out

    def encode_categorical(self, features, method="ordered", prior_weight=1.0, cv_folds=5, seed=0, order=None):
        """Target statistics of the categorical columns (tc_encode_categorical);
        `order`: the processing order (ordered) or each row's fold (cv)."""
        feats = np.ascontiguousarray(features, np.uint16)
        prm = CatParams(CAT_METHOD[method], prior_weight, cv_folds, seed)
        o = None if order is None else np.ascontiguousarray(order, np.uint32)
        self.eng._chk(lib().tc_encode_categorical(self.h, _p(feats), C.c_uint16(len(feats)), C.byref(prm), _p(o)))

    def category_table(self, feature):
        """(sorted categories, encodings) of one encoded column."""
        n = C.c_uint32(0)
        self.eng._chk(lib().tc_category_table(self.h, C.c_uint16(feature), None, None, C.byref(n)))
        keys = np.zeros(n.value, np.uint32)
        vals = np.zeros(n.value, np.float32)
        self.eng._chk(lib().tc_category_table(self.h, C.c_uint16(feature), _p(keys), _p(vals), C.byref(n)))
        return keys, vals

    def close(self):
        if self.h and lib is not None:  # at interpreter exit the module globals may be gone
            lib().tc_dataset_destroy(self.h)
            self.h = None

    __del__ = close


class Trainer:
    def __init__(self, eng, handle, K, ds=None):
        self.eng, self.h, self.K = eng, handle, K
        self.ds = ds  # the device dataset must outlive the trainer

    def step(self, iters, sync=True):
        self.eng._chk(lib().tc_trainer_step(self.h, C.c_int32(iters), C.c_int(1 if sync else 0)))

    def reset(self):
        self.eng._chk(lib().tc_trainer_reset(self.h))

    def stats(self) -> TrainStats:
        st = TrainStats()
        self.eng._chk(lib().tc_trainer_stats(self.h, C.byref(st)))
        return st

    def profile(self, iters):
        """Runs `iters` profiled iterations (inside a replayed CUDA graph on the
        batched path); returns {kernel: (launches, ms, alg_bytes)} plus
        "_hist_levels", "_part_levels", "_in_graph" and "_iteration_ms"."""
        pr = Profile()
        self.eng._chk(lib().tc_trainer_profile(self.h, C.c_int32(iters), C.byref(pr)))
        out = {pr.k[i].name.decode(): (pr.k[i].launches, pr.k[i].ms, pr.k[i].alg_bytes)
               for i in range(pr.n_kernels)}
        out["_hist_levels"] = [(pr.hist_level_ms[d], pr.hist_level_rows[d]) for d in range(16)]
        out["_part_levels"] = [pr.part_level_ms[d] for d in range(16)]
        out["_in_graph"] = bool(pr.in_graph)
        out["_iteration_ms"] = pr.iteration_ms
        return out

    def set_validation(self, vds, early_stopping_rounds=50):
        """Validation set (a Dataset with labels, not necessarily quantized) and
        early stopping; call before the first step."""
        self.vds = vds  # must outlive the trainer
        self.eng._chk(lib().tc_trainer_set_validation(self.h, vds.h, C.c_int32(early_stopping_rounds)))

    def valid_loss(self):
        out = np.zeros(max(1, self.stats().iterations_done), np.float64)
        self.eng._chk(lib().tc_trainer_valid_loss(self.h, _p(out)))
        return out[: self.stats().iterations_done]

    def scores(self, n):
        out = np.zeros((n, self.K), np.float32)
        self.eng._chk(lib().tc_trainer_train_scores(self.h, _p(out)))
        return out

    def sample_mask(self, n):
        """Rows (bool [n]) the last iteration's trees were built on."""
        words = np.zeros((n + 31) // 32, np.uint32)
        self.eng._chk(lib().tc_trainer_sample_mask(self.h, _p(words)))
        return np.unpackbits(words.view(np.uint8), bitorder="little")[:n].astype(bool)

    def model(self) -> Model:
        m = C.c_void_p()
        self.eng._chk(lib().tc_trainer_model(self.h, C.byref(m)))
        return Model(self.eng, m)

    def close(self):
        if self.h and lib is not None:  # at interpreter exit the module globals may be gone
            lib().tc_trainer_destroy(self.h)
            self.h = None

    __del__ = close


class Engine:
    """One tc_ctx on a CUDA device."""

    def __init__(self, device=0, mem_budget=0):
        self.ctx = C.c_void_p()
        st = lib().tc_ctx_create(C.c_int(device), C.c_size_t(mem_budget), C.byref(self.ctx))
        if st != TC_OK:
            raise TCError(st, f"tc_ctx_create(device={device}) failed (no usable sm_100 device?)")

    def _chk(self, st):
        if st != TC_OK:
            raise TCError(st, lib().tc_last_error(self.ctx).decode())

    def upload(self, X, y=None) -> Dataset:
        X = np.ascontiguousarray(X, np.float32)
        n, f = X.shape
        y = np.ascontiguousarray(y, np.float32) if y is not None else None
        h = C.c_void_p()
        self._chk(lib().tc_dataset_upload(self.ctx, _p(X), C.c_uint32(n), C.c_uint16(f), _p(y), C.byref(h)))
        return Dataset(self, h, n, f)

    def trainer(self, ds: Dataset, p: TrainParams) -> Trainer:
        h = C.c_void_p()
        self._chk(lib().tc_trainer_create(self.ctx, ds.h, C.byref(p), C.byref(h)))
        return Trainer(self, h, p.n_classes if p.loss == LOSS["softmax"] else 1, ds)

    def train(self, ds: Dataset, p: TrainParams):
        h = C.c_void_p()
        st = TrainStats()
        self._chk(lib().tc_train(self.ctx, ds.h, C.byref(p), C.byref(h), C.byref(st)))
        return Model(self, h), st

    def train_regular(self, ds: Dataset, p: TrainParams):
        """tc_train_regular: regular (depth-wise) trees, the reference's mode="small"."""
        h = C.c_void_p()
        st = TrainStats()
        self._chk(lib().tc_train_regular(self.ctx, ds.h, C.byref(p), C.byref(h), C.byref(st)))
        return Model(self, h), st

    def build_tree(self, ds: Dataset, g, h, p: TrainParams, want_hist=False):
        g = np.ascontiguousarray(g, np.float32)
        h = np.ascontiguousarray(h, np.float32)
        D = p.max_depth
        dep = C.c_int32()
        sf = np.zeros(D, np.uint16)
        sb = np.zeros(D, np.uint8)
        st = np.zeros(D, np.float32)
        sg = np.zeros(D, np.float64)
        s2 = np.zeros(D, np.float64)
        lv = np.zeros(1 << D, np.float32)
        li = np.zeros(ds.n, np.uint32)
        rh = np.zeros((ds.f, 256, 2), np.float64) if want_hist else None
        self._chk(lib().tc_build_tree(self.ctx, ds.h, _p(g), _p(h), C.byref(p), C.byref(dep), _p(sf), _p(sb),
                                      _p(st), _p(sg), _p(s2), _p(lv), _p(li), _p(rh)))
        d = dep.value
        return dict(depth=d, feature=sf[:d], bin=sb[:d], threshold=st[:d], gain=sg[:d], second=s2[:d],
                    leaves=lv[: 1 << d], leaf_index=li, root_hist=rh)

    def import_model(self, info: ModelInfo, arrays: dict) -> Model:
        h = C.c_void_p()
        a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        self._chk(lib().tc_model_import(self.ctx, C.byref(info), *[_p(a.get(k)) for k in (
            "depth", "feature", "bin", "threshold", "gain", "leaves", "weights", "edges", "n_edges")], C.byref(h)))
        return Model(self, h)

    def load_tcat(self, data: bytes) -> Model:
        h = C.c_void_p()
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        self._chk(lib().tc_model_load_tcat(self.ctx, buf, C.c_size_t(len(data)), C.byref(h)))
        return Model(self, h)

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        self._chk(lib().tc_ctx_memory(self.ctx, C.byref(a), C.byref(b)))
        return a.value, b.value

    def fail_next_allocs(self, k):
        self._chk(lib().tc_ctx_fail_next_allocs(self.ctx, C.c_int(k)))

    def synchronize(self, timeout_ms=10000):
        self._chk(lib().tc_ctx_synchronize(self.ctx, C.c_int(timeout_ms)))

    def set_latency_worker(self, enabled):
        """Small predict requests through the persistent latency worker (True,
        the default) or one kernel launch each (False)."""
        self._chk(lib().tc_ctx_set_latency_worker(self.ctx, C.c_int(1 if enabled else 0)))

    def close(self):
        if self.ctx:
            lib().tc_ctx_destroy(self.ctx)
            self.ctx = None


class Server:
    def __init__(self, eng: Engine, staging_bytes=0, max_batch_rows=65536, coalesce=True, max_inflight=4):
        self.eng = eng
        self.h = C.c_void_p()
        p = ServerParams(staging_bytes, max_batch_rows, 1 if coalesce else 0, max_inflight)
        eng._chk(lib().tc_server_create(eng.ctx, C.byref(p), C.byref(self.h)))

    def add_model(self, m: Model) -> int:
        mid = C.c_int32()
        self.eng._chk(lib().tc_server_add_model(self.h, m.h, C.byref(mid)))
        return mid.value

    def submit(self, model_id, X, out, transform="raw"):
        n, f = X.shape
        t = C.c_uint64()
        self.eng._chk(lib().tc_server_submit(self.h, C.c_int32(model_id), _p(X), C.c_uint32(n), C.c_uint16(f),
                                             C.c_int32(TRANSFORM[transform]), _p(out), C.byref(t)))
        return t.value

    def poll(self, ticket, timeout_us=1_000_000):
        done = C.c_int()
        lat = C.c_double()
        st = lib().tc_server_poll(self.h, C.c_uint64(ticket), C.c_int64(timeout_us), C.byref(done), C.byref(lat))
        if st == 3:
            return False, None
        self.eng._chk(st)
        return bool(done.value), lat.value

    def replay(self, reqs):
        """reqs: list of (arrival_s, model_id, X, out, transform)."""
        arr = (ReplayRequest * len(reqs))()
        for i, (t, mid, X, out, tr) in enumerate(reqs):
            arr[i] = ReplayRequest(t, mid, TRANSFORM[tr], X.ctypes.data, out.ctypes.data, X.shape[0], X.shape[1], 0)
        lat = np.zeros(len(reqs), np.float64)
        wall = C.c_double()
        self.eng._chk(lib().tc_server_replay(self.h, arr, C.c_int32(len(reqs)), _p(lat), C.byref(wall)))
        return lat, wall.value

    def stats(self):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.eng._chk(lib().tc_server_stats(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def close(self):
        if self.h and lib is not None:  # at interpreter exit the module globals may be gone
            lib().tc_server_destroy(self.h)
            self.h = None

    __del__ = close
