"""ctypes bindings for the CPU oracle (liboracle.so) and the reference probe
(oracle/_ref/libtcref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, always as the checker or the timed
CPU baseline -- never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_DEPTH = 16

LOSS_IDS = {"logloss": 0, "mse": 1, "focal": 2, "softmax": 3}


def _ptr(a, t=C.c_void_p):
    return C.cast(a.ctypes.data, t) if a is not None else None


class TreeParams(C.Structure):
    _fields_ = [
        ("max_depth", C.c_int32),
        ("max_bins", C.c_int32),
        ("min_samples_leaf", C.c_int32),
        ("lambda_l2", C.c_float),
        ("lambda_l1", C.c_float),
        ("min_child_weight", C.c_float),
        ("min_split_gain", C.c_float),
        ("max_delta_step", C.c_float),
    ]


class TreeOut(C.Structure):
    _fields_ = [
        ("depth", C.c_int32),
        ("feature", C.c_uint16 * MAX_DEPTH),
        ("bin", C.c_uint8 * MAX_DEPTH),
        ("threshold", C.c_float * MAX_DEPTH),
        ("gain", C.c_float * MAX_DEPTH),
        ("gain_top", C.c_double * MAX_DEPTH),
        ("gain_second", C.c_double * MAX_DEPTH),
        ("n_candidates", C.c_uint32 * MAX_DEPTH),
    ]


class FitParams(C.Structure):
    _fields_ = [
        ("loss", C.c_int32),
        ("n_classes", C.c_int32),
        ("n_estimators", C.c_int32),
        ("learning_rate", C.c_float),
        ("focal_gamma", C.c_float),
        ("focal_alpha", C.c_float),
        ("tree", TreeParams),
        ("subsample", C.c_float),
        ("colsample_bytree", C.c_float),
        ("seed", C.c_uint64),
        ("use_goss", C.c_int32),
        ("goss_top_rate", C.c_float),
        ("goss_other_rate", C.c_float),
    ]


class RefParams(C.Structure):
    _fields_ = [
        ("loss", C.c_int32),
        ("n_classes", C.c_int32),
        ("n_estimators", C.c_int32),
        ("max_depth", C.c_int32),
        ("max_bins", C.c_int32),
        ("min_samples_leaf", C.c_int32),
        ("learning_rate", C.c_float),
        ("lambda_l2", C.c_float),
        ("lambda_l1", C.c_float),
        ("min_child_weight", C.c_float),
        ("min_split_gain", C.c_float),
        ("max_delta_step", C.c_float),
        ("regular", C.c_int32),
    ]


@dataclass
class Hyper:
    """Hyper-parameters shared by the oracle, the reference probe and the device path."""

    loss: str = "logloss"
    n_classes: int = 1
    n_estimators: int = 10
    learning_rate: float = 0.1
    max_depth: int = 6
    max_bins: int = 255
    min_samples_leaf: int = 1
    lambda_l2: float = 1.0
    lambda_l1: float = 0.0
    min_child_weight: float = 1.0
    min_split_gain: float = 0.0
    max_delta_step: float = 0.0
    focal_gamma: float = 2.0
    focal_alpha: float = 0.25
    subsample: float = 1.0          # row sampling per iteration (BoostingConfig::subsample)
    colsample_bytree: float = 1.0   # advances the random state only (symmetric trees ignore it)
    seed: int = 42                  # Config::seed
    use_goss: bool = False          # GOSS row sampling (chosen over subsample)
    goss_top_rate: float = 0.2
    goss_other_rate: float = 0.1
    regular_trees: bool = False     # reference probe only: regular (depth-wise) trees

    def tree(self) -> TreeParams:
        return TreeParams(self.max_depth, self.max_bins, self.min_samples_leaf, self.lambda_l2,
                          self.lambda_l1, self.min_child_weight, self.min_split_gain,
                          self.max_delta_step)

    def fit(self) -> FitParams:
        return FitParams(LOSS_IDS[self.loss], self.n_classes if self.loss == "softmax" else 1,
                         self.n_estimators, self.learning_rate, self.focal_gamma,
                         self.focal_alpha, self.tree(), self.subsample, self.colsample_bytree, self.seed,
                         1 if self.use_goss else 0, self.goss_top_rate, self.goss_other_rate)

    def ref(self) -> RefParams:
        return RefParams(LOSS_IDS[self.loss], self.n_classes if self.loss == "softmax" else 2,
                         self.n_estimators, self.max_depth, self.max_bins, self.min_samples_leaf,
                         self.learning_rate, self.lambda_l2, self.lambda_l1,
                         self.min_child_weight, self.min_split_gain, self.max_delta_step,
                         1 if self.regular_trees else 0)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (run `make -C oracle`)")
        _lib = C.CDLL(path)
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libtcref.so"))


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libtcref.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libtcref.so is not built (make -f oracle/ref.mk)")
        _ref = C.CDLL(path)
        _ref.tcref_last_error.restype = C.c_char_p
    return _ref


# ---------------------------------------------------------------- oracle --

@dataclass
class Binned:
    bins: np.ndarray      # uint8 [f][n]
    edges: np.ndarray     # float32 [f][255]
    n_edges: np.ndarray   # uint16 [f]

    def edge_list(self, j):
        return self.edges[j, : self.n_edges[j]]


def quantize(X: np.ndarray, max_bins: int = 255, compat_u8: bool = True) -> Binned:
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, f = X.shape
    bins = np.zeros((f, n), np.uint8)
    edges = np.zeros((f, 255), np.float32)
    ne = np.zeros(f, np.uint16)
    rc = lib().tco_quantize(_ptr(X), C.c_uint32(n), C.c_uint32(f), C.c_int32(max_bins),
                            C.c_int32(1 if compat_u8 else 0), _ptr(bins), _ptr(edges), _ptr(ne))
    if rc:
        raise ValueError(f"tco_quantize failed ({rc})")
    return Binned(bins, edges, ne)


def gradients(loss: str, y, pred, K: int = 1, gamma=2.0, alpha=0.25):
    y = np.ascontiguousarray(y, np.float32)
    pred = np.ascontiguousarray(pred, np.float32)
    g = np.empty_like(pred)
    h = np.empty_like(pred)
    n = y.shape[0]
    L = lib()
    if loss == "logloss":
        L.tco_grad_logloss(_ptr(y), _ptr(pred), _ptr(g), _ptr(h), C.c_uint32(n))
    elif loss == "mse":
        L.tco_grad_mse(_ptr(y), _ptr(pred), _ptr(g), _ptr(h), C.c_uint32(n))
    elif loss == "focal":
        L.tco_grad_focal(_ptr(y), _ptr(pred), _ptr(g), _ptr(h), C.c_uint32(n), C.c_float(gamma),
                         C.c_float(alpha))
    elif loss == "softmax":
        L.tco_grad_softmax(_ptr(y), _ptr(pred), _ptr(g), _ptr(h), C.c_uint32(n), C.c_uint32(K))
    else:
        raise ValueError(loss)
    return g, h


def next_random(state: int):
    """One xorshift64* draw (src/boosting/booster.cpp:1219-1225): (new state, output)."""
    st = C.c_uint64(state)
    lib().tco_next_random.restype = C.c_uint64
    out = lib().tco_next_random(C.byref(st))
    return st.value, out


def goss_subsample(absg, top_rate: float, other_rate: float, seed: int) -> np.ndarray:
    """Rows of one GOSS selection (src/core/dataset.cpp:494-549) over per-row |g|, in the reference's order."""
    absg = np.ascontiguousarray(absg, np.float32)
    n = len(absg)
    out = np.zeros(max(1, n), np.uint32)
    lib().tco_goss_subsample.restype = C.c_uint32
    m = lib().tco_goss_subsample(C.c_uint32(n), _ptr(absg), C.c_float(top_rate), C.c_float(other_rate),
                                 C.c_uint64(seed), _ptr(out))
    return out[:m]


def init_prediction(loss: str, y) -> float:
    y = np.ascontiguousarray(y, np.float32)
    L = lib()
    L.tco_init_prediction.restype = C.c_float
    return float(L.tco_init_prediction(C.c_int32(LOSS_IDS[loss]), _ptr(y), C.c_uint32(y.shape[0])))


@dataclass
class Tree:
    depth: int
    feature: np.ndarray
    bin: np.ndarray
    threshold: np.ndarray
    gain: np.ndarray
    gain_top: np.ndarray
    gain_second: np.ndarray
    leaves: np.ndarray
    leaf_index: np.ndarray | None = None
    root_hist: np.ndarray | None = None

    def margins(self):
        """Relative margin of the chosen split over the runner-up, per level."""
        out = []
        for d in range(self.depth):
            top, sec = self.gain_top[d], self.gain_second[d]
            out.append(np.inf if sec <= -1e29 else (top - sec) / max(abs(top), 1e-300))
        return np.array(out)


def build_tree(b: Binned, g, h, hp: Hyper, mode: int = 0, want_rows=True, want_hist=False) -> Tree:
    f, n = b.bins.shape
    g = np.ascontiguousarray(g, np.float32)
    h = np.ascontiguousarray(h, np.float32)
    out = TreeOut()
    leaves = np.zeros(1 << hp.max_depth, np.float32)
    li = np.zeros(n, np.uint32) if want_rows else None
    rh = np.zeros((f, 256, 2), np.float64) if want_hist else None
    tp = hp.tree()
    rc = lib().tco_build_tree(_ptr(b.bins), C.c_uint32(n), C.c_uint32(f), _ptr(b.edges),
                              _ptr(b.n_edges), _ptr(g), _ptr(h), C.byref(tp), C.c_int32(mode),
                              C.byref(out), _ptr(leaves), _ptr(li), _ptr(rh))
    if rc:
        raise RuntimeError(f"tco_build_tree failed ({rc})")
    d = out.depth
    return Tree(d, np.array(out.feature[:d], np.uint16), np.array(out.bin[:d], np.uint8),
                np.array(out.threshold[:d], np.float32), np.array(out.gain[:d], np.float32),
                np.array(out.gain_top[:MAX_DEPTH]), np.array(out.gain_second[:MAX_DEPTH]),
                leaves[: 1 << d].copy(), li, rh)


def histogram(b: Binned, g, h, node_of_row, n_nodes: int) -> np.ndarray:
    f, n = b.bins.shape
    g = np.ascontiguousarray(g, np.float32)
    h = np.ascontiguousarray(h, np.float32)
    nodes = np.ascontiguousarray(node_of_row, np.uint32)
    out = np.zeros((n_nodes, f, 256, 2), np.float64)
    lib().tco_histogram(_ptr(b.bins), C.c_uint32(n), C.c_uint32(f), _ptr(g), _ptr(h),
                        _ptr(nodes), C.c_uint32(n_nodes), _ptr(out))
    return out


@dataclass
class Ensemble:
    """A flat symmetric ensemble (the FastFloatEnsemble layout)."""

    base: float
    n_classes: int
    max_depth: int
    depth: np.ndarray       # int32 [T]
    feature: np.ndarray     # uint16 [T][D]
    bin: np.ndarray         # uint8 [T][D]
    threshold: np.ndarray   # float32 [T][D]
    leaves: np.ndarray      # float32 [T][2^D]
    weights: np.ndarray     # float32 [T]
    gain: np.ndarray | None = None
    min_margin: float = np.inf
    train_pred: np.ndarray | None = None
    bin_edges: list = field(default_factory=list)

    @property
    def n_trees(self):
        return int(self.depth.shape[0])


def fit(b: Binned, y, hp: Hyper, mode: int = 0, want_pred=True, trace=False) -> Ensemble:
    f, n = b.bins.shape
    y = np.ascontiguousarray(y, np.float32)
    K = hp.n_classes if hp.loss == "softmax" else 1
    T = hp.n_estimators * K
    D = hp.max_depth
    depth = np.zeros(T, np.int32)
    feat = np.zeros((T, D), np.uint16)
    bins_ = np.zeros((T, D), np.uint8)
    thr = np.zeros((T, D), np.float32)
    leaves = np.zeros((T, 1 << D), np.float32)
    tp = np.zeros((n, K), np.float32) if want_pred else None
    base = C.c_float()
    mm = C.c_double()
    gain = np.zeros((T, D), np.float32)
    gt = np.zeros((hp.n_estimators, n, K), np.float32) if trace else None
    ht = np.zeros((hp.n_estimators, n, K), np.float32) if trace else None
    fp = hp.fit()
    rc = lib().tco_fit(_ptr(b.bins), C.c_uint32(n), C.c_uint32(f), _ptr(b.edges), _ptr(b.n_edges),
                       _ptr(y), C.byref(fp), C.c_int32(mode), C.byref(base), _ptr(depth),
                       _ptr(feat), _ptr(bins_), _ptr(thr), _ptr(leaves), _ptr(tp), C.byref(mm),
                       _ptr(gain), _ptr(gt), _ptr(ht))
    if rc:
        raise RuntimeError(f"tco_fit failed ({rc})")
    e = Ensemble(base.value, K, D, depth, feat, bins_, thr, leaves,
                 np.full(T, hp.learning_rate, np.float32), gain, mm.value, tp,
                 [b.edge_list(j).copy() for j in range(f)])
    e.grad_trace, e.hess_trace = gt, ht
    return e


def predict(ens: Ensemble, X) -> np.ndarray:
    """FP64 raw scores [n][K] (base included)."""
    X = np.ascontiguousarray(X, np.float32)
    n, f = X.shape
    out = np.zeros((n, ens.n_classes), np.float64)
    depth = np.ascontiguousarray(ens.depth, np.int32)
    feat = np.ascontiguousarray(ens.feature, np.uint16)
    thr = np.ascontiguousarray(ens.threshold, np.float32)
    leaves = np.ascontiguousarray(ens.leaves, np.float32)
    w = np.ascontiguousarray(ens.weights, np.float32)
    lib().tco_predict(_ptr(X), C.c_uint32(n), C.c_uint32(f), C.c_int32(ens.n_trees),
                      C.c_int32(ens.n_classes), C.c_int32(ens.max_depth), _ptr(depth), _ptr(feat),
                      _ptr(thr), _ptr(leaves), _ptr(w), C.c_float(ens.base), _ptr(out))
    return out


# ------------------------------------------------------------- reference --

def ref_quantize(X, max_bins=255) -> Binned:
    X = np.ascontiguousarray(X, np.float32)
    n, f = X.shape
    bins = np.zeros((f, n), np.uint8)
    edges = np.zeros((f, 255), np.float32)
    ne = np.zeros(f, np.uint16)
    R = ref()
    rc = R.tcref_bin(_ptr(X), C.c_uint32(n), C.c_uint16(f), C.c_int32(max_bins), _ptr(bins),
                     _ptr(edges), _ptr(ne))
    if rc:
        raise RuntimeError(R.tcref_last_error().decode())
    return Binned(bins, edges, ne)


def ref_fit(X, y, hp: Hyper, trace=False, want_pred=True):
    """Reference Booster::train; returns (Binned, TCAT bytes, grad trace, hess trace, train raw).
    want_pred=False skips the train predictions (the multiclass loop's
    predictions are [n][K], which this wrapper does not collect)."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n, f = X.shape
    bins = np.zeros((f, n), np.uint8)
    edges = np.zeros((f, 255), np.float32)
    ne = np.zeros(f, np.uint16)
    gt = np.zeros((hp.n_estimators, n), np.float32) if trace else None
    ht = np.zeros((hp.n_estimators, n), np.float32) if trace else None
    tp = np.zeros(n, np.float32) if want_pred else None
    mb = C.c_void_p()
    ml = C.c_size_t()
    rp = hp.ref()
    R = ref()
    rc = R.tcref_fit(_ptr(X), C.c_uint32(n), C.c_uint16(f), _ptr(y), C.byref(rp), _ptr(bins),
                     _ptr(edges), _ptr(ne), _ptr(gt), _ptr(ht), _ptr(tp), C.byref(mb), C.byref(ml))
    if rc < 0:
        raise RuntimeError(R.tcref_last_error().decode())
    data = C.string_at(mb, ml.value)
    R.tcref_free(mb)
    return Binned(bins, edges, ne), data, gt, ht, tp



def ref_fit_timed(X, y, hp: Hyper, max_trees: int, max_seconds: float = 1e30):
    """Reference Booster::train (binary / regression) stopped through its
    training callback after max_trees trees or max_seconds; returns
    (seconds of from_dense + compute_bins, [seconds from the start to the end
    of each tree built])."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n, f = X.shape
    setup = np.zeros(1)
    ends = np.zeros(max(1, max_trees))
    rp = hp.ref()
    R = ref()
    rc = R.tcref_fit_timed(_ptr(X), C.c_uint32(n), C.c_uint16(f), _ptr(y), C.byref(rp), C.c_int32(max_trees),
                           C.c_double(max_seconds), _ptr(setup), _ptr(ends))
    if rc < 0:
        raise RuntimeError(R.tcref_last_error().decode())
    return float(setup[0]), [float(v) for v in ends[:rc]]

def ref_predict(model: bytes, X, proba=False) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32)
    n, f = X.shape
    out = np.zeros(n, np.float32)
    R = ref()
    rc = R.tcref_predict(C.c_char_p(model), C.c_size_t(len(model)), _ptr(X), C.c_uint32(n),
                         C.c_uint16(f), C.c_int32(1 if proba else 0), _ptr(out))
    if rc:
        raise RuntimeError(R.tcref_last_error().decode())
    return out


def ref_build_tree(X, g, h, hp: Hyper):
    X = np.ascontiguousarray(X, np.float32)
    n, f = X.shape
    g = np.ascontiguousarray(g, np.float32)
    h = np.ascontiguousarray(h, np.float32)
    sf = np.zeros(64, np.uint16)
    sb = np.zeros(64, np.uint8)
    st = np.zeros(64, np.float32)
    sg = np.zeros(64, np.float32)
    lv = np.zeros(1 << hp.max_depth, np.float32)
    rp = hp.ref()
    R = ref()
    d = R.tcref_build_tree(_ptr(X), C.c_uint32(n), C.c_uint16(f), _ptr(g), _ptr(h), C.byref(rp),
                           _ptr(sf), _ptr(sb), _ptr(st), _ptr(sg), _ptr(lv))
    if d < 0:
        raise RuntimeError(R.tcref_last_error().decode())
    return d, sf[:d], sb[:d], st[:d], sg[:d], lv[: 1 << d]


def ref_fit_multiclass(X, y, hp: Hyper):
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n, f = X.shape
    K, D = hp.n_classes, hp.max_depth
    T = hp.n_estimators * K
    depth = np.zeros(T, np.int32)
    sf = np.zeros((T, D), np.uint16)
    sb = np.zeros((T, D), np.uint8)
    st = np.zeros((T, D), np.float32)
    lv = np.zeros((T, 1 << D), np.float32)
    tp = np.zeros((n, K), np.float32)
    rp = hp.ref()
    R = ref()
    rc = R.tcref_fit_multiclass(_ptr(X), C.c_uint32(n), C.c_uint16(f), _ptr(y), C.byref(rp),
                                _ptr(depth), _ptr(sf), _ptr(sb), _ptr(st), _ptr(lv), _ptr(tp))
    if rc:
        raise RuntimeError(R.tcref_last_error().decode())
    return depth, sf, sb, st, lv, tp


# --------------------------------------------------------------- TCAT v3 --

def parse_tcat(data: bytes) -> Ensemble:
    """Parse a TCAT v3 symmetric model (src/boosting/booster.cpp:1049-1118,
    src/tree/symmetric_tree.cpp:1199-1215); host-endian, size_t = 8 bytes."""
    off = 0

    def take(fmt):
        nonlocal off
        v = struct.unpack_from("<" + fmt, data, off)
        off += struct.calcsize("<" + fmt)
        return v

    if data[:4] != b"TCAT":
        raise ValueError("not a TCAT stream")
    off = 4
    (version,) = take("I")
    if version != 3:
        raise ValueError(f"TCAT version {version} not supported here")
    (base,) = take("f")
    (task,) = take("B")
    (n_classes,) = take("I")
    (lr,) = take("f")
    (max_depth,) = take("H")
    (lam,) = take("f")
    (sym,) = take("B")
    if not sym:
        raise ValueError("not a symmetric-tree model")
    (nf,) = take("Q")
    edges = []
    for _ in range(nf):
        (ne,) = take("Q")
        edges.append(np.array(take(f"{ne}f"), np.float32) if ne else np.zeros(0, np.float32))
    (nt,) = take("Q")
    weights = np.array(take(f"{nt}f"), np.float32) if nt else np.zeros(0, np.float32)
    D = max_depth
    depth = np.zeros(nt, np.int32)
    feat = np.zeros((nt, D), np.uint16)
    bins_ = np.zeros((nt, D), np.uint8)
    thr = np.zeros((nt, D), np.float32)
    gain = np.zeros((nt, D), np.float32)
    leaves = np.zeros((nt, 1 << D), np.float32)
    for t in range(nt):
        (d,) = take("H")
        depth[t] = d
        for k in range(d):
            (feat[t, k],) = take("H")
            (bins_[t, k],) = take("B")
            (thr[t, k],) = take("f")
            (gain[t, k],) = take("f")
        (nl,) = take("Q")
        leaves[t, :nl] = np.array(take(f"{nl}f"), np.float32)
    e = Ensemble(base, 1, D, depth, feat, bins_, thr, leaves, weights, gain)
    e.bin_edges = edges
    return e


# --------------------------------------------------------- early stopping --

def early_stopping(ens: Ensemble, Xv, yv, loss: str, n_estimators: int, rounds: int,
                   learning_rate: float, focal_gamma=2.0, focal_alpha=0.25):
    """Validation loss per iteration and the stopping iteration of
    Booster::train's valid_data branch (src/boosting/booster.cpp:255-371;
    multiclass 1405-1435), replayed over the iterations of `ens`:
    valid_pred += lr * leaf (FP32, fused multiply-add as the compiled
    reference), the loss's compute_loss term per row in FP32
    (src/boosting/loss.cpp:110-121, 232-244, 336-346, 475-503) summed in
    FP64, improvement when loss < best - 1e-10 (FP32), stop once
    iteration >= max(50, n_estimators / 10) and `rounds` iterations in a row
    did not improve.  Returns (losses, stop_iteration or -1, best_iteration)."""
    Xv = np.ascontiguousarray(Xv, np.float32)
    yv = np.ascontiguousarray(yv, np.float32)
    K = ens.n_classes
    nv = Xv.shape[0]
    iters = ens.n_trees // K
    pred = np.full((nv, K), np.float32(ens.base), np.float32)
    best, best_it, no_imp = np.float32(1e30), 0, 0
    min_it = max(50, n_estimators // 10)
    losses = []
    f32 = np.float32
    for it in range(iters):
        for k in range(K):
            t = it * K + k
            idx = np.zeros(nv, np.int64)
            for d in range(int(ens.depth[t])):
                idx = idx * 2 + (Xv[:, ens.feature[t, d]] >= ens.threshold[t, d])
            v = ens.leaves[t, idx].astype(np.float64)
            pred[:, k] = (np.float64(f32(learning_rate)) * v + pred[:, k].astype(np.float64)).astype(np.float32)
        if loss == "mse":
            diff = pred[:, 0] - yv
            term = diff * diff
        elif loss == "logloss":
            p = f32(1) / (f32(1) + np.exp(-pred[:, 0]))
            p = np.clip(p, f32(1e-7), f32(1) - f32(1e-7))
            term = -yv * np.log(p) - (f32(1) - yv) * np.log(f32(1) - p)
        elif loss == "focal":
            p = f32(1) / (f32(1) + np.exp(-pred[:, 0]))
            pt = yv * p + (f32(1) - yv) * (f32(1) - p)
            robust = f32(1) - f32(0.1) * np.abs(f32(2) * pt - f32(1)) ** f32(2)
            pt = np.maximum(pt, f32(1e-7))
            at = yv * f32(focal_alpha) + (f32(1) - yv) * (f32(1) - f32(focal_alpha))
            term = -at * (f32(1) - pt) ** f32(focal_gamma) * robust * np.log(pt)
        else:  # softmax cross entropy
            z = pred - pred.max(axis=1, keepdims=True)
            e = np.exp(z)
            pl = e[np.arange(nv), yv.astype(np.int64)] / e.sum(axis=1)
            term = -np.log(np.maximum(pl, f32(1e-7)))
        lv = float(np.sum(term.astype(np.float64)) / nv)
        losses.append(lv)
        if f32(lv) < best - f32(1e-10):
            best, best_it, no_imp = f32(lv), it, 0
        else:
            no_imp += 1
        if rounds >= 0 and it >= min_it and no_imp >= rounds:
            return np.array(losses), it, best_it
    return np.array(losses), -1, best_it


# ------------------------------------------------ regular (depth-wise) trees --
# Serving of models the reference trained with regular trees (mode="small").

@dataclass
class RegularModel:
    base: float
    task: int
    n_classes: int
    learning_rate: float
    max_depth: int
    lambda_l2: float
    edges: list          # per feature: float32 array of its bin edges
    weights: np.ndarray  # [T] float32
    trees: list          # per tree: dict of node arrays (feature, split_bin, is_leaf, left, right, value)


def parse_tcat_regular(data: bytes) -> RegularModel:
    """TCAT v3 holding regular trees: Booster::save_binary / load_binary
    (src/boosting/booster.cpp:1049-1110, 1140-1203) and Tree::save / load
    (src/tree/tree.cpp:1748-1840): per tree depth u16, classes u32, nodes u32,
    leaves u16, max_depth u16, lambda f32, then 16-byte nodes (feature u16,
    bin u8, flags u8 = is_leaf | default_left << 1, left u16, right u16,
    value f32, gain f32)."""
    import struct

    o = 0

    def rd(fmt):
        nonlocal o
        v = struct.unpack_from("<" + fmt, data, o)
        o += struct.calcsize("<" + fmt)
        return v if len(v) > 1 else v[0]

    assert data[:4] == b"TCAT"
    o = 4
    assert rd("I") == 3
    base = rd("f")
    task = rd("B")
    ncls = rd("I")
    lr = rd("f")
    md = rd("H")
    lam = rd("f")
    assert rd("B") == 0, "symmetric model"
    nf = rd("Q")
    edges = []
    for _ in range(nf):
        k = rd("Q")
        edges.append(np.frombuffer(data, np.float32, k, o).copy())
        o += 4 * k
    nt = rd("Q")
    w = np.frombuffer(data, np.float32, nt, o).copy()
    o += 4 * nt
    trees = []
    for _ in range(nt):
        _depth, tcls, nn, _nl, _md, _lam = rd("HIIHHf")
        rec = np.frombuffer(data, np.dtype([("feature", "<u2"), ("bin", "u1"), ("flags", "u1"), ("left", "<u2"),
                                            ("right", "<u2"), ("value", "<f4"), ("gain", "<f4")]), nn, o)
        o += 16 * nn
        assert tcls <= 1, "multiclass regular trees"
        trees.append(dict(feature=rec["feature"].astype(np.int64), split_bin=rec["bin"].astype(np.int64),
                          is_leaf=(rec["flags"] & 1).astype(bool), left=rec["left"].astype(np.int64),
                          right=rec["right"].astype(np.int64), value=rec["value"].copy()))
    return RegularModel(base, task, ncls, lr, md, lam, edges, w, trees)


def bin_regular(X, edges):
    """The reference's binning of prediction rows for regular trees
    (Booster::predict_raw_fast, src/boosting/booster.cpp:706-845): NaN -> 255;
    a feature of at most 16 edges takes the number of edges <= x (its linear
    scan), one of more edges std::lower_bound, the number of edges < x."""
    X = np.asarray(X, np.float32)
    out = np.zeros(X.shape, np.int64)
    for j, e in enumerate(edges):
        col = X[:, j]
        if len(e) == 0:
            b = np.zeros(len(col), np.int64)
        elif len(e) <= 16:
            b = np.searchsorted(e, col, side="right")
        else:
            b = np.searchsorted(e, col, side="left")
        out[:, j] = np.where(np.isnan(col), 255, b)
    return out


def predict_regular(m: RegularModel, X, fp64=False):
    """Raw scores (base included) of a regular-tree model
    (TreeEnsemble::predict_batch_optimized, src/tree/tree.cpp:1471-1560): per
    row, trees in order, walk to a leaf going right iff bin != 255 and
    bin > split_bin, sum += weight * value (one fused multiply-add in the
    reference's FP32 build; emulated through FP64), then + base."""
    B = bin_regular(X, m.edges)
    n = B.shape[0]
    out = np.zeros(n, np.float64 if fp64 else np.float32)
    for i in range(n):
        row = B[i]
        s = 0.0 if fp64 else np.float32(0.0)
        for t, tr in enumerate(m.trees):
            node = 0
            while not tr["is_leaf"][node]:
                b = row[tr["feature"][node]]
                node = tr["right"][node] if (b != 255 and b > tr["split_bin"][node]) else tr["left"][node]
            v = float(tr["value"][node])
            if fp64:
                s += float(m.weights[t]) * v
            else:
                s = np.float32(float(m.weights[t]) * v + float(s))
        out[i] = (s + m.base) if fp64 else np.float32(s + np.float32(m.base))
    return out


# ------------------------------------------- categorical target statistics --
# Dataset::compute_target_statistics and its two methods
# (src/core/dataset.cpp:679-865), the target-statistics binning rule of
# Dataset::compute_bins (src/core/dataset.cpp:183-240) and the categorical
# branch of Dataset::apply_bins (src/core/dataset.cpp:362-372), restated in
# float32 with the reference's order of additions.

F32 = np.float32


def category_of(v):
    """static_cast<Index>(val) as x86-64 compiles it (truncate to int64, keep the low 32 bits)."""
    return int(np.int64(np.trunc(v))) & 0xFFFFFFFF


def label_prior(y) -> np.float32:
    """std::accumulate(labels, 0.0f) / n_samples (src/core/dataset.cpp:685)."""
    acc = np.add.accumulate(np.asarray(y, F32), dtype=F32)[-1] if len(y) else F32(0)
    return F32(F32(acc) / F32(len(y)))


def _smooth(s, c, wp, pw):
    return F32(F32(F32(s) + wp) / F32(F32(c) + pw))


def ordered_ts(X, y, feats, order, prior_weight=1.0):
    """Ordered target statistics (src/core/dataset.cpp:722-780) with the
    processing order `order` (row of each position).  Returns (encoded X copy,
    {feature: (sorted categories, encodings)}, prior)."""
    X = np.array(X, F32, copy=True)
    y = np.asarray(y, F32)
    prior = label_prior(y)
    pw = F32(prior_weight)
    wp = F32(pw * prior)
    tables = {}
    for j in feats:
        col = X[:, j].copy()
        run = {}
        for row in order:
            v = col[row]
            if np.isnan(v):
                X[row, j] = prior
                continue
            c = category_of(v)
            s, k = run.get(c, (F32(0), 0))
            X[row, j] = _smooth(s, k, wp, pw) if k else prior
            run[c] = (F32(s + y[row]), k + 1)
        keys = np.array(sorted(run), np.uint32)
        tables[j] = (keys, np.array([_smooth(*run[int(c)], wp, pw) for c in keys], F32))
    return X, tables, prior


def cv_ts(X, y, feats, folds, n_folds, prior_weight=1.0):
    """Cross-validated target statistics (src/core/dataset.cpp:783-865) with
    each row's fold given."""
    X = np.array(X, F32, copy=True)
    y = np.asarray(y, F32)
    prior = label_prior(y)
    pw = F32(prior_weight)
    wp = F32(pw * prior)
    tables = {}
    for j in feats:
        col = X[:, j].copy()
        fs = {}
        for row in range(len(col)):
            v = col[row]
            if np.isnan(v):
                continue
            c = category_of(v)
            st = fs.setdefault(c, [[F32(0), 0] for _ in range(n_folds)])
            st[folds[row]][0] = F32(st[folds[row]][0] + y[row])
            st[folds[row]][1] += 1
        for row in range(len(col)):
            v = col[row]
            if np.isnan(v):
                X[row, j] = prior
                continue
            st = fs[category_of(v)]
            s, k = F32(0), 0
            for q in range(n_folds):
                if q != folds[row]:
                    s = F32(s + st[q][0])
                    k += st[q][1]
            X[row, j] = _smooth(s, k, wp, pw)
        keys = np.array(sorted(fs), np.uint32)
        vals = []
        for c in keys:
            s, k = F32(0), 0
            for q in range(n_folds):
                s = F32(s + fs[int(c)][q][0])
                k += fs[int(c)][q][1]
            vals.append(_smooth(s, k, wp, pw))
        tables[j] = (keys, np.array(vals, F32))
    return X, tables, prior


def quantize_ts(X, ts_feats, max_bins=255, compat_u8=True) -> Binned:
    """compute_bins with target-statistics columns: numeric columns by the
    quantile rule (quantize), TS columns by A = min(max_bins, U) edges, edge b
    = the distinct value of rank (b+1)*U/(A+1), bin = number of edges < x
    (std::lower_bound), NaN -> bin max_bins."""
    X = np.ascontiguousarray(X, F32)
    b = quantize(X, max_bins, compat_u8)
    for j in ts_feats:
        v = X[:, j]
        ok = ~np.isnan(v)
        u = np.unique(v[ok])
        U = len(u)
        b.edges[j] = 0
        if U == 0:
            b.edges[j, 0] = 0.0
            b.n_edges[j] = 1
            b.bins[j] = max_bins
            continue
        A = min(max_bins, (U & 255) if compat_u8 else U)
        e = np.array([u[min((k + 1) * U // (A + 1), U - 1)] for k in range(A)], F32)
        b.edges[j, :A] = e
        b.n_edges[j] = A
        bins = np.searchsorted(e, v, side="left")
        bins[~ok] = max_bins
        b.bins[j] = bins.astype(np.uint8)
    return b


def encode_test(X, tables):
    """apply_bins' categorical branch: category -> global encoding, 0.5 for an
    unseen one (include/turbocat/dataset.hpp:218-226); NaN stays NaN."""
    X = np.array(X, F32, copy=True)
    for j, (keys, vals) in tables.items():
        lut = {int(k): v for k, v in zip(keys, vals)}
        for r in range(X.shape[0]):
            v = X[r, j]
            if not np.isnan(v):
                X[r, j] = lut.get(category_of(v), F32(0.5))
    return X


def recover_order(X, y, feat, enc, prior_weight=1.0):
    """A processing order under which ordered_ts reproduces the per-row
    encodings `enc` of one categorical column (the reference draws its order
    from std::random_device).  Within a category the position of each row is
    found by stepping the running (sum, count) and matching the encodings;
    rows of equal (encoding, label) are interchangeable, and the label to take
    next is the one whose successor encoding exists.  Raises when the
    encodings fit no order."""
    X = np.asarray(X, F32)
    y = np.asarray(y, F32)
    prior = label_prior(y)
    pw = F32(prior_weight)
    wp = F32(pw * prior)
    col = X[:, feat]
    by_cat = {}
    nan_rows = []
    for r in range(len(col)):
        if np.isnan(col[r]):
            if enc[r] != prior:
                raise ValueError(f"NaN row {r} not encoded with the prior")
            nan_rows.append(r)
        else:
            by_cat.setdefault(category_of(col[r]), []).append(r)
    pos = {}
    for c, rows in by_cat.items():
        pool = {}  # encoding bits -> label -> rows
        for r in rows:
            pool.setdefault(enc[r].view(np.uint32).item(), {}).setdefault(y[r].item(), []).append(r)

        def target(s, k):
            return (prior if k == 0 else _smooth(s, k, wp, pw)).view(np.uint32).item()

        def solve(s, k):  # depth-first over the label taken at each step
            if k == len(rows):
                return []
            cand = pool.get(target(s, k), {})
            for lab in sorted(lb for lb, v in cand.items() if v):
                r = cand[lab].pop()
                rest = solve(F32(s + F32(lab)), k + 1)
                if rest is not None:
                    return [r] + rest
                cand[lab].append(r)
            return None

        import sys
        sys.setrecursionlimit(max(sys.getrecursionlimit(), 4 * len(rows) + 100))
        seq = solve(F32(0), 0)
        if seq is None:
            raise ValueError(f"category {c}: the encodings fit no order")
        for k, r in enumerate(seq):
            pos[r] = (k, c)
    order = sorted(pos, key=lambda r: pos[r]) + nan_rows
    return np.array(order, np.uint32)


def recover_folds(X, y, feat, enc, n_folds, prior_weight=1.0):
    """Fold ids under which cv_ts reproduces the per-row encodings `enc` of
    one categorical column: per category, rows with equal out-of-fold
    (sum, count) form whole folds of equal size and label sum; each group is
    split into folds of that size.  Raises when that is impossible."""
    X = np.asarray(X, F32)
    y = np.asarray(y, F32)
    prior = label_prior(y)
    pw = F32(prior_weight)
    wp = F32(pw * prior)
    col = X[:, feat]
    folds = np.zeros(len(col), np.uint32)
    by_cat = {}
    for r in range(len(col)):
        if not np.isnan(col[r]):
            by_cat.setdefault(category_of(col[r]), []).append(r)
    for c, rows in by_cat.items():
        N, P = len(rows), F32(np.add.accumulate(y[rows], dtype=F32)[-1])
        groups = {}
        for r in rows:
            groups.setdefault(enc[r].view(np.uint32).item(), []).append(r)
        q = 0
        for e, grp in groups.items():
            match = None
            gsum = F32(np.add.accumulate(y[grp], dtype=F32)[-1])
            for nf in range(1, N + 1):  # fold size: the out-of-fold count is N - nf
                if len(grp) % nf:
                    continue
                m = len(grp) // nf
                pos = gsum / F32(m)
                if _smooth(F32(P - pos), N - nf, wp, pw).view(np.uint32).item() == e:
                    match = nf
                    break
            if match is None:
                raise ValueError(f"category {c}: encoding fits no fold")
            labs = sorted(grp, key=lambda r: y[r])
            m = len(grp) // match
            for i in range(m):  # deal rows so every fold gets the same label mix
                for r in labs[i::m]:
                    folds[r] = q
                q += 1
            if q > n_folds:
                raise ValueError(f"category {c}: more than {n_folds} folds")
    return folds


def ref_cat_ts(X, y, cats, method="ordered", hp: Hyper | None = None, fit=False):
    """The reference's target statistics, bins and (fit) model on one dataset:
    (encodings [n_cat][n], Binned, {feature: (categories, encodings)}, TCAT or None)."""
    X = np.ascontiguousarray(X, F32)
    y = np.ascontiguousarray(y, F32)
    n, f = X.shape
    cats = np.ascontiguousarray(cats, np.uint16)
    nc = len(cats)
    hp = hp or Hyper(loss="logloss", n_estimators=1)
    enc = np.zeros((nc, n), F32)
    bins = np.zeros((f, n), np.uint8)
    edges = np.zeros((f, 255), F32)
    ne = np.zeros(f, np.uint16)
    cap = n
    tk = np.zeros((nc, cap), np.uint32)
    tv = np.zeros((nc, cap), F32)
    tl = np.zeros(nc, np.uint32)
    mb = C.c_void_p()
    ml = C.c_size_t()
    rp = hp.ref()
    R = ref()
    rc = R.tcref_cat_ts(_ptr(X), C.c_uint32(n), C.c_uint16(f), _ptr(y), _ptr(cats), C.c_int32(nc),
                        C.c_int32(1 if method == "cv" else 0), C.byref(rp), C.c_int32(1 if fit else 0), _ptr(enc),
                        _ptr(bins), _ptr(edges), _ptr(ne), _ptr(tk), _ptr(tv), _ptr(tl), C.c_uint32(cap),
                        C.byref(mb), C.byref(ml))
    if rc < 0:
        raise RuntimeError(R.tcref_last_error().decode())
    model = None
    if fit:
        model = C.string_at(mb, ml.value)
        R.tcref_free(mb)
    tables = {int(cats[c]): (tk[c, :tl[c]].copy(), tv[c, :tl[c]].copy()) for c in range(nc)}
    return enc, Binned(bins, edges, ne), tables, model


# ------------------------------------------------- regular (depth-wise) trees --
# Tree::build / build_recursive_optimized (src/tree/tree.cpp:162-407),
# SplitFinder::find_best_split(_feature) (src/tree/histogram.cpp:569-660),
# Tree::make_leaf (src/tree/tree.cpp:655-683) and Booster::build_tree's
# regular branch (src/boosting/booster.cpp:447-520), restated in FP64
# arithmetic: the reference's histograms are FP32 sums, so this oracle agrees
# with it wherever a node's top gain beats the runner-up by more than the
# FP32 error (the margin each node records).


def _regular_hist(bins, rows, g, h, max_bins, dt):
    """The node's histogram as the reference builds it (CPUHistogramBuilder::
    build, src/tree/histogram.cpp:62-176): per feature, the rows in order,
    each added into its bin (FP32 adds in that order when dt is float32); one
    row of max_bins slots per feature, a bin of max_bins or more (NaN: 255)
    landing in the following feature's slots, as the reference's flat array
    does."""
    f = bins.shape[0]
    idx = (np.arange(f)[:, None] * max_bins + bins[:, rows].astype(np.int64)).ravel()
    size = f * max_bins + 256
    G = np.zeros(size, dt)
    H = np.zeros(size, dt)
    np.add.at(G, idx, np.tile(np.asarray(g, dt)[rows], f))  # unbuffered: in index order
    np.add.at(H, idx, np.tile(np.asarray(h, dt)[rows], f))
    N = np.bincount(idx, None, size).astype(np.int64)
    k = f * max_bins
    return G[:k].reshape(f, max_bins), H[:k].reshape(f, max_bins), N[:k].reshape(f, max_bins)


def _regular_scan(hist, st, hp: Hyper, dt):
    """SplitFinder::find_best_split over a node's histogram (src/tree/histogram.cpp:569-660):
    left = prefix over bins 0 .. max_bins-2, right = node stats - left, both
    meeting min_samples_leaf and min_child_weight, gain 0.5 (GL^2/(HL+l) +
    GR^2/(HR+l) - G^2/(H+l)), first maximum in (feature, bin) order.  Returns
    (gain, runner-up gain of another partition, feature, bin, left stats,
    right stats) or None."""
    G, H, C = st
    lam, half, gamma = dt(hp.lambda_l2), dt(0.5), dt(0.0)
    msg, mcw, nb = dt(hp.min_split_gain), dt(hp.min_child_weight), int(hp.max_bins)
    HG, HH, HN = hist
    GL = np.cumsum(HG[:, : nb - 1], 1, dtype=dt)
    HL = np.cumsum(HH[:, : nb - 1], 1, dtype=dt)
    NL = np.cumsum(HN[:, : nb - 1], 1)
    GR, HR, NR = (G - GL).astype(dt), (H - HL).astype(dt), C - NL
    ok = (NL >= hp.min_samples_leaf) & (HL >= mcw) & (NR >= hp.min_samples_leaf) & (HR >= mcw)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        pg = dt(G * G) / dt(H + lam)
        gain = (half * (((GL * GL) / (HL + lam) + (GR * GR) / (HR + lam)) - pg) - gamma).astype(dt)
    gain = np.where(ok & (gain >= msg), gain, -np.inf)
    flat = gain.ravel()
    k = int(np.argmax(flat))  # first maximum in (feature, bin) order
    if not np.isfinite(flat[k]) or flat[k] <= -1e30:
        return None
    top = flat[k]
    other = flat[flat != top]
    second = other.max() if other.size else -np.inf
    fi, bi = divmod(k, nb - 1)
    return top, second, fi, bi, (GL[fi, bi], HL[fi, bi], NL[fi, bi]), (GR[fi, bi], HR[fi, bi], NR[fi, bi])


def build_regular_tree(b: Binned, g, h, hp: Hyper, rows=None, fp32=True):
    """One regular tree from the given gradients.  fp32: the reference's
    arithmetic (FP32 histograms in row order, the larger child's histogram as
    parent - smaller, FP32 prefix sums and gains); else FP64.  Returns the
    node arrays in the reference's numbering (children added in pairs, the
    smaller child's subtree built first) with each split node's margin (top
    gain - best gain of another partition) / |top gain| and each row's leaf."""
    dt = np.float32 if fp32 else np.float64
    bins = b.bins
    n = bins.shape[1]
    rows = np.arange(n) if rows is None else np.asarray(rows)
    lam = dt(hp.lambda_l2)
    mcw = dt(hp.min_child_weight)
    nb = int(hp.max_bins)
    max_leaves = 64  # TreeConfig::max_leaves (include/turbocat/config.hpp:29)
    keys = (("feature", 0), ("split_bin", 0), ("is_leaf", True), ("default_left", True), ("left", 0),
            ("right", 0), ("value", 0.0), ("gain", 0.0), ("margin", np.inf))
    nodes = {k: [v] for k, v in keys}
    leaf_of = np.zeros(n, np.int64)
    state = {"n_leaves": 0}

    def add_node():
        for k, v in keys:
            nodes[k].append(v)
        return len(nodes["value"]) - 1

    def make_leaf(i, st, r):
        v = dt(-st[0]) / dt(st[1] + lam)
        if hp.max_delta_step > 0:
            v = max(dt(-hp.max_delta_step), min(dt(hp.max_delta_step), v))
        nodes["is_leaf"][i] = True
        nodes["value"][i] = v
        leaf_of[r] = i
        state["n_leaves"] += 1

    def rec(i, r, st, hist, depth):
        G, H, C = st
        if (depth >= hp.max_depth or state["n_leaves"] >= max_leaves or len(r) < 2 * hp.min_samples_leaf
                or H < dt(2) * mcw):
            make_leaf(i, st, r)
            return
        sp = _regular_scan(hist, st, hp, dt)
        if sp is None:
            make_leaf(i, st, r)
            return
        top, second, fi, bi, sl, sr = sp
        nodes["feature"][i], nodes["split_bin"][i] = fi, bi
        nodes["is_leaf"][i] = False
        nodes["gain"][i] = top
        nodes["margin"][i] = float((top - second) / abs(top)) if np.isfinite(second) and top != 0 else np.inf
        col = bins[fi, r]
        go_left = np.where(col == 255, True, col <= bi)  # NaN: default_left (1 while partitioning)
        rl, rr = r[go_left], r[~go_left]
        if len(rl) != len(r) and len(rr) != len(r):
            nodes["default_left"][i] = len(rl) >= len(rr)
        li = add_node()
        ri = add_node()
        nodes["left"][i], nodes["right"][i] = li, ri
        small_left = len(rl) <= len(rr)
        hs = _regular_hist(bins, rl if small_left else rr, g, h, nb, dt)
        hb = tuple((p - q).astype(p.dtype) for p, q in zip(hist, hs))  # larger = parent - smaller
        if small_left:
            rec(li, rl, sl, hs, depth + 1)
            rec(ri, rr, sr, hb, depth + 1)
        else:
            rec(ri, rr, sr, hs, depth + 1)
            rec(li, rl, sl, hb, depth + 1)

    g_r = np.asarray(g, dt)[rows]
    h_r = np.asarray(h, dt)[rows]
    root = (np.add.accumulate(g_r, dtype=dt)[-1], np.add.accumulate(h_r, dtype=dt)[-1], len(rows))
    rec(0, rows, root, _regular_hist(bins, rows, g, h, nb, dt), 0)
    out = {k: np.array(v) for k, v in nodes.items()}
    out["value"] = out["value"].astype(np.float32)
    out["leaf_of"] = leaf_of
    return out


def fit_regular(b: Binned, y, hp: Hyper, grads=None, fp32=True):
    """Booster::train with regular trees (binary logloss / MSE, all rows, no
    sampling): base prediction, then per iteration the gradients of the FP32
    predictions, one tree, predictions += lr * leaf (one FP32 rounding).  With `grads`
    ((g, h) per iteration, e.g. the reference's own) the trees are built from
    those instead (teacher forcing).  Returns (trees, FP32 train predictions)."""
    y = np.asarray(y, np.float32)
    base = init_prediction(hp.loss, y)
    pred = np.full(len(y), base, np.float32)
    lr = np.float32(hp.learning_rate)
    trees = []
    for it in range(hp.n_estimators):
        if grads is None:
            g, h = gradients(hp.loss, y, pred)
        else:
            g, h = grads[0][it], grads[1][it]
        t = build_regular_tree(b, g, h, hp, fp32=fp32)
        trees.append(t)
        leaf = t["value"].astype(np.float32)[t["leaf_of"]]
        # predictions += lr * leaf, a fused multiply-add in the reference's build:
        # the product is exact in 80-bit precision, one rounding to float32
        pred = (pred.astype(np.longdouble) + np.longdouble(lr) * leaf.astype(np.longdouble)).astype(np.float32)
    return trees, pred, base


def build_regular_tree_levelwise(b: Binned, g, h, hp: Hyper):
    """The device's way to the same tree (FP64): grow every node level by
    level (stop rules other than the leaf cap decided when a child is made),
    then replay the reference's recursion -- smaller child first, a node
    visited with 64 leaves made becomes a leaf -- to apply the cap and number
    the nodes.  Equal to build_regular_tree(fp32=False) by construction of
    the replay; checked by the tests."""
    bins = b.bins
    n = bins.shape[1]
    g = np.asarray(g, np.float64)
    h = np.asarray(h, np.float64)
    lam, mcw, msl, nb = float(hp.lambda_l2), float(hp.min_child_weight), int(hp.min_samples_leaf), int(hp.max_bins)
    grown = [dict(depth=0, split=False)]
    slot = np.zeros(n, np.int64)
    open_ids, d = [0], 0
    while open_ids:
        nxt, feat, thr, ls, rs = [], [], [], [], []
        for a, gi in enumerate(open_ids):
            rows = np.nonzero(slot == a)[0]
            HG, HH, HN = _regular_hist(bins, rows, g, h, nb, np.float64)
            G, H, C = g[rows].sum(), h[rows].sum(), len(rows)
            GL, HL, CL = (np.cumsum(x[:, : nb - 1], 1) for x in (HG, HH, HN))
            GR, HR, CR = G - GL, H - HL, C - CL
            ok = (CL >= msl) & (CR >= msl) & (HL >= mcw) & (HR >= mcw)
            gain = 0.5 * ((GL * GL / (HL + lam) + GR * GR / (HR + lam)) - G * G / (H + lam))
            gain = np.where(ok & (gain >= hp.min_split_gain), gain, -np.inf).ravel()
            k = int(np.argmax(gain))
            nd = grown[gi]
            if d == 0:
                nd.update(G=G, H=H, C=C)
            feat.append(-1), thr.append(0), ls.append(-1), rs.append(-1)
            if (d == 0 and (C < 2 * msl or H < 2 * mcw)) or not np.isfinite(gain[k]):
                continue
            fi, bi = divmod(k, nb - 1)
            nd.update(split=True, feature=fi, bin=bi)
            feat[a], thr[a] = fi, bi
            for side, (cg, ch, cc) in enumerate(((GL[fi, bi], HL[fi, bi], CL[fi, bi]),
                                                 (GR[fi, bi], HR[fi, bi], CR[fi, bi]))):
                c = dict(depth=d + 1, split=False, G=cg, H=ch, C=cc)
                nd["right" if side else "left"] = len(grown)
                if not (c["depth"] >= hp.max_depth or cc < 2 * msl or ch < 2 * mcw):
                    (rs if side else ls)[a] = len(nxt)
                    nxt.append(len(grown))
                grown.append(c)
        new = np.full(n, -1, np.int64)
        for a in range(len(open_ids)):
            if feat[a] < 0:
                continue
            rows = np.nonzero(slot == a)[0]
            col = bins[feat[a], rows]
            right = (col != 255) & (col > thr[a])
            new[rows[right]] = rs[a]
            new[rows[~right]] = ls[a]
        slot, open_ids, d = new, nxt, d + 1
    out = dict(feature=[0], split_bin=[0], is_leaf=[True], left=[0], right=[0], value=[0.0])
    n_leaves, stack = 0, [(0, 0)]
    while stack:
        gi, fi = stack.pop()
        nd = grown[gi]
        if not nd["split"] or n_leaves >= 64:
            out["value"][fi] = np.float32(-nd["G"] / (nd["H"] + lam))
            n_leaves += 1
            continue
        li = len(out["value"])
        for k, v in (("feature", 0), ("split_bin", 0), ("is_leaf", True), ("left", 0), ("right", 0), ("value", 0.0)):
            out[k] += [v, v]
        out["feature"][fi], out["split_bin"][fi], out["is_leaf"][fi] = nd["feature"], nd["bin"], False
        out["left"][fi], out["right"][fi] = li, li + 1
        small_left = grown[nd["left"]]["C"] <= grown[nd["right"]]["C"]
        first, second = ((nd["left"], li), (nd["right"], li + 1)) if small_left else ((nd["right"], li + 1),
                                                                                       (nd["left"], li))
        stack += [second, first]
    return {k: np.array(v) for k, v in out.items()}


def build_leafwise_tree(b: Binned, g, h, hp: Hyper, fp32=True, max_leaves=64):
    """Tree::build_leafwise (src/tree/tree.cpp:685-907), the growth of the
    reference's regression preset (GrowPolicy::Lossguide,
    include/turbocat/config.hpp:266-274): the open leaf of the highest gain
    splits next (a max-heap of candidates; equal gains from different nodes
    do not occur in practice and are taken in insertion order here) until
    max_leaves leaves exist; a child is scored only when it can split
    (2 min_samples_leaf rows, 2 min_child_weight hessian) and one more leaf
    fits; the smaller child's histogram is built and the larger's is parent -
    smaller (built directly when the smaller cannot split).  fp32: the
    reference's arithmetic; else FP64.  Node arrays as build_regular_tree."""
    dt = np.float32 if fp32 else np.float64
    bins = b.bins
    n = bins.shape[1]
    nb = int(hp.max_bins)
    lam = dt(hp.lambda_l2)
    mcw2 = dt(2) * dt(hp.min_child_weight)
    msl2 = 2 * hp.min_samples_leaf
    keys = (("feature", 0), ("split_bin", 0), ("is_leaf", True), ("default_left", True), ("left", 0),
            ("right", 0), ("value", 0.0), ("gain", 0.0), ("margin", np.inf))
    nodes = {k: [v] for k, v in keys}
    leaf_of = np.zeros(n, np.int64)
    state = {"n_leaves": 0, "depth": 0, "seq": 0}

    def add_node():
        for k, v in keys:
            nodes[k].append(v)
        return len(nodes["value"]) - 1

    def make_leaf(i, st, r):
        v = dt(-st[0]) / dt(st[1] + lam)
        if hp.max_delta_step > 0:
            v = max(dt(-hp.max_delta_step), min(dt(hp.max_delta_step), v))
        nodes["is_leaf"][i] = True
        nodes["value"][i] = v
        leaf_of[r] = i
        state["n_leaves"] += 1

    rows = np.arange(n)
    root = (np.add.accumulate(np.asarray(g, dt), dtype=dt)[-1], np.add.accumulate(np.asarray(h, dt), dtype=dt)[-1], n)
    root_hist = _regular_hist(bins, rows, g, h, nb, dt)
    sp = _regular_scan(root_hist, root, hp, dt)
    if sp is None:
        make_leaf(0, root, rows)
        out = {k: np.array(v) for k, v in nodes.items()}
        out["value"] = out["value"].astype(np.float32)
        out["leaf_of"], out["depth"] = leaf_of, 0
        return out
    cands = [dict(node=0, split=sp, rows=rows, depth=0, stats=root, hist=root_hist, seq=0)]

    def pop_best():
        k = max(range(len(cands)), key=lambda j: (cands[j]["split"][0], -cands[j]["seq"]))
        return cands.pop(k)

    while cands and state["n_leaves"] < max_leaves:
        c = pop_best()
        i, (top, second, fi, bi, sl, sr), r, depth = c["node"], c["split"], c["rows"], c["depth"]
        if depth >= hp.max_depth:
            make_leaf(i, c["stats"], r)
            continue
        nodes["feature"][i], nodes["split_bin"][i] = fi, bi
        nodes["is_leaf"][i] = False
        nodes["gain"][i] = top
        nodes["margin"][i] = float((top - second) / abs(top)) if np.isfinite(second) and top != 0 else np.inf
        col = bins[fi, r]
        go_left = np.where(col == 255, True, col <= bi)
        rl, rr = r[go_left], r[~go_left]
        if len(rl) != len(r) and len(rr) != len(r):
            nodes["default_left"][i] = len(rl) >= len(rr)
        li = add_node()
        ri = add_node()
        nodes["left"][i], nodes["right"][i] = li, ri
        state["depth"] = max(state["depth"], depth + 1)
        left_small = len(rl) <= len(rr)
        lcan = len(rl) >= msl2 and sl[1] >= mcw2
        rcan = len(rr) >= msl2 and sr[1] >= mcw2
        hl = hr = None
        if lcan or rcan:
            if left_small:
                if lcan:
                    hl = _regular_hist(bins, rl, g, h, nb, dt)
                if rcan:
                    hr = (tuple((p - q).astype(p.dtype) for p, q in zip(c["hist"], hl)) if hl is not None
                          else _regular_hist(bins, rr, g, h, nb, dt))
            else:
                if rcan:
                    hr = _regular_hist(bins, rr, g, h, nb, dt)
                if lcan:
                    hl = (tuple((p - q).astype(p.dtype) for p, q in zip(c["hist"], hr)) if hr is not None
                          else _regular_hist(bins, rl, g, h, nb, dt))
        for node, can, hist, st, rr_ in ((li, lcan, hl, sl, rl), (ri, rcan, hr, sr, rr)):
            if can and state["n_leaves"] + 1 < max_leaves:
                csp = _regular_scan(hist, st, hp, dt)
                if csp is not None:
                    state["seq"] += 1
                    cands.append(dict(node=node, split=csp, rows=rr_, depth=depth + 1, stats=st, hist=hist,
                                      seq=state["seq"]))
                    continue
            make_leaf(node, st, rr_)
    while cands:
        c = pop_best()
        make_leaf(c["node"], c["stats"], c["rows"])
    out = {k: np.array(v) for k, v in nodes.items()}
    out["value"] = out["value"].astype(np.float32)
    out["leaf_of"], out["depth"] = leaf_of, state["depth"]
    return out


def fit_leafwise(b: Binned, y, hp: Hyper, fp32=True):
    """Booster::train with leaf-wise regular trees (the reference's MSE
    regression preset in mode="small"): base = mean label, per iteration the
    MSE gradients, one tree, predictions += lr * leaf (one FP32 rounding)."""
    y = np.asarray(y, np.float32)
    base = init_prediction(hp.loss, y)
    pred = np.full(len(y), base, np.float32)
    lr = np.float32(hp.learning_rate)
    trees = []
    for _ in range(hp.n_estimators):
        g, h = gradients(hp.loss, y, pred)
        t = build_leafwise_tree(b, g, h, hp, fp32=fp32)
        trees.append(t)
        leaf = t["value"].astype(np.float32)[t["leaf_of"]]
        pred = (pred.astype(np.longdouble) + np.longdouble(lr) * leaf.astype(np.longdouble)).astype(np.float32)
    return trees, pred, base


def fit_regular_multiclass(b: Binned, y, hp: Hyper, K: int, fp32=True):
    """Booster::train_multiclass (src/boosting/booster.cpp:1263-1395), the
    reference's multiclass loop in every mode: base predictions 0, per
    iteration the softmax gradients of all classes
    (CrossEntropyLoss::compute_multiclass_gradients), then one regular
    depth-wise tree per class on that class's gradient column, predictions
    [:, k] += lr * leaf (one FP32 rounding).  Trees iteration-major,
    class-minor, as the reference saves them."""
    y = np.asarray(y, np.float32)
    n = len(y)
    pred = np.zeros((n, K), np.float32)
    lr = np.longdouble(np.float32(hp.learning_rate))
    trees = []
    for _ in range(hp.n_estimators):
        g, h = gradients("softmax", y, pred.ravel(), K)
        g, h = g.reshape(n, K), h.reshape(n, K)
        for k in range(K):
            t = build_regular_tree(b, g[:, k].copy(), h[:, k].copy(), hp, fp32=fp32)
            trees.append(t)
            leaf = t["value"].astype(np.float32)[t["leaf_of"]]
            pred[:, k] = (pred[:, k].astype(np.longdouble) + lr * leaf.astype(np.longdouble)).astype(np.float32)
    return trees, pred
