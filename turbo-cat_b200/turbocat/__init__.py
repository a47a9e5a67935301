"""TurboCat symmetric-tree path on NVIDIA B200.

Drop-in for the reference package's facade (python/turbocat/__init__.py:290-875):
the same classes, constructor arguments and defaults, and the same
fit / predict / predict_proba / save / load surface, backed by the pybind11
module `_turbocat` (csrc/bindings.cpp), which calls the device engine
(libtcgpu.so, include/tcgpu.h).  Every call runs on the GPU; there is no CPU
fallback.

Put the directory that holds this package on sys.path and `import turbocat`.
"""
from __future__ import annotations

import numpy as np

__version__ = "0.4.2+b200"

from ._turbocat import (  # noqa: E402  (fails loudly when the extension is not built)
    TurboCatClassifier as _TurboCatClassifier,
    TurboCatRegressor as _TurboCatRegressor,
    print_info,
)


def _f32(X):
    # the reference forces C-contiguous float32 (python/turbocat/__init__.py:441-446)
    return np.ascontiguousarray(np.asarray(X, dtype=np.float32))


class TurboCatClassifier:
    """Gradient-boosted symmetric (oblivious) trees, binary or multiclass.

    Same constructor signature and defaults as the reference facade
    (python/turbocat/__init__.py:340-363).  Binary tasks use logloss or focal
    loss; labels with more than two classes train one symmetric tree per
    class and iteration on softmax gradients.
    """

    def __init__(self, n_estimators=1000, learning_rate=0.1, max_depth=6, max_bins=255, subsample=0.8,
                 colsample_bytree=0.8, min_child_weight=1.0, lambda_l2=1.0, loss="logloss", mode="auto",
                 use_goss=False, goss_top_rate=0.2, goss_other_rate=0.1, use_gradtree=False, use_symmetric=False,
                 use_ordered_boosting=False, early_stopping_rounds=50, n_jobs=-1, n_threads=None, seed=42,
                 verbosity=1):
        threads = n_threads if n_threads is not None else n_jobs
        if use_symmetric and mode == "auto":
            mode = "large"
        self._model = _TurboCatClassifier(
            n_estimators=n_estimators, learning_rate=learning_rate, max_depth=max_depth, max_bins=max_bins,
            subsample=subsample, colsample_bytree=colsample_bytree, min_child_weight=min_child_weight,
            lambda_l2=lambda_l2, loss=loss, mode=mode, use_goss=use_goss, goss_top_rate=goss_top_rate,
            goss_other_rate=goss_other_rate, use_gradtree=use_gradtree,
            use_ordered_boosting=use_ordered_boosting, early_stopping_rounds=early_stopping_rounds,
            n_threads=threads, seed=seed, verbosity=verbosity)
        self._params = dict(n_estimators=n_estimators, learning_rate=learning_rate, max_depth=max_depth,
                            max_bins=max_bins, subsample=subsample, colsample_bytree=colsample_bytree,
                            min_child_weight=min_child_weight, lambda_l2=lambda_l2, loss=loss, mode=mode,
                            use_goss=use_goss, goss_top_rate=goss_top_rate, goss_other_rate=goss_other_rate,
                            use_gradtree=use_gradtree, use_ordered_boosting=use_ordered_boosting,
                            early_stopping_rounds=early_stopping_rounds, n_jobs=n_jobs, seed=seed,
                            verbosity=verbosity)

    def fit(self, X, y, X_val=None, y_val=None, cat_features=None):
        X = _f32(X)
        y = _f32(y)
        if X_val is not None:
            X_val, y_val = _f32(X_val), _f32(y_val)
        else:
            X_val = np.zeros((0, X.shape[1] if X.ndim > 1 else 0), np.float32)
            y_val = np.zeros(0, np.float32)
        self._model.fit(X, y, X_val, y_val, list(cat_features or []))
        return self

    def predict_proba(self, X):
        return np.asarray(self._model.predict_proba(_f32(X)), dtype=np.float32)

    def predict_proba_nobinning_fast(self, X):
        return np.asarray(self._model.predict_proba_nobinning_fast(_f32(X)), dtype=np.float32)

    def predict(self, X, threshold=0.5):
        proba = self.predict_proba(X)
        if proba.shape[1] == 2:
            return (proba[:, 1] >= threshold).astype(np.int32)
        return np.argmax(proba, axis=1).astype(np.int32)

    def feature_importance(self):
        return self._model.feature_importance()

    def save(self, path):
        self._model.save(path)

    def load(self, path):
        self._model.load(path)
        return self

    def get_params(self, deep=True):
        return dict(self._params)

    def set_params(self, **params):
        self._params.update(params)
        return self

    @property
    def n_trees(self):
        return self._model.n_trees

    @property
    def n_classes_(self):
        return self._model.n_classes_

    @property
    def train_seconds(self):
        """Device seconds of the boosting iterations of the last fit."""
        return self._model.train_seconds


class TurboCatRegressor:
    """Gradient-boosted symmetric trees for regression (MSE).

    Same constructor signature and defaults as the reference facade
    (python/turbocat/__init__.py:628-646), including lambda_l2=0.0.
    """

    def __init__(self, n_estimators=1000, learning_rate=0.1, max_depth=6, loss="mse", mode="auto", subsample=0.8,
                 colsample_bytree=0.8, use_goss=False, goss_top_rate=0.2, goss_other_rate=0.1,
                 early_stopping_rounds=50, lambda_l2=0.0, n_jobs=-1, n_threads=None, seed=42, verbosity=1):
        threads = n_threads if n_threads is not None else n_jobs
        self._model = _TurboCatRegressor(
            n_estimators=n_estimators, learning_rate=learning_rate, max_depth=max_depth, loss=loss, mode=mode,
            subsample=subsample, colsample_bytree=colsample_bytree, use_goss=use_goss, goss_top_rate=goss_top_rate,
            goss_other_rate=goss_other_rate, early_stopping_rounds=early_stopping_rounds, lambda_l2=lambda_l2,
            n_threads=threads, seed=seed, verbosity=verbosity)
        self._params = dict(n_estimators=n_estimators, learning_rate=learning_rate, max_depth=max_depth, loss=loss,
                            mode=mode, subsample=subsample, colsample_bytree=colsample_bytree, use_goss=use_goss,
                            lambda_l2=lambda_l2, n_jobs=n_jobs, seed=seed, verbosity=verbosity)

    def fit(self, X, y):
        self._model.fit(_f32(X), _f32(y))
        return self

    def predict(self, X, timing=False):
        return np.asarray(self._model.predict(_f32(X), timing), dtype=np.float32)

    def predict_fast(self, X, timing=False):
        return np.asarray(self._model.predict_fast(_f32(X), timing), dtype=np.float32)

    def predict_nobinning(self, X, timing=False):
        return np.asarray(self._model.predict_nobinning(_f32(X), timing), dtype=np.float32)

    def predict_nobinning_fast(self, X, timing=False):
        return np.asarray(self._model.predict_nobinning_fast(_f32(X), timing), dtype=np.float32)

    def debug_info(self):
        info = self._model.debug_info()
        info["params"] = self._params
        return info

    def tree_info(self):
        """Per tree: node and leaf counts, leaf sum, single-leaf flag."""
        return self._model.tree_info()

    def debug_predict(self, X):
        """Bins of the first rows under the training edges, the first tree's
        path for the first samples, and train/test value ranges."""
        return self._model.debug_predict(_f32(X))

    @property
    def n_trees(self):
        return self._model.n_trees

    @property
    def base_prediction_(self):
        return self._model.base_prediction

    @property
    def train_seconds(self):
        return self._model.train_seconds

    def feature_importance(self):
        return self._model.feature_importance()

    def get_params(self, deep=True):
        return dict(self._params)

    def set_params(self, **params):
        self._params.update(params)
        return self

    def save(self, path):
        self._model.save(path)

    def load(self, path):
        self._model.load(path)
        return self


__all__ = ["TurboCatClassifier", "TurboCatRegressor", "print_info", "__version__"]
