"""Host-side checks that need no GPU: the C ABI library loads, exports every
symbol include/tcgpu.h declares, and fails cleanly without a device."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "tcgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_list_agree(capi):
    assert _declared() == sorted(capi.SYMBOLS)


def test_library_exports_every_declared_symbol(capi):
    lib = capi.lib()
    missing = [s for s in _declared() if not hasattr(lib, s)]
    assert not missing, missing


def test_context_creation_fails_cleanly_without_device(capi):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    st = capi.lib().tc_ctx_create(0, 0, C.byref(ctx))
    assert st != 0 and not ctx.value


def test_null_arguments_are_rejected(capi):
    lib = capi.lib()
    assert lib.tc_ctx_create(0, 0, None) == 1
    assert lib.tc_quantize(None, 255, 1, None, None) == 1
    assert lib.tc_trainer_step(None, 1, 1) == 1
    assert lib.tc_predict(None, None, None, 0, 1, 0, None) == 1
    assert lib.tc_server_poll(None, 1, 0, None, None) == 1
    assert lib.tc_last_error(None) is not None


def test_facade_surface_without_device():
    import inspect

    import turbocat

    sig = inspect.signature(turbocat.TurboCatClassifier.__init__)
    d = {k: v.default for k, v in sig.parameters.items() if k != "self"}
    # reference facade defaults, python/turbocat/__init__.py:340-363
    assert d["n_estimators"] == 1000 and d["learning_rate"] == 0.1 and d["subsample"] == 0.8
    assert d["colsample_bytree"] == 0.8 and d["loss"] == "logloss" and d["mode"] == "auto"
    r = inspect.signature(turbocat.TurboCatRegressor.__init__)
    assert r.parameters["lambda_l2"].default == 0.0
    clf = turbocat.TurboCatClassifier(n_estimators=3, verbosity=0)
    with pytest.raises(RuntimeError, match="not fitted"):
        clf.predict_proba([[0.0, 1.0]])
