"""The pybind11 module's surface against the reference's own module (built
from its sources in oracle/_ref), on CPU: every class member and `metrics`
function the reference binds exists here with the same argument names and
defaults (python/bindings.cpp:1045-1131, 1139-1224).  Each module is
introspected in its own interpreter (both are named `_turbocat`)."""
import glob
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _surface(pattern, what=None):
    paths = glob.glob(os.path.join(ROOT, pattern))
    if not paths:
        return None
    cmd = [sys.executable, os.path.join(ROOT, "tests", "surface_dump.py"), paths[0]] + ([what] if what else [])
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    return json.loads(out)


@pytest.mark.skipif(not glob.glob(os.path.join(ROOT, "oracle", "_ref", "_turbocat*.so")),
                    reason="reference build oracle/_ref not present")
def test_surface_matches_reference_module():
    ref = _surface("oracle/_ref/_turbocat*.so")
    ours = _surface("turbo-cat_b200/turbocat/_turbocat*.so")
    assert ours is not None
    for section, members in ref.items():
        for name, sig in members.items():
            assert name in ours[section], f"{section}.{name} missing"
            assert ours[section][name] == sig, (section, name, ours[section][name], sig)


@pytest.mark.skipif(not glob.glob(os.path.join(ROOT, "oracle", "_ref", "_turbocat*.so")),
                    reason="reference build oracle/_ref not present")
def test_metrics_equal_reference_values():
    """The metric functions whose formulas the reference defines
    (include/turbocat/metrics.hpp:363-470) give the reference module's values
    bit for bit (FP32 sums in row order)."""
    ref = _surface("oracle/_ref/_turbocat*.so", "metrics")
    ours = _surface("turbo-cat_b200/turbocat/_turbocat*.so", "metrics")
    assert ours == ref


def test_metrics_without_source_raise():
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "turbo-cat_b200"))
    from turbocat import _turbocat as T

    y = np.ones(4, np.float32)
    for fn in (T.metrics.roc_auc, T.metrics.pr_auc):
        with pytest.raises(RuntimeError, match="unavailable"):
            fn(y, y)
    with pytest.raises(RuntimeError, match="unavailable"):
        T.metrics.find_optimal_threshold(y, y, T.metrics.MetricType.F1, 10)
