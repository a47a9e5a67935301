"""Prints the pybind11 surface of a `_turbocat` extension module as JSON:
class constructor and method signatures (names, argument names, defaults)
and the `metrics` submodule.  Used by test_surface.py on the reference's
module (oracle/_ref) and on this package's."""
import importlib.util
import json
import re
import sys


def sig_lines(doc):
    if not doc:
        return []
    out = []
    for line in doc.splitlines():
        line = line.strip()
        m = re.match(r"^(?:\d+\.\s*)?(\w+)\((.*)\)(?:\s*->\s*(.*))?$", line)
        if m:
            args = re.sub(r"\b_turbocat\.", "", m.group(2))
            args = re.sub(r"self: [\w.]+,?\s*", "", args)
            out.append(f"{m.group(1)}({args})")
    return out


def main(path):
    spec = importlib.util.spec_from_file_location("_turbocat", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for cls in ("TurboCatClassifier", "TurboCatRegressor"):
        C = getattr(mod, cls)
        members = {}
        for name in dir(C):
            if name.startswith("_") and name != "__init__":
                continue
            attr = getattr(C, name)
            members[name] = sig_lines(getattr(attr, "__doc__", None)) if callable(attr) else "property"
        out[cls] = members
    met = {}
    for name in dir(mod.metrics):
        if name.startswith("_"):
            continue
        attr = getattr(mod.metrics, name)
        met[name] = sig_lines(getattr(attr, "__doc__", None)) if callable(attr) and not isinstance(attr, type) \
            else type(attr).__name__
    out["metrics"] = met
    print(json.dumps(out))




def metric_values(path):
    """Values of the metrics submodule's functions on fixed seeded inputs."""
    import numpy as np

    spec = importlib.util.spec_from_file_location("_turbocat", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rng = np.random.default_rng(5)
    yt = (rng.random(1001) < 0.3).astype(np.float32)
    yp = rng.random(1001).astype(np.float32)
    yp[:3] = [0.0, 1.0, 0.5]
    M = mod.metrics
    out = {"log_loss": M.log_loss(yt, yp), "log_loss_eps": M.log_loss(yt, yp, 1e-3),
           "mse": M.mse(yt, yp), "mae": M.mae(yt, yp), "rmse": M.rmse(yt, yp)}
    for thr in (0.5, 0.2, 0.97):
        for fn in ("accuracy", "precision", "recall", "f1_score"):
            out[f"{fn}@{thr}"] = getattr(M, fn)(yt, yp, thr)
    out["empty_precision"] = M.precision(np.zeros(4, np.float32), np.zeros(4, np.float32))
    print(json.dumps(out))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "metrics":
        metric_values(sys.argv[1])
    else:
        main(sys.argv[1])
