"""Benchmark: symmetric-tree training on the imbalanced focal-loss configuration.

Workload (seeded synthetic data with the configuration's shapes and value
distributions; no public dataset is involved): 10,000,000 rows x 200 float32
features -- 100 N(0,1), 100 LogNormal(0,1) -- with about 1% positives from
thresholding a sparse linear score (20 active features) plus N(0, 0.5);
focal loss (gamma 2, alpha 0.25), 1000 symmetric trees, depth 8, learning
rate 0.1, 255 bins, lambda_l2 1.  This is the largest configuration that fits
one GPU.

Metric: training seconds per 100 trees (lower is better).  A step is 100
boosting iterations of the configuration's 1000-tree fit; the fit restarts
from the base prediction after every 10 steps (untimed), so no step trains a
tree beyond the configuration.  `value` times the steps on device-resident
data (CUDA events on the engine's stream, a 256 MiB L2 flush between steps;
the 2 GB of bins are larger than L2 anyway).  `e2e` times whole fits through
the public API (turbocat.TurboCatClassifier.fit) from pinned host memory:
upload, device binning, 1000 trees, model download.  The line also carries
the regression configuration (1M x 100, MSE, 500 trees, depth 8) as a
secondary object, device-timed the same way.

--impl reference runs the reference's own CPU implementation (its sources
compiled in oracle/_ref) on the same data on all host cores: Booster::train
with the configuration's 1000 trees, stopped through its training callback
after warm-up + timed trees; the full fit is extrapolated from the measured
set-up and per-tree times (stated in the line).

Multi-GPU: replicas only (one independent fit per rank, no collective on the
data path); value aggregates over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "turbo-cat_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

N_ROWS, N_FEAT, DEPTH, LR, TREES, L2 = 10_000_000, 200, 8, 0.1, 1000, 1.0
TREES_PER_STEP = 100
STEPS_PER_FIT = TREES // TREES_PER_STEP
METRIC = "train_s_per_100_trees"
UNIT = "s/100 trees"
CONFIG = {"workload": "imbalanced classification 10M x 200 float32 (100 N(0,1), 100 LogNormal(0,1), ~1% positives), "
                      "focal loss (gamma 2, alpha 0.25), 1000 symmetric trees, depth 8, lr 0.1, 255 bins, "
                      "lambda_l2 1",
          "rows": N_ROWS, "features": N_FEAT, "trees": TREES, "depth": DEPTH, "bins": 255,
          "step": "100 boosting iterations of the 1000-tree fit (restarted from the base prediction every 10 steps)",
          "l2": "inputs larger than L2 (2 GB of bins) plus a 256 MiB flush between timed steps"}
C2 = dict(n=1_000_000, f=100, depth=8, lr=0.05, trees=500, l2=0.0)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic_ratio(name):
    """DRAM bytes over algorithmic bytes of the histogram kernel, recorded from
    an ncu capture in a committed profile summary (a profile constant, not
    measured in this run)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("dram_over_algorithmic:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi clock sampling during the timed region."""

    def __init__(self, gpu):
        # raw samples: $BENCH_CLOCKS_DIR if set (kept as evidence), else the temp directory
        out = os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"bench_clocks_{gpu}_{os.getpid()}.csv")
        os.makedirs(out, exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(loaded)) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def dist_max(x, ws, device=None):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device=device) if device is not None else torch.tensor([float(x)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def make_data():
    from datagen import imbalanced_c5

    return imbalanced_c5(N_ROWS, N_FEAT, seed=5)


def ref_hyper(n_estimators=TREES):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    return O, O.Hyper(loss="focal", n_estimators=n_estimators, learning_rate=LR, max_depth=DEPTH, lambda_l2=L2,
                      min_child_weight=1.0, focal_gamma=2.0, focal_alpha=0.25)


def reference_timed(X, y, warm_trees, timed_trees, max_seconds):
    """The reference's own Booster::train (oracle/_ref, its sources compiled
    with its own flags) on X, y with the configuration's 1000 trees, stopped
    after warm_trees + timed_trees trees (or max_seconds).  Returns
    (full-fit seconds extrapolated to 1000 trees, detail)."""
    O, hp = ref_hyper()
    setup, ends = O.ref_fit_timed(X, y, hp, warm_trees + timed_trees, max_seconds)
    built = len(ends)
    w = min(warm_trees, max(0, built - 2))
    per_tree = (ends[-1] - ends[w - 1]) / (built - w) if w >= 1 else (ends[-1] - setup) / max(1, built)
    full = ends[-1] + (TREES - built) * per_tree
    steps_ms = [1e3 * (ends[i] - (ends[i - 1] if i else setup)) for i in range(w, built)]
    return full, {"setup_s": setup, "first_tree_end_s": ends[0], "last_tree_end_s": ends[-1],
                  "trees_built": built, "trees_timed": built - w,
                  "per_tree_s": per_tree, "tree_ms": steps_ms,
                  "extrapolation": "full fit = end of the last built tree + (1000 - built) x mean per-tree time "
                                   "of the timed trees"}


def run_reference(args):
    # rank 0 alone measures the host CPU; other ranks exit without work
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libtcref.so")):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
        return
    t0 = time.perf_counter()
    X, y = make_data()
    log(f"reference arm: data in {time.perf_counter() - t0:.1f} s")
    cores = os.cpu_count()
    full, detail = reference_timed(X, y, args.warmup, args.steps, args.reference_seconds)
    value = full / STEPS_PER_FIT
    detail["timed_region_s"] = float(np.sum(detail["tree_ms"]) / 1e3)
    cfg = dict(CONFIG, step="one boosting iteration (tree) of the reference's 1000-tree fit; value is the "
                            "extrapolated full fit (binning included) per 100 trees")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": detail["trees_timed"],
            "warmup": detail["trees_built"] - detail["trees_timed"],
            "ms_per_step": detail["per_tree_s"] * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"reference Booster::train on the full 10M x 200 data, stopped after "
                                       f"{detail['trees_built']} of 1000 trees ({detail['trees_timed']} timed); "
                                       "set-up + per-tree time extrapolated to the 1000-tree fit",
                             "detail": detail},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def windowed_profile(tr, total_trees, windows=4, per=3):
    """In-graph kernel profile of `per` iterations at `windows` points spread
    over a fit of `total_trees` iterations (a tree's cost changes along the
    fit), summed; the fit restarts from the base prediction first."""
    tr.reset()
    out = None
    for w in range(windows):
        start = w * total_trees // windows
        done = tr.stats().iterations_done
        if start > done:
            tr.step(start - done)
        prof = tr.profile(per)
        if out is None:
            out = prof
            continue
        for k, v in prof.items():
            if k in ("_hist_levels", "_part_levels", "_in_graph"):
                continue
            if k == "_iteration_ms":
                out[k] += v
            else:
                out[k] = tuple(a + b for a, b in zip(out[k], v))
        out["_in_graph"] = out["_in_graph"] and prof["_in_graph"]
    out["_iters"] = windows * per
    out["_windows"] = [w * total_trees // windows for w in range(windows)]
    return out


def hist_roofline(prof, peak, peak_kind, traffic_file):
    """Roofline of the histogram kernel from an in-graph profile."""
    hl, hms, hbytes = prof["hist"]
    achieved = hbytes / (hms * 1e-3) / 1e9 if hms > 0 else None
    kern = {k: v for k, v in prof.items() if not k.startswith("_")}
    dominant = max((v[1], k) for k, v in kern.items())[1]
    iters = max(1, prof.get("_iters", 3))
    ratio = profile_traffic_ratio(traffic_file)
    return {"kernel": "k_hist (histogram)", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
            "traffic": ratio * hbytes / max(1, hl) if ratio else None,
            "traffic_source": f"per launch: algorithmic bytes x the DRAM/algorithmic ratio {ratio} of an ncu "
                              f"capture of a smaller case (profiles/{traffic_file}); a profile constant",
            "alg_bytes_per_launch": hbytes / max(1, hl), "avg_launch_ms": hms / max(1, hl),
            "timing": "CUDA events recorded as nodes of the replayed iteration graph" if prof["_in_graph"]
                      else "CUDA events around launches outside a graph",
            "dominant_kernel_by_time": dominant,
            "kernel_ms_per_iter": {k: round(v[1] / iters, 4) for k, v in kern.items() if v[0]},
            "kernels_sum_ms_per_iter": sum(v[1] for v in kern.values()) / iters,
            "profiled_iteration_ms": prof["_iteration_ms"] / iters,
            "profiled_iterations": f"{prof.get('_iters')} iterations in windows starting at "
                                   f"{prof.get('_windows')} of the fit"}


def c2_secondary(eng, _capi, peak, peak_kind, steps):
    """The regression configuration, device-timed like the headline."""
    import torch

    from datagen import regression_c2

    X, y = regression_c2(C2["n"], C2["f"], seed=2)
    ds = eng.upload(X, y)
    ds.quantize(255)
    p = _capi.params(loss="mse", n_estimators=C2["trees"], max_depth=C2["depth"], learning_rate=C2["lr"],
                     lambda_l2=C2["l2"], max_bins=255)
    tr = eng.trainer(ds, p)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    per_fit = C2["trees"] // TREES_PER_STEP
    for _ in range(3):
        tr.step(TREES_PER_STEP)
    tr.reset()
    step_s = []
    for i in range(steps):
        if i and i % per_fit == 0:
            tr.reset()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        s0 = tr.stats().seconds
        tr.step(TREES_PER_STEP)
        step_s.append(tr.stats().seconds - s0)
    prof = windowed_profile(tr, C2["trees"])
    out = {"workload": "regression 1M x 100 float32 (60 N(0,1), 30 U(-3,3), 10 t(3)), MSE, 500 symmetric trees, "
                       "depth 8, lr 0.05, 255 bins, lambda_l2 0",
           "value": float(np.mean(step_s)), "unit": UNIT, "steps": steps,
           "roofline": hist_roofline(prof, peak, peak_kind, "k_hist_c2_regression.md")}
    tr.close()
    ds.close()
    return out


def run_ours(args):
    ws, rank, local = dist_setup("nccl")
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    os.environ["TURBOCAT_DEVICE"] = str(local)
    from turbocat import _capi

    eng = _capi.Engine(local)
    t0 = time.perf_counter()
    X, y = make_data()
    log(f"data in {time.perf_counter() - t0:.1f} s")
    ds = eng.upload(X, y)
    ds.quantize(255)
    p = _capi.params(loss="focal", n_estimators=TREES, max_depth=DEPTH, learning_rate=LR, lambda_l2=L2,
                     max_bins=255, focal_gamma=2.0, focal_alpha=0.25)
    tr = eng.trainer(ds, p)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2

    def next_step(timed):
        if tr.stats().iterations_done >= TREES:
            tr.reset()  # the fit restarts: a step never trains a tree beyond the configuration
        if not timed:
            tr.step(TREES_PER_STEP)
            return 0.0
        flush.fill_(1.0)
        torch.cuda.synchronize()
        s0 = tr.stats().seconds
        tr.step(TREES_PER_STEP)  # synchronises; seconds from CUDA events on the engine stream
        return tr.stats().seconds - s0

    for _ in range(args.warmup):
        next_step(False)
    tr.reset()
    torch.cuda.synchronize()
    dist_barrier(ws)
    clocks = Clocks(local)
    launches0 = tr.stats().kernel_launches
    step_s = [next_step(True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = tr.stats().kernel_launches - launches0
    dist_barrier(ws)
    total = dist_max(sum(step_s), ws, dev)
    # whole job: ws replicas x steps x 100 trees in `total` seconds
    value = total / (args.steps * ws)

    # roofline of the dominant kernel (histogram), timed inside the iteration graph
    peak, peak_kind = load_peaks()
    prof = windowed_profile(tr, TREES)
    roofline = hist_roofline(prof, peak, peak_kind, "k_hist_c5_focal.md")
    tr.close()

    # end to end through the public API, pinned host inputs
    import turbocat

    Xp = torch.empty((N_ROWS, N_FEAT), dtype=torch.float32, pin_memory=True).numpy()
    yp = torch.empty(N_ROWS, dtype=torch.float32, pin_memory=True).numpy()
    Xp[:] = X
    yp[:] = y
    ds.close()
    e2e_s = []
    for i in range(1 + args.e2e_fits):
        m = turbocat.TurboCatClassifier(n_estimators=TREES, learning_rate=LR, max_depth=DEPTH, loss="focal",
                                        mode="large", subsample=1.0, colsample_bytree=1.0, lambda_l2=L2,
                                        min_child_weight=1.0, verbosity=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m.fit(Xp, yp)
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_s.append(dt)
        del m
    e2e_fit = dist_max(float(np.median(e2e_s)), ws, dev) if e2e_s else None
    model_bytes = TREES * (DEPTH * 11 + (1 << DEPTH) * 4 + 8)
    e2e = {"value": e2e_fit / STEPS_PER_FIT / ws if e2e_fit else None, "unit": UNIT,
           "h2d_bytes_per_step": int((X.nbytes + y.nbytes) / STEPS_PER_FIT),
           "d2h_bytes_per_step": int(model_bytes / STEPS_PER_FIT),
           "fit_seconds": e2e_fit, "fits_timed": args.e2e_fits, "fit_seconds_each": e2e_s,
           "path": "turbocat.TurboCatClassifier.fit (pybind -> C ABI): upload, device binning, 1000 trees, model"}
    del Xp, yp

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            sub = 1_000_000
            full_sub, detail = reference_timed(np.ascontiguousarray(X[:sub]), np.ascontiguousarray(y[:sub]), 2, 6,
                                               60.0)
            scale = N_ROWS / sub
            # per-tree work scales with the rows; binning sorts (n log n)
            setup_full = detail["setup_s"] * scale * np.log(N_ROWS) / np.log(sub)
            fit_full = setup_full + (detail["first_tree_end_s"] - detail["setup_s"]) * scale + \
                (TREES - 1) * detail["per_tree_s"] * scale
            cpu = {"value": fit_full / STEPS_PER_FIT, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": "reference Booster::train on the first 1M of the 10M rows (all 200 features), "
                             f"{detail['trees_built']} trees built, {detail['trees_timed']} timed; per-tree time "
                             "scaled by 10 (rows), binning by 10 x log(10M)/log(1M), extrapolated to 1000 trees",
                   "detail": detail}
        except Exception as e:  # reference build absent
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    secondary = None
    if rank == 0 and ws == 1 and not args.no_c2:
        secondary = c2_secondary(eng, _capi, peak, peak_kind, steps=5)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": CONFIG,
                "parallelism": f"replicas x{ws}", "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clk, "gpu_launches": int(launches),
                "trees_per_s": args.steps * TREES_PER_STEP * ws / total,
                "secondary": {"c2_regression": secondary} if secondary else None}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------- suite --
# Secondary configurations (not the headline line): run with --suite; writes
# one JSON object per configuration to stdout.

def _pct(a, q):
    return float(np.percentile(np.asarray(a), q)) if len(a) else None


def suite_c1(eng, _capi, ref_ok):
    from datagen import binary_c1

    X, y = binary_c1()
    ds = eng.upload(X, y)
    ds.quantize(255)
    tr = eng.trainer(ds, _capi.params(loss="logloss", n_estimators=400, max_depth=6, learning_rate=0.1))
    tr.step(100)
    tr.reset()
    s0 = tr.stats().seconds
    tr.step(100)
    dev = tr.stats().seconds - s0
    out = {"config": "binary 50k x 20, logloss, 100 trees, depth 6", "device_s_per_100_trees": dev}
    prof = tr.profile(5)
    out["kernel_ms_per_iteration"] = {k: [v[0] / 5, v[1] / 5] for k, v in prof.items() if not k.startswith("_")}
    out["profiled_iteration_ms"] = prof["_iteration_ms"]
    if ref_ok:
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import _turbocat as ref

        m = ref.TurboCatClassifier(n_estimators=100, learning_rate=0.1, max_depth=6, max_bins=255, subsample=1.0,
                                   colsample_bytree=1.0, min_child_weight=1.0, lambda_l2=1.0, loss="logloss",
                                   mode="large", verbosity=0)
        t0 = time.perf_counter()
        m.fit(X, y)
        out["reference_cpu_fit_s"] = time.perf_counter() - t0
        out["reference_cores"] = os.cpu_count()
    return out


def suite_regular(eng, _capi, ref_ok):
    """Regular (depth-wise) trees, the reference's mode="small": binary
    50k x 20, logloss, depth 6, 100 trees, every row.  Device: tc_train_regular
    (one-shot, wall time of the call); reference: its own Booster::train with
    regular trees on the same data (timed trees through its callback)."""
    from datagen import binary_c1

    X, y = binary_c1()
    ds = eng.upload(X, y)
    ds.quantize(255)
    prm = _capi.params(loss="logloss", n_estimators=100, max_depth=6, learning_rate=0.1)
    eng.train_regular(ds, _capi.params(loss="logloss", n_estimators=2, max_depth=6))[0].close()  # warm-up
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        m, st = eng.train_regular(ds, prm)
        dt = time.perf_counter() - t0
        m.close()
        best = dt if best is None else min(best, dt)
    out = {"config": "regular trees, binary 50k x 20, logloss, depth 6, 100 trees", "device_s_per_100_trees": best,
           "kernel_launches_per_fit": st.kernel_launches}
    if ref_ok:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        hp = O.Hyper(loss="logloss", n_estimators=100, max_depth=6, learning_rate=0.1, regular_trees=True)
        setup, ends = O.ref_fit_timed(X, y, hp, 100, 60.0)
        out["reference_cpu_s_per_100_trees"] = (ends[-1] - ends[0]) * 100.0 / max(1, len(ends) - 1) if len(ends) > 1 else None
        out["reference_trees_timed"] = len(ends)
        out["reference_threads"] = os.cpu_count()
    ds.close()
    return out


def suite_cat(eng, _capi, ref_ok):
    return {"cardinality_1000": _cat_case(eng, ref_ok, cardinality=1000),
            "cardinality_8": _cat_case(eng, ref_ok, cardinality=8)}


def _cat_case(eng, ref_ok, n=10_000_000, f=20, n_cat=4, cardinality=1000):
    """Categorical target statistics at scale: n rows, n_cat categorical
    columns of `cardinality` ids (3% NaN) among f, class-id labels.  Device:
    tc_encode_categorical (ordered and cross-validated; host-synchronous
    calls, wall time) and the binning after it; reference: its own
    compute_target_statistics on a 1M-row slice, scaled to n."""
    rng = np.random.default_rng(17)
    X = rng.standard_normal((n, f), dtype=np.float32)
    cats = list(range(1, 2 * n_cat, 2))
    logit = X[:, 0].copy()
    for j in cats:
        c = rng.integers(0, cardinality, n)
        X[:, j] = c
        logit += ((c % 7) - 3) * 0.3
        X[rng.random(n, dtype=np.float32) < 0.03, j] = np.nan
    y = (rng.random(n, dtype=np.float32) < 1.0 / (1.0 + np.exp(-logit))).astype(np.float32)
    out = {"config": f"categorical target statistics, {n} rows x {f} features, {n_cat} categorical "
                     f"({cardinality} ids, 3% NaN)"}
    for method in ("ordered", "cv"):
        best = None
        for _ in range(3):
            ds = eng.upload(X, y)
            t0 = time.perf_counter()
            ds.encode_categorical(cats, method, seed=1)
            t1 = time.perf_counter()
            ds.quantize(255)
            t2 = time.perf_counter()
            ds.close()
            best = min(best or (9e9, 9e9), (t1 - t0, t2 - t1))
        out[f"{method}_encode_ms"] = best[0] * 1e3
        out[f"{method}_rows_x_columns_per_s"] = n * n_cat / best[0]
        out[f"{method}_quantize_after_ms"] = best[1] * 1e3
    if ref_ok:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ctypes as C

        import oracle as O

        m = 1_000_000
        Xs, ys = np.ascontiguousarray(X[:m]), np.ascontiguousarray(y[:m])
        cs = np.array(cats, np.uint16)
        for method, mid in (("ordered", 0), ("cv", 1)):
            sec = C.c_double()
            rc = O.ref().tcref_cat_ts_timed(Xs.ctypes.data_as(C.c_void_p), C.c_uint32(m), C.c_uint16(f),
                                            ys.ctypes.data_as(C.c_void_p), cs.ctypes.data_as(C.c_void_p),
                                            C.c_int32(len(cats)), C.c_int32(mid), C.byref(sec))
            if rc == 0:
                out[f"reference_{method}_ms_1M_rows"] = sec.value * 1e3
                out[f"reference_{method}_ms_scaled_to_n"] = sec.value * 1e3 * n / m
        out["reference_threads"] = 1  # compute_target_statistics runs on one thread
    return out


def suite_c3(eng, _capi, iters=10):
    from datagen import multiclass_c3

    X, y = multiclass_c3()
    ds = eng.upload(X, y)
    ds.quantize(255)
    res = {"config": "multiclass 2M x 50, K=10 softmax, depth 6 (200 iterations x 10 trees in the config)"}
    for batched in (1, 0):
        tr = eng.trainer(ds, _capi.params(loss="softmax", n_classes=10, n_estimators=iters + 3, max_depth=6,
                                          learning_rate=0.1, batched=batched))
        tr.step(2)
        s0 = tr.stats().seconds
        tr.step(iters)
        dt = (tr.stats().seconds - s0) / iters
        res["batched_s_per_iter" if batched else "plain_s_per_iter"] = dt
        tr.close()
    res["batched_speedup_vs_plain"] = res["plain_s_per_iter"] / res["batched_s_per_iter"]
    res["batched_s_per_100_trees"] = res["batched_s_per_iter"] * 10
    return res


def suite_goss(eng, _capi, iters=10):
    """GOSS on the regression configuration's data (1M x 100, MSE, depth 8,
    top 0.2, other 0.1): wall time per iteration (the host ranks the
    iteration's gradients and draws the sample; the device waits) against
    the device kernel time of such iterations."""
    from datagen import regression_c2

    X, y = regression_c2(C2["n"], C2["f"], seed=2)
    ds = eng.upload(X, y)
    ds.quantize(255)
    p = _capi.params(loss="mse", n_estimators=3 + iters + 5, max_depth=C2["depth"], learning_rate=C2["lr"],
                     lambda_l2=C2["l2"], use_goss=True, goss_top_rate=0.2, goss_other_rate=0.1)
    tr = eng.trainer(ds, p)
    tr.step(3)
    t0 = time.perf_counter()
    tr.step(iters)
    wall = (time.perf_counter() - t0) / iters
    prof = tr.profile(5)
    dev = sum(v[1] for k, v in prof.items() if not k.startswith("_")) / 5 * 1e-3
    return {"config": "GOSS (top 0.2, other 0.1) on regression 1M x 100, MSE, depth 8",
            "wall_s_per_iter": wall, "device_kernel_s_per_iter": dev,
            "host_selection_and_sync_s_per_iter": wall - dev}


def _train_serving_models(eng, _capi):
    rng = np.random.default_rng(4)
    n, f = 200_000, 100
    X = rng.standard_normal((n, f)).astype(np.float32)
    w = rng.standard_normal(f).astype(np.float32)
    y = ((X @ w + rng.normal(0, 1.0, n).astype(np.float32)) > 0).astype(np.float32)
    ds = eng.upload(X, y)
    ds.quantize(255)
    models = []
    for T, D in ((1000, 6), (200, 4), (500, 8), (2000, 10)):
        m, _ = eng.train(ds, _capi.params(loss="logloss", n_estimators=T, max_depth=D, learning_rate=0.1))
        models.append(m)
    return models


def _device_predict(models, f):
    """Device-resident prediction throughput of every model: 1M rows, kernel
    only (CUDA events on the launching stream, L2 flushed between launches)."""
    import torch

    n_dev = 1 << 20
    Xd = torch.randn((n_dev, f), dtype=torch.float32, device="cuda")
    od = torch.empty((n_dev, 1), dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()  # a real stream handle (0 would select the engine's own stream)
    torch.cuda.synchronize()
    dev_tp = {}
    for m in models:
        info = m.info
        exp = m.export()
        compares = float(np.sum(exp["depth"])) * n_dev
        for _ in range(3):
            m.predict_device(Xd.data_ptr(), n_dev, f, od.data_ptr(), "sigmoid", stream.cuda_stream)
        ts = []
        for _ in range(10):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            m.predict_device(Xd.data_ptr(), n_dev, f, od.data_ptr(), "sigmoid", stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        t = float(np.median(ts))
        dev_tp[f"{info.n_trees}xd{info.max_depth}"] = {
            "rows": n_dev, "ms": t * 1e3, "rows_per_s": n_dev / t, "gcompare_per_s": compares / t / 1e9,
            "input_gbs": n_dev * f * 4 / t / 1e9}
    del Xd, od, flush
    return dev_tp


def suite_c4(eng, _capi, seconds=3.0, rate=20_000.0, ref_ok=False):
    import torch

    models = _train_serving_models(eng, _capi)
    f = 100
    rng = np.random.default_rng(44)
    pool = torch.empty((65536 + 65536, f), dtype=torch.float32, pin_memory=True).numpy()
    pool[:] = rng.standard_normal(pool.shape).astype(np.float32)
    res = {"config": "serving: 4 resident models (1000xd6, 200xd4, 500xd8, 2000xd10) on 100 features; "
                     f"Poisson {rate:.0f} req/s for {seconds:.1f} s, rows log-uniform [1, 65536]"}
    # fixed-batch latency of the 1000 x depth-6 model (host buffers, H2D + kernel + D2H)
    lat = {}
    for rows in (1, 64, 4096, 65536):
        Xb = pool[:rows]
        for _ in range(3):
            models[0].predict(Xb, "sigmoid")
        ts = []
        for _ in range(30):
            t0 = time.perf_counter()
            models[0].predict(Xb, "sigmoid")
            ts.append(time.perf_counter() - t0)
        lat[str(rows)] = {"p50_us": _pct(ts, 50) * 1e6, "p99_us": _pct(ts, 99) * 1e6,
                          "rows_per_s": rows / _pct(ts, 50)}
    res["fixed_batch_1000xd6"] = lat
    # the same through the reference-shaped facade: TurboCatClassifier.predict_proba
    # on host (pageable) buffers, the model loaded from its TCAT file
    import turbocat

    path = os.path.join(tempfile.mkdtemp(), "m.tcat")
    with open(path, "wb") as fh:
        fh.write(models[0].tcat())
    clf = turbocat.TurboCatClassifier(verbosity=0).load(path)
    flat = {}
    for rows in (1, 64, 4096, 65536):
        Xb = np.ascontiguousarray(pool[:rows])
        for _ in range(3):
            clf.predict_proba(Xb)
        ts = []
        for _ in range(100 if rows <= 64 else 30):
            t0 = time.perf_counter()
            clf.predict_proba(Xb)
            ts.append(time.perf_counter() - t0)
        flat[str(rows)] = {"p50_us": _pct(ts, 50) * 1e6, "p99_us": _pct(ts, 99) * 1e6,
                           "rows_per_s": rows / _pct(ts, 50)}
    res["facade_predict_proba_1000xd6"] = flat
    res["device_predict_1M_rows"] = _device_predict(models, f)
    if ref_ok:
        sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
        import _turbocat as ref

        path = os.path.join(tempfile.mkdtemp(), "m.tcat")
        with open(path, "wb") as fh:
            fh.write(models[0].tcat())
        rm = ref.TurboCatClassifier(verbosity=0)
        rm.load(path)
        rl = {}
        for rows in (1, 64, 4096, 65536):
            Xb = np.ascontiguousarray(pool[:rows])
            rm.predict_proba(Xb)
            ts = []
            for _ in range(100 if rows <= 64 else 30):
                t0 = time.perf_counter()
                rm.predict_proba(Xb)
                ts.append(time.perf_counter() - t0)
            rl[str(rows)] = {"p50_us": _pct(ts, 50) * 1e6, "p99_us": _pct(ts, 99) * 1e6,
                             "rows_per_s": rows / _pct(ts, 50)}
        res["reference_cpu_fixed_batch_1000xd6"] = rl
        res["reference_cores"] = os.cpu_count()
    # open-loop Poisson streams: the configuration's rate (its mean request,
    # ~5.9k rows x 400 B, asks ~47 GB/s of host-to-device copies, about what
    # the PCIe link carries, so queues build up), and half of it
    n_out = 2048
    outs = [torch.empty((65536, 1), dtype=torch.float32, pin_memory=True).numpy() for _ in range(n_out)]
    for r in (rate, rate / 2):
        n_req = int(seconds * r)
        arr = np.cumsum(rng.exponential(1.0 / r, n_req))
        sizes = np.minimum(65536, np.floor(np.exp(rng.uniform(0, np.log(65537), n_req)))).astype(np.int64)
        mids = rng.integers(0, 4, n_req)
        offs = rng.integers(0, 65536, n_req)
        tag = "" if r == rate else f"_at_{int(r)}_per_s"
        for mode in ("coalesced", "plain"):
            srv = _capi.Server(eng, staging_bytes=0, max_batch_rows=262144, coalesce=(mode == "coalesced"),
                               max_inflight=4)
            ids = [srv.add_model(m) for m in models]
            reqs = [(float(arr[i]), ids[mids[i]], pool[offs[i]:offs[i] + sizes[i]], outs[i % n_out][:sizes[i]],
                     "sigmoid") for i in range(n_req)]
            lat_s, wall = srv.replay(reqs)
            done, launches, rows = srv.stats()
            res[mode + tag] = {"p50_ms": _pct(lat_s, 50) * 1e3, "p99_ms": _pct(lat_s, 99) * 1e3,
                               "rows_per_s": float(rows) / wall, "h2d_gbs": float(rows) * f * 4 / wall / 1e9,
                               "requests": int(done), "launches": int(launches), "wall_s": wall}
            srv.close()
    res["p99_improvement_vs_plain"] = res["plain"]["p99_ms"] / res["coalesced"]["p99_ms"]
    half = f"_at_{int(rate / 2)}_per_s"
    res["p99_improvement_vs_plain" + half] = res["plain" + half]["p99_ms"] / res["coalesced" + half]["p99_ms"]
    return res


def run_suite(args):
    import torch

    torch.cuda.set_device(0)
    from turbocat import _capi

    eng = _capi.Engine(0)
    ref_ok = os.path.exists(os.path.join(ROOT, "oracle", "_ref")) and not args.no_cpu_baseline
    for name in args.suite.split(","):
        t0 = time.perf_counter()
        if name == "c1":
            r = suite_c1(eng, _capi, ref_ok)
        elif name == "c3":
            r = suite_c3(eng, _capi)
        elif name == "c4":
            r = suite_c4(eng, _capi, ref_ok=ref_ok)
        elif name == "c2":  # the regression configuration alone, device-timed like the headline
            peak, kind = load_peaks()
            r = c2_secondary(eng, _capi, peak, kind, steps=5)
        elif name == "goss":
            r = suite_goss(eng, _capi)
        elif name == "cat":
            r = suite_cat(eng, _capi, ref_ok)
        elif name == "regular":
            r = suite_regular(eng, _capi, ref_ok)
        elif name == "c4dev":  # the four serving models' device-resident prediction only
            r = {"config": "serving models (1000xd6, 200xd4, 500xd8, 2000xd10) on 100 features, 1M resident rows",
                 "device_predict_1M_rows": _device_predict(_train_serving_models(eng, _capi), 100)}
        else:
            continue
        r["suite"] = name
        r["wall_s"] = time.perf_counter() - t0
        print(json.dumps(r), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-fits", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c2", action="store_true", help="leave out the secondary regression configuration")
    ap.add_argument("--reference-seconds", type=float, default=240.0,
                    help="reference arm: stop building trees once this many seconds have passed")
    ap.add_argument("--suite", default="", help="secondary configurations, e.g. c1,c2,c3,c4,goss,cat,regular")
    ap.add_argument("--rows", type=int, default=0,
                    help="rows of the workload (default: the configuration's 10M); a smaller case of the same "
                         "workload for profiler captures")
    args = ap.parse_args()
    if args.rows > 0:
        global N_ROWS
        N_ROWS = args.rows
        CONFIG["rows"] = N_ROWS
        CONFIG["workload"] = CONFIG["workload"].replace("10M x 200", f"{N_ROWS:,} x 200")
    if args.suite:
        run_suite(args)
        return
    if args.warmup < 3:
        log("warm-up raised to 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
