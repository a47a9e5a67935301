"""The multi-process plumbing of bench.py, on CPU with the gloo backend and
two ranks: process-group set-up from the torchrun environment, the barrier,
the max-over-ranks timing that the whole-job number is built from, and the
reference arm's rule that only rank 0 measures."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    os.environ.update({"WORLD_SIZE": str(ws), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, local = bench.dist_setup("gloo")
    assert (w, r, local) == (ws, rank, rank)
    # per-rank "step seconds": rank r took 1 + r seconds; the job is as slow as its slowest rank
    mine = 1.0 + rank
    total = bench.dist_max(mine, w)
    bench.dist_barrier(w)
    steps = 5
    value = total / (steps * w)  # the whole-job aggregate bench.py reports (seconds per 100 trees)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump({"total": total, "value": value}, fh)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp

    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]
    for r in res:
        assert r["total"] == pytest.approx(2.0)          # max over ranks, not rank 0's own
        assert r["value"] == pytest.approx(2.0 / (5 * 2))


def test_reference_arm_runs_on_rank0_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(type("A", (), {"steps": 1, "warmup": 0, "gpus": 2})())
    assert buf.getvalue() == ""  # a non-zero rank exits without work and prints nothing
