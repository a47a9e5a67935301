"""The ctypes mirrors of the C ABI's structs (turbocat/_capi.py) have the
sizes and field offsets of include/tcgpu.h as a C compiler lays them out: a
probe compiled with gcc against the header prints both, on the CPU."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [("TrainParams", "tc_train_params"), ("TrainStats", "tc_train_stats"), ("KernelTime", "tc_kernel_time"),
         ("Profile", "tc_profile"), ("ModelInfo", "tc_model_info"), ("ServerParams", "tc_server_params"),
         ("ReplayRequest", "tc_replay_request"), ("CatParams", "tc_cat_params")]


def _probe(capi):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tcgpu.h"', "int main(void) {"]
    for py, c in PAIRS:
        cls = getattr(capi, py)
        lines.append(f'  printf("{c} size %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'  printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as td:
        src, exe = os.path.join(td, "probe.c"), os.path.join(td, "probe")
        open(src, "w").write("\n".join(lines) + "\n")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True,
                       capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        c, field, v = line.split()
        got[(c, field)] = int(v)
    return got


def test_ctypes_structs_match_the_header(capi):
    import ctypes as C

    if subprocess.run(["which", "gcc"], capture_output=True).returncode != 0:
        pytest.skip("no C compiler")
    got = _probe(capi)
    for py, c in PAIRS:
        cls = getattr(capi, py)
        assert C.sizeof(cls) == got[(c, "size")], (py, C.sizeof(cls), got[(c, "size")])
        for name, _ in cls._fields_:
            assert getattr(cls, name).offset == got[(c, name)], (py, name)
