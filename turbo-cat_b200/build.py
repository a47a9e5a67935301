"""Build script for the B200 engine.

Compiles, in-tree:
  turbocat/libtcgpu.so            the CUDA kernels + C ABI (include/tcgpu.h), sm_100a only
  turbocat/_turbocat<ext-suffix>  the pybind11 module mirroring the reference's
                                  python/bindings.cpp surface, linked to libtcgpu.so

Usage: python turbo-cat_b200/build.py [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "turbocat")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"  # the image's CXX wrapper cannot link OpenMP/shared objects reliably
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                     f"-I{INCLUDE}", f"-I{CSRC}", "--expt-relaxed-constexpr", "-Xptxas", "-v"]

CU_SOURCES = ["tc_context.cu", "tc_data.cu", "tc_train.cu", "tc_predict.cu", "tc_server.cu", "tc_noalloc.cu",
              "tc_regular.cu"]
HOST_SOURCES = ["bindings.cpp"]

LIB = os.path.join(PKG, "libtcgpu.so")
EXT = os.path.join(PKG, "_turbocat" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def _run(cmd, log):
    p = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as fh:
        fh.write(" ".join(cmd) + "\n" + p.stdout + p.stderr)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... (log {log})")
    return p


def build(force: bool = False) -> None:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(INCLUDE, "tcgpu.h"), os.path.join(CSRC, "tc_internal.h"), os.path.join(CSRC, "tc_loss.cuh")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer([s] + headers, o):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        futs = [ex.submit(_run, j, j[-1] + ".log") for j in jobs]
        for f in futs:
            f.result()
    if force or _newer(objs, LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs, os.path.join(OBJ, "link.log"))

    import pybind11

    py_inc = sysconfig.get_paths()["include"]
    srcs = [os.path.join(CSRC, s) for s in HOST_SOURCES]
    if force or _newer(srcs + headers + [LIB], EXT):
        _run([CXX, "-O3", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", f"-I{INCLUDE}",
              f"-I{py_inc}", f"-I{pybind11.get_include()}", *srcs, "-o", EXT, f"-L{PKG}", "-ltcgpu",
              "-Wl,-rpath,$ORIGIN"], os.path.join(OBJ, "bindings.log"))


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("built", LIB, EXT)
