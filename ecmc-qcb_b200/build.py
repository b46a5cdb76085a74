"""Builds libqcb.so (CUDA kernels + C ABI) in-tree for sm_100a with nvcc.

    python ecmc-qcb_b200/build.py [-v]

Each translation unit under csrc/ is compiled to _build/*.o in parallel and linked
into ecmc-qcb_b200/libqcb.so; the same sources compiled with -DQCB_CHECKED into
_build/checked/*.o give libqcb_checked.so, whose kernels validate every field index
(the out-of-bounds record of qcb_debug_oob).  Objects are rebuilt when a source or
header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqcb.so")
CHECKED_LIB = os.path.join(HERE, "libqcb_checked.so")
HOST = os.path.join(HERE, "host", "src")
COMPAT = os.path.join(HERE, "libqcb_compat.a")
DRIVER = os.path.join(HERE, "qcb_hb_cb")
CXX = "/usr/bin/g++"
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++"]


def _deps_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def _compile(src: str, verbose: bool, checked: bool = False) -> str:
    out = os.path.join(BUILD, "checked") if checked else BUILD
    obj = os.path.join(out, os.path.basename(src).rsplit(".", 1)[0] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *(["-DQCB_CHECKED"] if checked else []), "-c", src, "-o", obj]
    if verbose and not checked:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def _link(lib: str, objs: list) -> None:
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-ccbin", "/usr/bin/g++"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of {os.path.basename(lib)} failed:\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False) -> str:
    os.makedirs(os.path.join(BUILD, "checked"), exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = [(s, False) for s in srcs] + [(s, True) for s in srcs]
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 8)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], verbose, j[1]), jobs))
    _link(LIB, objs[:len(srcs)])
    _link(CHECKED_LIB, objs[len(srcs):])
    build_host()
    return LIB


def build_host() -> None:
    """The C++ layer with the reference's signatures (libqcb_compat.a) and the run driver."""
    srcs = [os.path.join(HOST, "qcb_compat.cpp"), os.path.join(HOST, "io", "io.cpp")]
    objs = []
    for src in srcs:
        obj = os.path.join(BUILD, "host_" + os.path.basename(src).replace(".cpp", ".o"))
        hdr = max(os.path.getmtime(h) for h in glob.glob(os.path.join(HOST, "**", "*.h"), recursive=True))
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr):
            r = subprocess.run([CXX, "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", "-c", src, "-o", obj],
                               capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"g++ failed on {src}:\n{r.stderr}")
        objs.append(obj)
    if not os.path.exists(COMPAT) or os.path.getmtime(COMPAT) < max(os.path.getmtime(o) for o in objs):
        if os.path.exists(COMPAT):
            os.remove(COMPAT)
        subprocess.run(["ar", "rcs", COMPAT, *objs], check=True)
    drv = os.path.join(HOST, "bin", "gauge_hb_cb.cpp")
    if not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < max(os.path.getmtime(drv), os.path.getmtime(COMPAT),
                                                                   os.path.getmtime(LIB)):
        r = subprocess.run([CXX, "-std=c++17", "-O2", "-Wall", "-Wextra", drv, COMPAT, "-L" + HERE, "-lqcb",
                            "-Wl,-rpath,$ORIGIN", "-o", DRIVER], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver link failed:\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
