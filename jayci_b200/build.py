"""Build libjci.so (and the jci / jci_dyson driver programs) in-tree for sm_100a.

    python -m jayci_b200.build [--force]

Every CUDA unit is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; host units
with the same nvcc driver.  Objects go to ``jayci_b200/_build/``; the shared
library lands next to this file so that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libjci.so")
EXE = os.path.join(HERE, "jci")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["jci_space.cpp", "jci_io.cpp", "jci_api.cpp", "jci_server.cpp", "jci_device.cu", "jci_fci.cu",
           "jci_fci_ab.cu", "jci_fci_tc.cu", "jci_fci_group.cu", "jci_fci_pairs.cu", "jci_davidson.cu", "jci_dyson.cu"]
# driver programs: (source, executable)
PROGRAMS = [("jci_main.c", "jci"), ("jci_dyson_main.c", "jci_dyson")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: libjci needs the CUDA toolkit to build")


def host_compiler() -> list[str]:
    # the system g++ ships libgomp/libstdc++ matching the CUDA toolkit
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _deps(src: str) -> list[str]:
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return [src, os.path.join(INCLUDE, "jci.h")] + hdrs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def compile_one(src: str, force: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if force or _stale(obj, _deps(path)):
        cmd = [nvcc(), *host_compiler(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
               "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC, "-c", path, "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-warn-spills"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), SOURCES))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    for src, exe in PROGRAMS:
        main, out = os.path.join(CSRC, src), os.path.join(HERE, exe)
        if force or _stale(out, [main, LIB, os.path.join(INCLUDE, "jci.h")]):
            cmd = ["/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc", "-O2",
                   "-std=gnu11", "-I", INCLUDE, main, "-o", out, "-L", HERE, "-ljci",
                   "-Wl,-rpath,$ORIGIN", "-lm"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, verbose=True)
