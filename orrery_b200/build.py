"""Builds the native library ``orrery_b200/_native/liborrery_lbm.so`` in-tree.

Every CUDA translation unit is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), host C++ with the same nvcc
driver, and the objects are linked into one shared library with the CUDA
runtime linked statically.  The binary64 kernel unit is compiled with
``-fmad=false`` so its arithmetic rounds like the reference CPU solver.

Usage: ``python -m orrery_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
OUT_DIR = os.path.join(HERE, "_native")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIBRARY = os.path.join(OUT_DIR, "liborrery_lbm.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I", INCLUDE, "-I", CSRC]

SOURCES = {
    "common.cpp": [],
    "host_copy.cpp": [],
    "plan.cpp": [],
    "kernels_f32.cu": [],
    "kernels_f16.cu": [],
    "kernels_bf16.cu": [],
    "kernels_f64.cu": ["-fmad=false"],
    "solver3d.cu": [],
    "solver2d.cu": [],
    "force_static.cu": [],
    "tiles.cu": [],
    "gl3d.cu": [],
    "gl2d.cu": [],
    "batch3d.cu": [],
    "serve3d.cu": [],
    "voxel.cu": ["-fmad=false"],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the native library needs the CUDA toolkit")
    return path


def _headers() -> list[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    files.append(os.path.join(INCLUDE, "orrery_lbm.h"))
    return files


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra: list[str], verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, src + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + _headers()
    if not _stale(obj, deps):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    cmd = [nvcc()] + ARCH + COMMON + extra + lang + ["-c", path, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles what changed and links the library; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    if force:
        for f in os.listdir(OBJ_DIR):
            os.remove(os.path.join(OBJ_DIR, f))
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        futures = [pool.submit(_compile, src, extra, verbose) for src, extra in SOURCES.items()]
        objects = [f.result() for f in futures]
    if force or _stale(LIBRARY, objects):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIBRARY] + objects + ["-cudart", "static"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIBRARY


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
