"""Build recipe for libqes_b200.so (sm_100a), in-tree next to this file.

    python -m pyqusolver_b200.build            # rebuild if any source is newer
    python -m pyqusolver_b200.build --force

nvcc cross-compiles for sm_100a without a GPU.  The library is plain C ABI
(``include/qes_b200.h``); Python binds it with ctypes.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_NAME = "libqes_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)
SOURCES = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
HEADERS = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(ROOT, "include", "qes_b200.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS)


OBJ_DIR = os.path.join(HERE, "_build")


def _obj(src: str) -> str:
    return os.path.join(OBJ_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel (objects older than their source or any header
    are rebuilt), then link the shared library."""
    if not force and not needs_build():
        return LIB_PATH
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in HEADERS + glob.glob(os.path.join(HERE, "csrc", "*.h")))
    todo = [s for s in SOURCES if force or not os.path.exists(_obj(s)) or
            os.path.getmtime(_obj(s)) < max(os.path.getmtime(s), newest_header)]
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"] + ["-c"]

    def compile_one(src):
        cmd = [_nvcc()] + compile_flags + ["-o", _obj(src) + ".tmp", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode == 0:
            os.replace(_obj(src) + ".tmp", _obj(src))
        return src, res

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, todo))
    failed = [(s, r) for s, r in results if r.returncode != 0]
    for s, r in failed:
        sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(s) for s, _ in failed))
    tmp = LIB_PATH + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-o", tmp] + \
        [_obj(s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking " + LIB_NAME)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=True))
