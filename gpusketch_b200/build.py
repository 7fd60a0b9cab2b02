"""Builds the gpusketch_b200 native library in-tree for sm_100a.

    python -m gpusketch_b200.build          # incremental
    python -m gpusketch_b200.build --clean  # from scratch

Outputs gpusketch_b200/libgpusketch_b200.so (CUDA kernels + the C ABI of include/gpusketch.h,
cudart linked statically) and gpusketch_b200/_build/*.o.  Also builds the C++ drop-in example
program gpusketch_b200/_build/cc_dropin_demo from gpusketch_b200/cpp/ when it exists.
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
LIB = os.path.join(HERE, "libgpusketch_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
                     "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I/usr/local/cuda/include",
             "-I" + os.path.join(ROOT, "include")]


def _deps() -> list[str]:
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hdrs + [os.path.join(ROOT, "include", "gpusketch.h")]


def _stale(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def _compile(src: str, deps: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _stale(obj, src, deps):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, deps), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    _build_cpp_dropin(verbose)
    return LIB


def _build_cpp_dropin(verbose: bool) -> None:
    """Compiles the C++ drop-in demo (reference-named classes over the C ABI), if present."""
    cpp_dir = os.path.join(HERE, "cpp")
    demo = os.path.join(cpp_dir, "cc_dropin_demo.cpp")
    if not os.path.exists(demo):
        return
    out = os.path.join(BUILD, "cc_dropin_demo")
    hdrs = [os.path.join(cpp_dir, f) for f in os.listdir(cpp_dir) if f.endswith(".h")]
    if os.path.exists(out) and all(os.path.getmtime(out) > os.path.getmtime(p) for p in hdrs + [demo, LIB]):
        return
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I" + os.path.join(ROOT, "include"), "-I" + cpp_dir,
           demo, "-o", out, "-L" + HERE, "-lgpusketch_b200", "-Wl,-rpath,$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"drop-in demo build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args()
    build(clean=a.clean, verbose=True)
    sys.exit(0)
