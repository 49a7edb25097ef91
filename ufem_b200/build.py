"""Build libufem_gpu.so in-tree for sm_100a (B200).

    python -m ufem_b200.build          # or: python ufem_b200/build.py

Every source of ufem_b200/csrc (host model code and CUDA) is compiled to an
object file in ufem_b200/_build by its own nvcc process, the processes run in
parallel, and one nvcc link step makes ufem_b200/lib/libufem_gpu.so.  No
translation unit references another's device code (no relocatable device
code), so the objects link like host objects.  nvcc cross-compiles, so this
runs without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libufem_gpu.so")

SOURCES = ["model.cpp", "kernels.cu", "solve.cu", "batch.cu", "capi.cu", "monte.cu", "mcout.cu", "mlp.cu", "warm.cu",
           "selftest.cu", "pattern.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr",
]
LINK_FLAGS = ARCH + ["-shared", "-Xlinker", "--no-undefined", "-cudart", "static"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "ufem_gpu.h"))
    return [h for h in hs if os.path.exists(h)]


def _obj(src):
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in sources() + _headers())


def _compile(nvcc, src, force, newest_header, verbose):
    obj = _obj(src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
        return obj, None
    cmd = [nvcc, *COMPILE_FLAGS, "-c", "-o", obj, src]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    return obj, (None if r.returncode == 0 else r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    newest_header = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(nvcc, s, force, newest_header, verbose), srcs))
    errs = [e for _, e in results if e]
    if errs:
        sys.stderr.write("\n".join(errs))
        raise RuntimeError("nvcc failed compiling libufem_gpu.so")
    cmd = [nvcc, *LINK_FLAGS, "-o", LIB, *[o for o, _ in results]]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libufem_gpu.so")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
