"""Build the in-tree shared library cipher_b200/libcipher_b200.so.

CUDA sources are compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); host C sources with gcc.  nvcc links the
CUDA runtime statically, so the library needs no toolkit at run time and
travels with the repository snapshot.

Usage: ``python -m cipher_b200.build`` (or ``cipher_b200.build.build()``).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD_DIR = os.path.join(ROOT, "_build", "cipher_b200")
LIB = os.path.join(HERE, "libcipher_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# FP64 translation units keep the reference's IEEE arithmetic: no multiply-add
# contraction (the reference's x86-64 build has none either).
NVCC_COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + os.path.join(CSRC, "cuda")]
NVCC_EXACT = ["--fmad=false"]
# sources whose arithmetic may contract (mixed-precision kernels)
FAST_SOURCES: set[str] = {"rhs_mixed.cu"}

CC_FLAGS = ["-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
            "-I" + INCLUDE]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build cipher_b200")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    out = []
    for d in (INCLUDE, os.path.join(CSRC, "cuda"), os.path.join(CSRC, "host")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                out.append(os.path.join(d, f))
    return out


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA and host source and link the shared library."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    objs = []
    jobs = []
    cu_dir = os.path.join(CSRC, "cuda")
    for f in sorted(os.listdir(cu_dir)):
        if not f.endswith(".cu"):
            continue
        src = os.path.join(cu_dir, f)
        obj = os.path.join(BUILD_DIR, f[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            flags = NVCC_COMMON + ([] if f in FAST_SOURCES else NVCC_EXACT)
            if ptxas_info:
                flags = flags + ["-Xptxas", "-v"]
            jobs.append([nvcc] + ARCH + flags + ["-c", src, "-o", obj])
    # the translation units are independent: compile them concurrently
    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        for fut in [pool.submit(_run, cmd, verbose or ptxas_info) for cmd in jobs]:
            fut.result()
    host_dir = os.path.join(CSRC, "host")
    cc = shutil.which("gcc") or "cc"
    for f in sorted(os.listdir(host_dir)):
        if not f.endswith(".c"):
            continue
        src = os.path.join(host_dir, f)
        obj = os.path.join(BUILD_DIR, "host_" + f[:-2] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            _run([cc] + CC_FLAGS + ["-c", src, "-o", obj], verbose)
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
