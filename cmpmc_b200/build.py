"""Builds the in-tree shared library cmpmc_b200/_lib/libcmpmc_b200.so.

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
The batched phonon kernels use FP32 intrinsics (``--use_fast_math``). The plain FP64
transport translation unit is compiled with ``--fmad=false`` so that its
arithmetic rounds like the CPU reference (x86-64 SSE, no FMA contraction); the host
sources are compiled the same way for the same reason (the lattice tables and the host
make_track must be bit-identical to the reference's).

Usage: python -m cmpmc_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "libcmpmc_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
                      "-I", INCLUDE, "-Xptxas", "-v"]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-pthread", "-I", INCLUDE]

# source -> extra flags
SOURCES = {
    "lattice_host.cpp": [],
    "host.cpp": [],
    "mesh_host.cpp": [],
    "partition_host.cpp": [],
    "kaplan_lut.cpp": [],
    "transport_plain.cu": ["--fmad=false"],
    "partition_gpu.cu": ["--fmad=false"],
    # FP32 intrinsics for the batched phonon kernels (about 3 % faster; the chi^2 parity and
    # the FP64 ledger are unchanged); the FP64 Kaplan cascade is not affected
    "transport_batched.cu": ["--use_fast_math"],
    "charges_batched.cu": [],
    "finish.cu": [],
    "capi.cu": [],
}


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build cmpmc_b200")


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs.append(os.path.join(INCLUDE, "cmpmc_gpu.h"))
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, extra: list[str], force: bool) -> tuple[str, str]:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if not force and not _stale(obj, [path] + _headers()):
        return obj, ""
    if src.endswith(".cu"):
        cmd = [_nvcc()] + NVCC_COMMON + extra + ["-c", path, "-o", obj]
    else:
        cmd = [os.environ.get("CXX", "g++")] + CXX_FLAGS + extra + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = {ex.submit(_compile, s, f, force): s for s, f in SOURCES.items()}
        objs, logs = [], {}
        for fut in cf.as_completed(futs):
            obj, log = fut.result()
            objs.append(obj)
            logs[futs[fut]] = log
    objs.sort()
    lib = os.path.join(LIBDIR, LIBNAME)
    if force or _stale(lib, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-Xcompiler", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        for s, log in sorted(logs.items()):
            if log:
                print(f"== {s}\n{log}", file=sys.stderr)
    return lib


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("-v", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, jobs=args.j, verbose=args.v))


if __name__ == "__main__":
    main()
