"""Builds libdgsem_b200.so in-tree for sm_100a.

  python -m dgsem_b200.build            # incremental
  python -m dgsem_b200.build --force    # rebuild everything

CUDA sources are compiled with nvcc (-gencode arch=compute_100a,code=sm_100a
-lineinfo -O3), the host table precompute (tables.cpp) with the host C++
compiler and -ffp-contract=off (it restates the reference's host arithmetic
bit for bit).  Objects go to dgsem_b200/_build, the library to
dgsem_b200/_lib/libdgsem_b200.so.
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
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libdgsem_b200.so")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-I", CSRC, "-I", os.path.join(ROOT, "include"),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _hostcxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("host C++ compiler not found")


def _deps_newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers() -> list[str]:
    out = [os.path.join(ROOT, "include", "dgsem_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cuh", ".hpp", ".h")):
            out.append(os.path.join(CSRC, f))
    return out


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    sys.path.insert(0, HERE)
    import gen_engines  # noqa: E402

    gen = gen_engines.generate()
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    cu_sources = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
    cu_sources += [g for g in gen if g.endswith(".cu")]
    jobs_list = []
    objects = []
    for src in cu_sources:
        obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
        objects.append(obj)
        if force or _deps_newer(obj, [src] + headers):
            jobs_list.append([nvcc] + NVCC_FLAGS + ["-c", src, "-o", obj])
    tables_obj = os.path.join(BUILD, "tables.o")
    objects.append(tables_obj)
    tables_src = os.path.join(CSRC, "tables.cpp")
    if force or _deps_newer(tables_obj, [tables_src] + headers):
        jobs_list.append([_hostcxx(), "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off",
                          "-I", CSRC, "-c", tables_src, "-o", tables_obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    n_jobs = jobs or max(1, min(len(jobs_list), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(max_workers=n_jobs) as ex:
        list(ex.map(run, jobs_list))
    if force or jobs_list or _deps_newer(LIB, objects):
        run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB]
            + objects + ["-Xcompiler", "-fPIC"])
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, jobs=a.jobs))


if __name__ == "__main__":
    main()
