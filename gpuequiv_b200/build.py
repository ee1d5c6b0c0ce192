"""Build libgeq.so (the C-ABI solver library) in-tree for sm_100a.

    python gpuequiv_b200/build.py            # gpuequiv_b200/libgeq.so
    python gpuequiv_b200/build.py --checked  # gpuequiv_b200/libgeq_checked.so

(Run it as a script: importing the package loads the library it builds.)

The checked variant compiles every device load/store of the solver with an
index check that records the offending line and stops the solve instead of
touching memory out of range.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["engine.cu", "gbuild.cu", "wide.cu", "api.cpp", "lts.cpp", "gamebuild.cpp", "pipeline.cpp", "server.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(checked: bool = False, force: bool = False, verbose: bool = False) -> str:
    name = "libgeq_checked.so" if checked else "libgeq.so"
    out = os.path.join(HERE, name)
    bdir = os.path.join(HERE, "_build", "checked" if checked else "release")
    os.makedirs(bdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "geq.h"))
    flags = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fvisibility=hidden",
                    "-I", INCLUDE, "-I", CSRC]
    if checked:
        flags += ["-DGEQ_CHECKED=1"]
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + headers):
            cmd = [nvcc()] + flags + (["-x", "cu"] if src.endswith(".cu") else []) + ["-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not _newer(out, objs):
        run([nvcc()] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    if not checked:
        build_loadgen(force)
    return out


def build_loadgen(force: bool = False) -> str:
    """libgeq_load.so: the serving loop's native load driver (csrc/loadgen.cpp,
    no CUDA), used by the bench and its CPU test."""
    src = os.path.join(CSRC, "loadgen.cpp")
    out = os.path.join(HERE, "libgeq_load.so")
    if force or not _newer(out, [src]):
        r = subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", src, "-o", out],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed: loadgen.cpp\n" + r.stdout + r.stderr)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--checked", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(checked=a.checked, force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
