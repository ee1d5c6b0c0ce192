"""The device game builder's level loop (gbuild.cuh) and the device
minimisation (refine.cuh), compiled for the host and run through a sequential
backend (tests/gbuild_host.cpp), against the host GameBuilder
(src/gamebuild.rs restated in gamebuild.cpp) and Lts::minimize
(src/lib.rs:413-478): exact CSR, numbering, the position bound, start sets of
compare_all, capacity hints, partitions and minimised systems.  No GPU needed:
the kernels run the same functors on the device."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpuequiv_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("gbuild") / "gbuild_host"
    cmd = ["g++", "-O2", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "gbuild_host.cpp"), os.path.join(CSRC, "gamebuild.cpp"),
           os.path.join(CSRC, "lts.cpp"), "-o", str(out), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(out)


def run(driver, *args):
    r = subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("bad 0 of"), r.stdout
    return r.stdout


# jobs, max states, max positions (0: none), seed, transitions per state, labels, warp-path |Q| (huge: none), compare_all
BUILD_CASES = [
    (200, 30, 0, 7, 3, 4, 4, 0),          # compare, the warp-path split as on the device
    (200, 30, 0, 8, 3, 4, 0xFFFFFFFF, 0),  # every attack position on the thread path
    (100, 20, 20000, 3, 8, 2, 1, 0),      # dense, bounded: jobs over the bound refused
    (300, 15, 0, 6, 2, 3, 2, 0),          # sparse, many jobs
    (40, 25, 100000, 3, 3, 3, 4, 1),      # compare_all start sets
    (50, 1, 0, 9, 0, 1, 4, 1),            # no start pairs at all
]


@pytest.mark.parametrize("case", BUILD_CASES, ids=[f"build{i}" for i in range(len(BUILD_CASES))])
def test_level_loop_vs_host_builder(driver, case):
    run(driver, "build", *case)


# jobs, max states, seed, transitions per state, labels
REFINE_CASES = [(80, 40, 5, 2, 2), (60, 200, 9, 1, 1), (200, 60, 11, 4, 6), (20, 1, 3, 0, 1)]


@pytest.mark.parametrize("case", REFINE_CASES, ids=[f"refine{i}" for i in range(len(REFINE_CASES))])
def test_refinement_vs_host_minimize(driver, case):
    run(driver, "refine", *case)
