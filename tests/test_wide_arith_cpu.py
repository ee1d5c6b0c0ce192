"""The multi-word solver's arithmetic (wide_arith.cuh: SWAR field-wise <= and
max, the inverse update) compiled for the host, against the oracle's
restatement of shadergen.rs:55-157 on random energies and updates of many
EnergyConfs -- fields of 1 to 32 bits, one to several words."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import ora

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpuequiv_b200", "csrc")

CONFS = [(1, 0xFFFFFFFF), (1, 1), (6, 3), (8, 2), (30, 3), (3, 1000), (16, 7), (100, 1), (2, 65535),
         (5, 0xFFFF), (12, 15), (7, 200), (40, 1)]


@pytest.fixture(scope="module")
def wa(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    out = tmp_path_factory.mktemp("wa") / "libwa.so"
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "wide_arith_host.cpp"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(str(out))
    p = C.POINTER(C.c_uint32)
    L.wa_leq.argtypes = [C.c_uint32, C.c_uint32, p, p]
    L.wa_leq.restype = C.c_int
    L.wa_max.argtypes = [C.c_uint32, C.c_uint32, p, p, p]
    L.wa_inv_update.argtypes = [C.c_uint32, C.c_uint32, p, p, p]
    return L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def rand_energy(rng, el, mx):
    hi = min(mx, 2**32 - 1)
    v = rng.integers(0, hi + 1, el, dtype=np.uint64)
    # values at the edges of the range as well (saturation, u32 wrap)
    edge = rng.random(el) < 0.25
    v[edge] = rng.choice(np.array([0, hi, max(hi - 1, 0)], dtype=np.uint64), int(edge.sum()))
    return ora.pack_energy(el, mx, v.astype(np.uint32))


def rand_update(rng, el):
    u = np.zeros(el, np.int32)
    for i in range(el):
        r = rng.random()
        if r < 0.3:
            u[i] = -1
        elif r < 0.5:
            u[i] = int(rng.integers(1, el + 1))
    return u


@pytest.mark.parametrize("conf", CONFS)
def test_swar_and_inverse_update_vs_oracle(wa, conf):
    el, mx = conf
    rng = np.random.default_rng(el * 7919 + (mx & 0xFFFF))
    for _ in range(300):
        a, b = rand_energy(rng, el, mx), rand_energy(rng, el, mx)
        va, vb = ora.unpack_energy(el, mx, a), ora.unpack_energy(el, mx, b)
        assert wa.wa_leq(el, mx, _p(a), _p(b)) == int(bool(np.all(va <= vb)))
        assert wa.wa_leq(el, mx, _p(a), _p(a)) == 1
        out = np.zeros_like(a)
        wa.wa_max(el, mx, _p(a), _p(b), _p(out))
        assert np.array_equal(ora.unpack_energy(el, mx, out), np.maximum(va, vb))
        u = ora.pack_update(el, mx, rand_update(rng, el))
        got = np.zeros_like(a)
        wa.wa_inv_update(el, mx, _p(a), _p(u), _p(got))
        assert np.array_equal(got, ora.inv_update(el, mx, a, u)), (conf, va, ora.unpack_update(el, mx, u))
