"""The engine's shared host/device arithmetic against the oracle, on the CPU.

Smoothing and the continuous-barrier bridge are written once (MCG_HD in
rust-pricing-library_b200/csrc) for both the path kernels and the host.  Here
they are compiled for the host with the same -fmad=false flag the kernels use
and compared with the oracle's restatement of
crates/pricing/src/product/smoothing.rs and
crates/pricing/src/engine/payoff/barrier_bridge.rs on seeded random inputs.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import helpers as H

SRC = os.path.join(H.ROOT, "tests", "host_math", "host_math.cu")
OUT = os.path.join(H.ROOT, "tests", "host_math", "_build", "libhostmath.so")


@pytest.fixture(scope="module")
def hm():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    csrc = os.path.join(H.ROOT, "rust-pricing-library_b200", "csrc")
    deps = [SRC] + [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith((".cuh", ".h"))]
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in deps):
        subprocess.run([nvcc, "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-shared", SRC, "-o", OUT],
                       check=True, capture_output=True)
    lib = C.CDLL(OUT)
    dp = C.POINTER(C.c_double)
    lib.hm_smoothing.argtypes = [C.c_double, C.c_double, dp]
    lib.hm_barrier_path.argtypes = [C.c_int, C.c_double, C.c_double, dp, dp, dp, C.c_uint, dp, dp]
    lib.hm_barrier_path.restype = C.c_int
    lib.hm_interval_adjoint.argtypes = [C.c_int] + [C.c_double] * 8 + [dp]
    return lib


def test_smoothing_matches_oracle(hm, oracle):
    rng = np.random.default_rng(3)
    for h in (0.5, 2.0, 1e-3):
        for x in np.concatenate([rng.uniform(-1.5 * h, 1.5 * h, 400), [-h, h, 0.0, h * (1 - 1e-16)]]):
            a, b = np.zeros(5), np.zeros(6)
            hm.hm_smoothing(h, float(x), H.dptr(a))
            oracle.oracle_smoothing(h, float(x), H.dptr(b))
            assert a[0] == b[0] and a[1] == b[1]      # indicator value and slope
            assert a[3] == b[3] and a[4] == b[4]      # positive part value and slope


@pytest.mark.parametrize("h", [0.0, 0.5])
@pytest.mark.parametrize("up", [0, 1])
def test_barrier_bridge_matches_oracle(hm, oracle, h, up):
    rng = np.random.default_rng(11 + up)
    for trial in range(60):
        n = 30
        t = np.linspace(0.0, 1.0, n + 1)
        drift = (-0.04 if not up else 0.04) * (trial % 3)
        z = rng.standard_normal(n)
        s = 100.0 * np.exp(np.concatenate([[0.0], np.cumsum(0.25 * np.sqrt(1.0 / n) * z + drift)]))
        v = rng.uniform(0.01, 0.09, n + 1)
        barrier = 85.0 if not up else 115.0
        a_s, b_s = C.c_double(), C.c_double()
        a_d, b_d = np.zeros(8), np.zeros(8)
        s, v, t = (np.ascontiguousarray(x) for x in (s, v, t))
        assert hm.hm_barrier_path(up, barrier, h, H.dptr(s), H.dptr(v), H.dptr(t), n + 1, C.byref(a_s), H.dptr(a_d)) == 0
        assert oracle.oracle_barrier_path(up, barrier, h, H.dptr(s), H.dptr(v), H.dptr(t), n + 1, C.byref(b_s), H.dptr(b_d)) == 0
        assert a_s.value == b_s.value
        assert np.array_equal(a_d, b_d)


@pytest.mark.parametrize("h", [0.0, 0.5])
def test_barrier_interval_adjoint_matches_oracle(hm, oracle, h):
    """The reverse of one bridge interval, used by the adjoint path kernel."""
    rng = np.random.default_rng(5)
    for _ in range(500):
        up = int(rng.integers(0, 2))
        barrier = 100.0
        ls = barrier * np.exp((1 if not up else -1) * rng.uniform(-0.01, 0.2))
        rs = barrier * np.exp((1 if not up else -1) * rng.uniform(-0.01, 0.2))
        lv, rv, dt, lsa = rng.uniform(0.01, 0.09), rng.uniform(0.01, 0.09), 1.0 / 252, rng.normal()
        a, b = np.zeros(4), np.zeros(4)
        hm.hm_interval_adjoint(up, barrier, h, lsa, ls, rs, lv, rv, dt, H.dptr(a))
        if oracle.oracle_interval_adjoint(up, barrier, h, lsa, ls, rs, lv, rv, dt, H.dptr(b)) != 0:
            continue
        assert np.array_equal(a, b), (up, ls, rs, a, b)
