"""GPU sampling primitives against the oracle: bit-exact Philox normals and
scrambled Sobol words, and the SSVI -> Dupire grid within 1e-13."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import sobol
from rust_pricing_b200 import workloads as W
import gpu_common as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("domain", [0, 1])
def test_philox_normals_bit_exact(oracle, engine, domain):
    n, dims, first = 2048, 9, (1 << 33) - 100
    out = np.zeros(n * dims)
    N.check(engine.mcg_philox_normals(W.SEED, first, n, dims, domain, H.dptr(out)))
    ref = np.array([[oracle.oracle_philox_normal(W.SEED, first + i, d, domain) for i in range(n)]
                    for d in range(dims)]).ravel()
    assert np.array_equal(out.view(np.uint64), ref.view(np.uint64))


def test_rqmc_words_bit_exact(oracle, engine):
    dims, n = 40, 1024
    dirs = np.ascontiguousarray(sobol.direction_words(dims))
    for scramble in (0, 5):
        words = np.zeros(n * dims, dtype=np.uint32)
        N.check(engine.mcg_rqmc_words(H.uptr(dirs), dims, W.SEED, scramble, 1000, n, H.uptr(words)))
        ref = np.array([[oracle.oracle_rqmc_word(H.uptr(dirs[d]), W.SEED, scramble, d, 1000 + i)
                         for i in range(n)] for d in range(dims)], dtype=np.uint32).ravel()
        assert np.array_equal(words, ref)


def test_rqmc_scramble_known_words(engine):
    dirs = np.ascontiguousarray(sobol.direction_words(2))
    words = np.zeros(8 * 2, dtype=np.uint32)
    N.check(engine.mcg_rqmc_words(H.uptr(dirs), 2, 0x0123456789ABCDEF, 0, 0, 8, H.uptr(words)))
    assert words[0] == 0x46C5FD35 and words[1] == 0xE684A5D7 and words[8 + 2] == 0x7D21CC82


def test_ssvi_local_variance_grid(engine):
    surface = W.SsviSurface()
    gpu = G.gpu_grid(surface, 1e-8, 4.0)
    ref = G.oracle_grid(surface, 1e-8, 4.0)
    assert gpu.shape == (31, 100)
    assert np.max(np.abs(gpu - ref) / np.abs(ref)) < 1e-13
