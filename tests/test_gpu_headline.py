"""Parity at the benchmark's own sizes.

The small-size parity tests run a few thousand Sobol points, so they exercise
only the low Gray-code bits of the point index.  The benchmark prices 2^20
points per scramble; these tests compare the engine with the oracle where the
high bits are set:

* the local-volatility RQMC workload (SSVI -> Dupire 31 x 100 grid, 252 daily
  steps, Brownian bridge, Asian call and discrete down-and-out call on the same
  draws) at its full 2^20 points, for two scrambles -- the last two of the
  benchmark's sixteen (an RQMC estimate needs two replicates) -- engine vs
  oracle within the 1e-12 component tolerance, and each scramble's mean;
* the scrambled Sobol words that the path kernels form warp by warp, at
  32-aligned point indices up to 2^20 - 1 (all twenty Gray-code bits), bit for
  bit against the oracle's word-by-word construction;
* the American put by LSM (50 exercise dates) at 2^18 training and 2^18
  valuation paths: every stopping index, the exercise counts and the price
  against the oracle.
"""
import os

import numpy as np
import pytest

import gpu_common as G
import helpers as H
from rust_pricing_b200 import _native as N
from rust_pricing_b200 import sobol
from rust_pricing_b200 import workloads as W
from test_gpu_lsm import assert_same_result

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


def test_local_vol_rqmc_workload_full_points_last_scrambles(engine):
    spec = W.local_vol_rqmc(G.gpu_grid, points=1 << 20, scrambles=2)
    spec.scramble_begin = 14
    engine_buf, oracle_buf = G.assert_parity(spec, threads=THREADS)
    assert engine_buf.result.evaluated_paths == 2 << 20
    for k in range(2):
        got, want = engine_buf.replicate_means(k), oracle_buf.replicate_means(k)
        assert len(got) == 2
        for a, b in zip(got, want):
            assert abs(a - b) <= G.DIRECT_TOL * abs(b)


@pytest.mark.parametrize("first", [(1 << 20) - 4096, (1 << 19) - 2048, 0xAAAA0])
def test_warp_sobol_words_at_high_point_indices(oracle, engine, first):
    dims, n = 252, 4096 if first == (1 << 20) - 4096 else 2048
    dirs = np.ascontiguousarray(sobol.direction_words(dims))
    assert first % 32 == 0 and n % 32 == 0  # the warp-cooperative path
    for scramble in (0, 15):
        words = np.zeros(n * dims, dtype=np.uint32)
        N.check(engine.mcg_rqmc_words(H.uptr(dirs), dims, W.SEED, scramble, first, n, H.uptr(words)))
        words = words.reshape(dims, n)
        for d in (0, 1, 7, 100, 251):
            ref = np.array([oracle.oracle_rqmc_word(H.uptr(dirs[d]), W.SEED, scramble, d, first + i)
                            for i in range(n)], dtype=np.uint32)
            assert np.array_equal(words[d], ref), (scramble, d)


def test_unaligned_words_match_the_warp_path(engine):
    """The per-thread form (unaligned start) and the warp form give the same words."""
    dims = 16
    dirs = np.ascontiguousarray(sobol.direction_words(dims))
    first = (1 << 20) - 1024
    a = np.zeros(1024 * dims, dtype=np.uint32)
    b = np.zeros(1023 * dims, dtype=np.uint32)
    N.check(engine.mcg_rqmc_words(H.uptr(dirs), dims, W.SEED, 3, first, 1024, H.uptr(a)))
    N.check(engine.mcg_rqmc_words(H.uptr(dirs), dims, W.SEED, 3, first + 1, 1023, H.uptr(b)))
    assert np.array_equal(a.reshape(dims, 1024)[:, 1:], b.reshape(dims, 1023))


def test_american_put_at_a_quarter_million_paths(engine):
    spec, lsm = W.american_bs(dates=50, units=1 << 18, training_units=1 << 18)
    got = N.lsm_price(spec, lsm, stopping=True)
    want = H.oracle_lsm(spec, lsm, stopping=True, threads=THREADS)
    assert_same_result(spec, lsm, got, want)
