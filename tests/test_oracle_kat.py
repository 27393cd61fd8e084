"""Known-answer tests of the CPU oracle's sampling primitives.

Values are the reference's own unit-test vectors:
crates/pricing/src/engine/sampling/random.rs:290-356,
crates/pricing/src/engine/sampling/qmc.rs:377-482,
crates/pricing/src/engine/sampling/bridge.rs:482-580.
"""
import ctypes as C
import math

import numpy as np
import pytest

import helpers as H
from rust_pricing_b200 import sobol


def test_philox_random123_zero_vector(oracle):
    out = (C.c_uint32 * 4)()
    oracle.oracle_philox_block(0, (C.c_uint32 * 4)(0, 0, 0, 0), out)
    assert list(out) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_philox_lanes_follow_dimension(oracle):
    out = (C.c_uint32 * 4)()
    oracle.oracle_philox_block(17, (C.c_uint32 * 4)(29, 0, 0, 0), out)
    for d in range(4):
        assert oracle.oracle_philox_word(17, 29, d, 0) == out[d]
    # next block of dimensions: counter word 2 = dimension / 4, domain in word 3
    oracle.oracle_philox_block(17, (C.c_uint32 * 4)(9, 0, 1, 3), out)
    assert oracle.oracle_philox_word(17, 9, 4, 3) == out[0]


def test_domains_separate_streams(oracle):
    assert oracle.oracle_philox_word(42, 5, 7, 0) != oracle.oracle_philox_word(42, 5, 7, 1)


def test_open_unit_interval_midpoints(oracle):
    assert oracle.oracle_open_unit_interval(0) == 2.0 ** -33
    assert oracle.oracle_open_unit_interval(0xFFFFFFFF) == 1.0 - 2.0 ** -33


def test_as241_reference_quantiles(oracle):
    assert oracle.oracle_inverse_normal(0.5) == 0.0
    upper = oracle.oracle_inverse_normal(0.975)
    assert abs(upper - 1.959963984540054) < 2.0e-15
    assert abs(oracle.oracle_inverse_normal(1.0e-10) - -6.361340902404056) < 2.0e-15
    assert abs(upper + oracle.oracle_inverse_normal(0.025)) < 2.0e-15
    for bad in (0.0, 1.0, float("nan")):
        assert math.isnan(oracle.oracle_inverse_normal(bad))


def test_joe_kuo_first_three_dimensions(oracle):
    dirs = np.ascontiguousarray(sobol.direction_words(3))
    expected = [[0, 0, 0], [0x80000000] * 3, [0xC0000000, 0x40000000, 0x40000000],
                [0x40000000, 0xC0000000, 0xC0000000], [0x60000000, 0x60000000, 0xA0000000],
                [0xE0000000, 0xE0000000, 0x20000000], [0xA0000000, 0x20000000, 0xE0000000],
                [0x20000000, 0xA0000000, 0x60000000]]
    for point, row in enumerate(expected):
        for d in range(3):
            assert oracle.oracle_sobol_word(H.uptr(dirs[d]), point) == row[d]


def test_direction_table_matches_reference_digest():
    assert sobol.verify_full_table()


def test_scramble_abi_known_words(oracle):
    seed = 0x0123456789ABCDEF
    dirs = np.ascontiguousarray(sobol.direction_words(2))
    word = lambda s, p, d: oracle.oracle_rqmc_word(H.uptr(dirs[d]), seed, s, d, p)
    assert word(0, 0, 0) == 0x46C5FD35
    assert word(0, 1, 0) == 0xE684A5D7
    assert word(0, 2, 1) == 0x7D21CC82
    assert word(1, 2, 0) == 0xAA93E083
    assert word(2, 7, 1) == 0xC2B40C80


def test_lms_rows_unit_lower_triangular(oracle):
    shift = C.c_uint32()
    rows = (C.c_uint32 * 32)()
    oracle.oracle_scramble(123, 4, 7, C.byref(shift), rows)
    assert rows[0] == 0x80000000
    for r in range(32):
        diag = 1 << (31 - r)
        assert rows[r] & diag
        assert rows[r] & (diag - 1) == 0


def _bridge(oracle, times):
    t = np.ascontiguousarray(times, dtype=np.float64)
    n = len(t) - 1
    nodes = (C.c_uint32 * n)()
    ranks = (C.c_uint32 * n)()
    lw, rw, sd = (np.zeros(n) for _ in range(3))
    count = oracle.oracle_bridge_compile(H.dptr(t), len(t), nodes, ranks, H.dptr(lw), H.dptr(rw), H.dptr(sd))
    return count, list(nodes), list(ranks), lw, rw, sd


def test_bridge_uniform_order(oracle):
    count, nodes, ranks, *_ = _bridge(oracle, [0.0, 0.25, 0.5, 0.75, 1.0])
    assert count == 4 and nodes == [4, 2, 1, 3] and ranks == [0, 1, 2, 3]


def test_bridge_nonuniform_coefficients(oracle):
    count, nodes, _, lw, rw, sd = _bridge(oracle, [0.0, 0.1, 0.4, 1.0])
    assert nodes[:2] == [3, 2]
    assert lw[1] == 0.6 and rw[1] == 0.4 and sd[1] == math.sqrt(0.24)


def test_bridge_forward_known_values(oracle):
    t = np.array([0.0, 0.25, 0.5, 0.75, 1.0])
    z = np.array([1.0, 2.0, 3.0, 4.0])
    inc = np.zeros(4)
    oracle.oracle_bridge_apply(H.dptr(t), 5, H.dptr(z), H.dptr(inc))
    r = math.sqrt(0.125)
    expected = [2 * (0.75 + 3 * r), 2 * (0.75 - 3 * r), 2 * (-0.25 + 4 * r), 2 * (-0.25 - 4 * r)]
    assert np.max(np.abs(inc - expected)) < 2e-15


def test_bridge_reverse_is_transpose(oracle):
    t = np.array([0.0, 0.1, 0.4, 0.7, 1.0])
    z = np.array([0.3, -1.1, 0.7, 2.0])
    a = np.array([-0.2, 0.9, 1.3, -0.4])
    inc, back = np.zeros(4), np.zeros(4)
    oracle.oracle_bridge_apply(H.dptr(t), 5, H.dptr(z), H.dptr(inc))
    oracle.oracle_bridge_reverse(H.dptr(t), 5, H.dptr(a), H.dptr(back))
    assert abs(float(inc @ a) - float(z @ back)) < 2e-15


def test_bridge_rejects_invalid_grids(oracle):
    for times in ([0.0], [-0.0, 1.0], [0.0, 0.5, 0.5], [0.0, float("nan")]):
        assert _bridge(oracle, times)[0] == -1
