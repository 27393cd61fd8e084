"""Scramble shards across ranks: two gloo ranks on the CPU each run the oracle
on their own scrambles of one RQMC plan (scramble_begin = S r) and gather their
scramble means to rank 0, whose two-pass over all 2 S of them equals the
single-process evaluation of all 2 S scrambles bit for bit (value, standard
error and bounds)."""
import multiprocessing as mp
import os
import socket

import pytest

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import shards
from rust_pricing_b200.desc import PlanSpec, ProductSpec

SCRAMBLES = 4


def spec(scramble_begin=0, scrambles=SCRAMBLES):
    times = [(i + 1) / 12 for i in range(12)]
    return PlanSpec(observation_times=times,
                    products=[ProductSpec(kind=A.PRODUCT_ASIAN, strike=100.0, weights=[1.0 / 12] * 12),
                              ProductSpec(kind=A.PRODUCT_DISCRETE_BARRIER, strike=100.0, barrier=85.0,
                                          barrier_direction=A.BARRIER_DOWN, barrier_style=A.KNOCK_OUT,
                                          rebate=1.0)],
                    engine=A.ENGINE_RQMC, master_seed=0x5EED, sampling_units=1024, scramble_count=scrambles,
                    scramble_begin=scramble_begin, brownian_bridge=False)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    buf = H.oracle_evaluate(spec(scramble_begin=rank * SCRAMBLES), threads=2)
    merged = shards.gather_prices(buf, 2, rank, world)
    if rank == 0:
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_scramble_shards_merge_to_the_whole_plan():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    merged = out.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    whole = H.oracle_evaluate(spec(scrambles=2 * SCRAMBLES), threads=4)
    for k in range(2):
        want = whole.products[k].price
        got = merged[k]
        assert got["effective_sampling_units"] == 2 * SCRAMBLES
        assert got["value"] == want.value
        assert got["standard_error"] == want.standard_error
        assert (got["confidence_lower"], got["confidence_upper"]) == (want.confidence_lower,
                                                                      want.confidence_upper)
        c = whole.products[k].components[A.PRICE]
        reps = whole.replicate_means(k)
        st = shards.two_pass(reps)
        assert (st.sum, st.correction, st.count, st.mean, st.m2) == (c.sum, c.correction, c.count, c.mean,
                                                                     c.second_moment)


def test_merge_is_the_reference_merge():
    """CenteredMoment::merged of two halves equals one pass over the whole (to rounding)."""
    import random
    rnd = random.Random(7)
    vals = [rnd.gauss(0, 1) for _ in range(101)]

    def one_pass(vs):
        s, c, n, mean, m2 = 0.0, 0.0, 0, 0.0, 0.0
        for v in vs:
            s, c = shards._neumaier_add(s, c, v)
            n += 1
            d = v - mean
            mean = mean + d / n
            m2 += d * (v - mean)
        return shards.Stat(s, c, n, mean, m2)

    parts = [one_pass(vals[i:i + 10]) for i in range(0, 101, 10)]
    whole, merged = one_pass(vals), shards.tree_merge(parts)
    assert merged.count == whole.count
    assert abs((merged.sum + merged.correction) - (whole.sum + whole.correction)) < 1e-13
    assert abs(merged.m2 - whole.m2) < 1e-12 * whole.m2
