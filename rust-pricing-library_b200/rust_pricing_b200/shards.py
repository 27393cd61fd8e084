"""Scramble shards of one RQMC plan across ranks, and the merge of their
statistics.

`bench.py --gpus N` gives rank r the scrambles [S r, S r + S) of one plan
(`scramble_begin` of the descriptor); the paths are independent, so no
collective touches the data path.  After the timed region every rank's
per-product statistics of its scramble means travel to rank 0, which merges
them in rank order with the reference's own merges -- NeumaierSum::merged and
CenteredMoment::merged (Chan--Golub--LeVeque), fixed pairwise tree
(crates/pricing-numerics/src/reduction.rs:3-272) -- and forms the estimate as
estimate_from_statistics does (crates/pricing/src/engine/risk/report.rs:454-473).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

NORMAL_95 = 1.959_963_984_540_054


@dataclass
class Stat:
    """mcg_statistics: Neumaier (sum, correction), CGL (count, mean, m2)."""
    sum: float = 0.0
    correction: float = 0.0
    count: int = 0
    mean: float = 0.0
    m2: float = 0.0

    @staticmethod
    def of(s) -> "Stat":
        return Stat(s.sum, s.correction, int(s.count), s.mean, s.second_moment)


def _neumaier_add(total: float, corr: float, value: float):
    updated = total + value
    if abs(total) >= abs(value):
        corr += (total - updated) + value
    else:
        corr += (value - updated) + total
    return updated, corr


def merge(left: Stat, right: Stat) -> Stat:
    """NeumaierSum::merged and CenteredMoment::merged of two shards."""
    s, c = 0.0, 0.0
    for v in (left.sum, left.correction, right.sum, right.correction):
        s, c = _neumaier_add(s, c, v)
    if left.count == 0:
        return Stat(s, c, right.count, right.mean, right.m2)
    if right.count == 0:
        return Stat(s, c, left.count, left.mean, left.m2)
    n = left.count + right.count
    delta = right.mean - left.mean
    lw, rw, nf = float(left.count), float(right.count), float(n)
    mean = left.mean + delta * (rw / nf)
    between = delta * delta * (lw * rw / nf)
    return Stat(s, c, n, mean, (left.m2 + right.m2) + between)


def tree_merge(stats: list) -> Stat:
    """fixed_tree_reduce: pairwise levels in order, the odd tail carried."""
    level = list(stats)
    if not level:
        return Stat()
    while len(level) > 1:
        nxt = [merge(level[i], level[i + 1]) for i in range(0, len(level) - 1, 2)]
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0]


def estimate(s: Stat, units: int) -> dict:
    """estimate_from_statistics with scale 1: value, standard error, 95 % bounds."""
    inv = 1.0 / float(units)
    value = (s.sum + s.correction) * inv
    var = s.m2 / float(s.count - 1) if s.count > 1 else 0.0
    se = math.sqrt(var * inv)
    return {"value": value, "standard_error": se, "confidence_lower": value - NORMAL_95 * se,
            "confidence_upper": value + NORMAL_95 * se, "effective_sampling_units": units}


def gather_prices(buf, product_count: int, rank: int, world: int):
    """All ranks: send this rank's price statistics; rank 0 returns the merged
    estimate of every product over all ranks' scrambles (None elsewhere)."""
    import torch.distributed as dist
    mine = [Stat.of(buf.products[k].components[0]) for k in range(product_count)]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out = []
    for k in range(product_count):
        merged = tree_merge([g[k] for g in gathered])
        out.append(estimate(merged, merged.count))
    return out
