"""Scramble shards of one RQMC plan across ranks, and the merge of their
statistics.

`bench.py --gpus N` gives rank r the scrambles [S r, S r + S) of one plan
(`scramble_begin` of the descriptor); the paths are independent, so no
collective touches the data path.  After the timed region every rank sends
rank 0 its scrambles' means (the RQMC replicates, `replicate_means` of the
result), rank 0 joins them in scramble order and runs the reference's
replicate two-pass over all of them -- NeumaierSum over the replicates, then
CenteredMoment::from_ordered_values_two_pass
(crates/pricing/src/engine/risk/valuation.rs:349-361,
crates/pricing-numerics/src/reduction.rs:3-122) -- the same operations, in the
same order, as one evaluation of every scramble, so the merged estimate equals
the single-GPU one bit for bit; the estimate is formed as
estimate_from_statistics does (crates/pricing/src/engine/risk/report.rs:454-473).
`merge` / `tree_merge` are the reference's NeumaierSum::merged and
CenteredMoment::merged (Chan--Golub--LeVeque) with its fixed pairwise tree,
for records that are not replicates (reduction.rs:123-272).
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


def two_pass(values: list) -> Stat:
    """NeumaierSum over the replicates in order, then the centred second
    moment about their mean (from_ordered_values_two_pass): the engine's and
    the oracle's RQMC statistics, operation for operation."""
    if not values:
        return Stat()
    s, c = 0.0, 0.0
    for v in values:
        s, c = _neumaier_add(s, c, v)
    mean = (s + c) / float(len(values))
    qs, qc = 0.0, 0.0
    for v in values:
        d = v - mean
        qs, qc = _neumaier_add(qs, qc, d * d)
    return Stat(s, c, len(values), mean, qs + qc)


def estimate(s: Stat, units: int) -> dict:
    """estimate_from_statistics with scale 1: value, standard error, 95 % bounds."""
    inv = 1.0 / float(units)
    value = (s.sum + s.correction) * inv
    var = s.m2 / float(s.count - 1) if s.count > 1 else 0.0
    se = math.sqrt(var * inv)
    return {"value": value, "standard_error": se, "confidence_lower": value - NORMAL_95 * se,
            "confidence_upper": value + NORMAL_95 * se, "effective_sampling_units": units}


def gather_prices(buf, product_count: int, rank: int, world: int):
    """All ranks: send this rank's scramble means of every product's price;
    rank 0 returns the estimate of every product over all ranks' scrambles
    (None elsewhere)."""
    import torch.distributed as dist
    mine = [buf.replicate_means(k) for k in range(product_count)]
    if any(not m for m in mine):
        raise ValueError("the shard merge needs the RQMC scramble means (replicate_means) of every product")
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out = []
    for k in range(product_count):
        reps = [v for g in gathered for v in g[k]]  # rank order = scramble order
        merged = two_pass(reps)
        out.append(estimate(merged, merged.count))
    return out
