"""Builds `mcg_plan_desc` descriptors (include/mcg.h) from Python values.

A `PlanSpec` owns every array the descriptor points at, so the descriptor stays
valid for as long as the spec lives.  This is the data the reference keeps in
its compiled `SimulationPlan` (crates/pricing/src/engine/plan/simulation.rs:73-119):
market curves, model, observation times, products and the risk request.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi as A
from . import sobol


def _f64(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.float64))


def _ptr(array: Optional[np.ndarray], ctype=C.c_double):
    if array is None:
        return C.POINTER(ctype)()
    return array.ctypes.data_as(C.POINTER(ctype))


@dataclass
class ProductSpec:
    kind: int
    side: int = A.CALL
    strike: float = 100.0
    notional: float = 1.0
    digital_payout: int = A.DIGITAL_CASH
    payout: float = 1.0
    barrier_direction: int = A.BARRIER_DOWN
    barrier_style: int = A.KNOCK_OUT
    barrier: float = 0.0
    rebate: Optional[float] = None
    weights: Optional[Sequence[float]] = None
    initial_state: Optional[float] = None


@dataclass
class LocalVarianceSpec:
    time_nodes: Sequence[float]
    log_moneyness_nodes: Sequence[float]
    values: np.ndarray
    floor: float = 1e-8
    cap: float = 4.0


@dataclass
class SurfaceSpec:
    """An implied-variance surface (mcg_surface_desc): standard SSVI with a
    PCHIP theta curve and power-law or Heston-like phi
    (crates/pricing/src/market/ssvi.rs), or eSSVI slices
    (crates/pricing/src/market/essvi.rs)."""

    kind: int
    theta_times: Sequence[float] = ()
    theta_values: Sequence[float] = ()
    terminal_theta_slope: float = 0.0
    rho: float = 0.0
    eta: float = 0.0
    gamma: float = 0.0
    lam: float = 0.0
    slice_times: Sequence[float] = ()
    slice_thetas: Sequence[float] = ()
    slice_psis: Sequence[float] = ()
    slice_rho_psis: Sequence[float] = ()
    _keep: list = field(default_factory=list, repr=False)

    def desc(self) -> A.SurfaceDesc:
        keep = self._keep
        keep.clear()
        d = A.SurfaceDesc()
        d.kind = self.kind
        arrays = {}
        for name in ("theta_times", "theta_values", "slice_times", "slice_thetas", "slice_psis", "slice_rho_psis"):
            values = getattr(self, name)
            arrays[name] = _f64(values) if len(values) else None
            keep.append(arrays[name])
            setattr(d, name, _ptr(arrays[name]))
        d.theta_count = len(self.theta_times)
        d.slice_count = len(self.slice_times)
        d.terminal_theta_slope = self.terminal_theta_slope
        d.rho, d.eta, d.gamma, d.lambda_ = self.rho, self.eta, self.gamma, self.lam
        keep.append(d)
        return d


@dataclass
class PlanSpec:
    observation_times: Sequence[float]
    products: Sequence[ProductSpec]
    model: int = A.MODEL_BLACK_SCHOLES
    engine: int = A.ENGINE_PSEUDO
    precision: int = A.PRECISION_F64
    master_seed: int = 0x0123456789ABCDEF
    sampling_units: int = 1 << 14
    scramble_count: int = 16
    scramble_begin: int = 0
    antithetic: bool = False
    brownian_bridge: bool = False
    reduction_block_size: int = 4096
    spot: float = 100.0
    discount_times: Sequence[float] = (0.0, 1.0)
    discount_factors: Sequence[float] = (1.0, float(np.exp(-0.03)))
    dividend_times: Sequence[float] = (0.0, 1.0)
    dividend_factors: Sequence[float] = (1.0, float(np.exp(-0.01)))
    volatility: float = 0.2
    local_variance: Optional[LocalVarianceSpec] = None
    payment_time: Optional[float] = None
    request_delta: bool = False
    request_gamma: bool = False
    request_vega: bool = False
    request_local_vega_nodes: bool = False
    gamma_bump_relative: bool = True
    gamma_bump: float = 0.01
    smoothing_half_width: float = 0.0
    checkpoint_interval: int = 16
    # Discrete dividends of the escrowed affine model: (ex-time, fixed cash, proportional fraction)
    dividends: Sequence[tuple] = ()
    _keep: list = field(default_factory=list, repr=False)

    def steps(self) -> int:
        return len(self.observation_times)

    def desc(self) -> A.PlanDesc:
        keep = self._keep
        keep.clear()
        d = A.PlanDesc()
        d.abi_version = A.ABI_VERSION
        d.model = self.model
        d.engine = self.engine
        d.precision = self.precision
        d.master_seed = self.master_seed & 0xFFFFFFFFFFFFFFFF
        d.sampling_units = self.sampling_units
        d.scramble_count = self.scramble_count
        d.scramble_begin = self.scramble_begin
        d.antithetic = int(self.antithetic)
        d.brownian_bridge = int(self.brownian_bridge)
        d.reduction_block_size = self.reduction_block_size
        if self.engine == A.ENGINE_RQMC:
            dims = self._dimension_hint()
            words = np.ascontiguousarray(sobol.direction_words(dims))
            keep.append(words)
            d.sobol_dimension_count = dims
            d.sobol_directions = _ptr(words, C.c_uint32)
        d.spot = self.spot
        for name, times, factors in (("discount_curve", self.discount_times, self.discount_factors),
                                     ("dividend_curve", self.dividend_times, self.dividend_factors)):
            t, f = _f64(times), _f64(factors)
            keep += [t, f]
            curve = A.Curve(len(t), _ptr(t), _ptr(f))
            setattr(d, name, curve)
        d.volatility = self.volatility
        if self.local_variance is not None:
            g = self.local_variance
            t, x, v = _f64(g.time_nodes), _f64(g.log_moneyness_nodes), _f64(g.values).ravel()
            keep += [t, x, v]
            d.local_variance = A.LocalVarianceGrid(len(t), len(x), _ptr(t), _ptr(x), _ptr(v),
                                                   g.floor, g.cap)
        obs = _f64(self.observation_times)
        keep.append(obs)
        d.observation_count = len(obs)
        d.observation_times = _ptr(obs)
        d.payment_time = float(obs[-1] if self.payment_time is None else self.payment_time)
        products = (A.ProductDesc * len(self.products))()
        for i, p in enumerate(self.products):
            q = products[i]
            q.kind, q.side, q.strike, q.notional = p.kind, p.side, p.strike, p.notional
            q.digital_payout, q.payout = p.digital_payout, p.payout
            q.barrier_direction, q.barrier_style = p.barrier_direction, p.barrier_style
            q.barrier = p.barrier
            q.has_rebate = int(p.rebate is not None)
            q.rebate = 0.0 if p.rebate is None else p.rebate
            if p.weights is not None:
                w = _f64(p.weights)
                keep.append(w)
                q.observation_weights = _ptr(w)
            q.has_initial_state = int(p.initial_state is not None)
            q.initial_state = 0.0 if p.initial_state is None else p.initial_state
        keep.append(products)
        d.product_count = len(self.products)
        d.products = C.cast(products, C.POINTER(A.ProductDesc))
        d.request_delta = int(self.request_delta)
        d.request_gamma = int(self.request_gamma)
        d.request_vega = int(self.request_vega)
        d.request_local_vega_nodes = int(self.request_local_vega_nodes)
        d.gamma_bump_relative = int(self.gamma_bump_relative)
        d.gamma_bump = self.gamma_bump
        d.smoothing_half_width = self.smoothing_half_width
        d.checkpoint_interval = self.checkpoint_interval
        if self.dividends:
            ex, cash, beta = (_f64([float(x[i]) for x in self.dividends]) for i in range(3))
            keep += [ex, cash, beta]
            d.discrete_dividends = A.Dividends(len(ex), _ptr(ex), _ptr(cash), _ptr(beta))
        keep.append(d)
        return d

    def _dimension_hint(self) -> int:
        """Sobol dimensions the plan may need (time steps, including substeps)."""
        if self.model == A.MODEL_LOCAL_VOLATILITY and self.local_variance is not None:
            union = np.union1d(np.asarray(self.local_variance.time_nodes, dtype=np.float64),
                               np.asarray(self.observation_times, dtype=np.float64))
            ex = [float(d[0]) for d in self.dividends if float(d[0]) <= float(self.observation_times[-1])]
            if ex:
                union = np.union1d(union, np.asarray(ex, dtype=np.float64))
            gaps = np.diff(np.asarray(self.local_variance.time_nodes, dtype=np.float64))
            step = float(gaps.max())
            count = int(np.sum(np.maximum(1, np.ceil(np.diff(np.concatenate([[0.0], union])) / step))))
            return min(max(count + 8, 1), sobol.DIMENSIONS)
        return min(len(self.observation_times), sobol.DIMENSIONS)

    def grid_value_count(self) -> int:
        if self.local_variance is None:
            return 0
        return len(self.local_variance.time_nodes) * len(self.local_variance.log_moneyness_nodes)


@dataclass
class LsmSpec:
    """The reference's LsmConfig for one spot state variable
    (crates/pricing/src/engine/mc/lsm.rs:328-495): polynomial degree, CPQR rank
    tolerances, ITM tolerance, matrix-size limit, and the training engine (of
    the valuation plan's kind)."""

    training_seed: int
    training_units: int
    training_scramble_count: int = 0
    training_antithetic: bool = False
    training_brownian_bridge: bool = False
    max_degree: int = 3
    itm_abs_tolerance: float = 0.0
    cpqr_abs_tolerance: float = 1e-14
    cpqr_rel_tolerance: float = 1e-12
    max_matrix_elements: int = 1_000_000
    continuation: int = A.CONTINUATION_POLYNOMIAL
    mlp_epochs: int = 0
    mlp_batch: int = 0
    mlp_learning_rate: float = 0.0
    mlp_seed: int = 0
    _keep: list = field(default_factory=list, repr=False)

    def desc(self) -> A.LsmDesc:
        d = A.LsmDesc()
        d.max_degree = self.max_degree
        d.itm_abs_tolerance = self.itm_abs_tolerance
        d.cpqr_abs_tolerance = self.cpqr_abs_tolerance
        d.cpqr_rel_tolerance = self.cpqr_rel_tolerance
        d.max_matrix_elements = self.max_matrix_elements
        d.training_seed = self.training_seed & 0xFFFFFFFFFFFFFFFF
        d.training_units = self.training_units
        d.training_scramble_count = self.training_scramble_count
        d.training_antithetic = int(self.training_antithetic)
        d.training_brownian_bridge = int(self.training_brownian_bridge)
        d.continuation = self.continuation
        d.mlp_epochs = self.mlp_epochs
        d.mlp_batch = self.mlp_batch
        d.mlp_learning_rate = self.mlp_learning_rate
        d.mlp_seed = self.mlp_seed & 0xFFFFFFFFFFFFFFFF
        self._keep[:] = [d]
        return d


@dataclass
class AssetSpec:
    """One asset of a multi-asset plan: Black--Scholes (volatility) or local
    volatility (its own variance grid), its spot and dividend-yield curve."""

    spot: float = 100.0
    volatility: float = 0.2
    model: int = A.MODEL_BLACK_SCHOLES
    local_variance: Optional[LocalVarianceSpec] = None
    dividend_times: Sequence[float] = (0.0, 1.0)
    dividend_factors: Sequence[float] = (1.0, 1.0)


@dataclass
class MultiAssetSpec:
    """mcg_multi_asset_desc: correlated assets, a correlation term structure
    (matrices in force from their times), the common time grid's maximum step,
    the engine and a basket or worst-of option."""

    assets: Sequence[AssetSpec]
    correlations: Sequence  # list of (time, n x n matrix)
    expiry: float = 1.0
    payment_time: Optional[float] = None
    maximum_step: float = 0.25
    product: int = A.MULTI_BASKET
    side: int = A.CALL
    strike: float = 100.0
    notional: float = 1.0
    weights: Optional[Sequence[float]] = None
    scales: Optional[Sequence[float]] = None
    smoothing_half_width: float = 0.0
    engine: int = A.ENGINE_PSEUDO
    master_seed: int = 511
    sampling_units: int = 4096
    scramble_count: int = 8
    antithetic: bool = True
    brownian_bridge: bool = True
    reduction_block_size: int = 256
    discount_times: Sequence[float] = (0.0, 2.0)
    discount_factors: Sequence[float] = (1.0, float(np.exp(-0.06)))
    _keep: list = field(default_factory=list, repr=False)

    def desc(self) -> A.MultiAssetDesc:
        keep = self._keep
        keep.clear()
        n = len(self.assets)
        d = A.MultiAssetDesc()
        d.abi_version = A.ABI_VERSION
        d.asset_count = n
        arr = (A.AssetDesc * n)()
        for i, a in enumerate(self.assets):
            q = arr[i]
            q.model, q.spot, q.volatility = a.model, a.spot, a.volatility
            t, f = _f64(a.dividend_times), _f64(a.dividend_factors)
            keep += [t, f]
            q.dividend_curve = A.Curve(len(t), _ptr(t), _ptr(f))
            if a.local_variance is not None:
                g = a.local_variance
                gt, gx, gv = _f64(g.time_nodes), _f64(g.log_moneyness_nodes), _f64(g.values).ravel()
                keep += [gt, gx, gv]
                q.local_variance = A.LocalVarianceGrid(len(gt), len(gx), _ptr(gt), _ptr(gx), _ptr(gv), g.floor, g.cap)
        keep.append(arr)
        d.assets = C.cast(arr, C.POINTER(A.AssetDesc))
        t, f = _f64(self.discount_times), _f64(self.discount_factors)
        keep += [t, f]
        d.discount_curve = A.Curve(len(t), _ptr(t), _ptr(f))
        ct = _f64([c[0] for c in self.correlations])
        cm = _f64([np.asarray(c[1], dtype=np.float64).ravel() for c in self.correlations]).ravel()
        keep += [ct, cm]
        d.correlation_count = len(ct)
        d.correlation_times = _ptr(ct)
        d.correlations = _ptr(cm)
        d.maximum_step = self.maximum_step
        d.expiry = self.expiry
        d.payment_time = self.expiry if self.payment_time is None else self.payment_time
        d.engine = self.engine
        d.master_seed = self.master_seed & 0xFFFFFFFFFFFFFFFF
        d.sampling_units = self.sampling_units
        d.scramble_count = self.scramble_count
        d.antithetic = int(self.antithetic)
        d.brownian_bridge = int(self.brownian_bridge)
        d.reduction_block_size = self.reduction_block_size
        if self.engine == A.ENGINE_RQMC:
            dims = min(sobol.DIMENSIONS, n * self.step_hint())
            words = np.ascontiguousarray(sobol.direction_words(dims))
            keep.append(words)
            d.sobol_dimension_count = dims
            d.sobol_directions = _ptr(words, C.c_uint32)
        d.product, d.side, d.strike, d.notional = self.product, self.side, self.strike, self.notional
        w = _f64(self.weights if self.weights is not None else [1.0 / n] * n)
        sc = _f64(self.scales if self.scales is not None else [1.0] * n)
        keep += [w, sc]
        d.weights, d.scales = _ptr(w), _ptr(sc)
        d.smoothing_half_width = self.smoothing_half_width
        keep.append(d)
        return d

    def step_hint(self) -> int:
        """An upper bound of the common time grid's steps."""
        events = {0.0, float(self.expiry)}
        events |= {float(c[0]) for c in self.correlations if 0.0 < float(c[0]) < self.expiry}
        for a in self.assets:
            if a.local_variance is not None:
                events |= {float(t) for t in a.local_variance.time_nodes if float(t) <= self.expiry}
        ev = sorted(events)
        return int(sum(max(1, int(np.ceil((b - a) / self.maximum_step))) for a, b in zip(ev, ev[1:]))) + 4
