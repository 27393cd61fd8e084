"""Closed-form Black--Scholes with continuous yields: the analytic benchmark.

Restates the forward Black--Scholes formula of
crates/pricing/src/engine/analytic/closed_form.rs:191-223 (price, spot Delta,
spot Gamma, unit-volatility Vega) for the statistical acceptance tests.
"""
import math


def ndtr(x: float) -> float:
    return 0.5 * math.erfc(-x / math.sqrt(2.0))


def npdf(x: float) -> float:
    return math.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def black_scholes(call: bool, spot: float, strike: float, t: float, rate: float, dividend: float,
                  vol: float) -> dict:
    df = math.exp(-rate * t)
    qf = math.exp(-dividend * t)
    forward = spot * qf / df
    sd = vol * math.sqrt(t)
    d1 = (math.log(forward / strike) + 0.5 * sd * sd) / sd
    d2 = d1 - sd
    if call:
        price = df * (forward * ndtr(d1) - strike * ndtr(d2))
        delta = qf * ndtr(d1)
    else:
        price = df * (strike * ndtr(-d2) - forward * ndtr(-d1))
        delta = -qf * ndtr(-d1)
    gamma = qf * npdf(d1) / (spot * sd)
    vega = spot * qf * npdf(d1) * math.sqrt(t)
    return {"price": price, "delta": delta, "gamma": gamma, "vega": vega}
