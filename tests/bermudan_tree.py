"""Cox--Ross--Rubinstein binomial tree for Bermudan and American options.

The independent benchmark of the early-exercise prices: a recombining tree with
`steps` steps over the horizon, exercise allowed at the tree steps that fall
on the exercise dates (every steps / dates steps for equally spaced dates).
Backward induction in numpy, O(steps^2) node updates (25e6 for 5000 steps).
"""
import math

import numpy as np


def bermudan_binomial(spot: float, strike: float, rate: float, dividend: float, vol: float, horizon: float,
                      steps: int, exercise_steps, put: bool = True) -> float:
    dt = horizon / steps
    up = math.exp(vol * math.sqrt(dt))
    down = 1.0 / up
    growth = math.exp((rate - dividend) * dt)
    p = (growth - down) / (up - down)
    disc = math.exp(-rate * dt)
    exercise = set(int(s) for s in exercise_steps)
    j = np.arange(steps + 1, dtype=np.float64)
    s = spot * up ** (steps - j) * down ** j
    v = np.maximum(strike - s, 0.0) if put else np.maximum(s - strike, 0.0)
    for n in range(steps - 1, -1, -1):
        v = disc * (p * v[:-1] + (1.0 - p) * v[1:])
        if n in exercise and n > 0:
            jn = np.arange(n + 1, dtype=np.float64)
            sn = spot * up ** (n - jn) * down ** jn
            v = np.maximum(v, np.maximum(strike - sn, 0.0) if put else np.maximum(sn - strike, 0.0))
    return float(v[0])


def bermudan_equally_spaced(spot, strike, rate, dividend, vol, horizon, dates, steps=5000, put=True):
    per = steps // dates
    assert per * dates == steps, "tree steps must be a multiple of the exercise dates"
    return bermudan_binomial(spot, strike, rate, dividend, vol, horizon, steps,
                             [per * k for k in range(1, dates + 1)], put)
