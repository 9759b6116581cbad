"""Benchmark configurations of the LMM pricing path (pure Python: numpy and
the standard library only, so a caller can read them without loading the
CUDA library).

The benchmark configurations are those of the reference's LMM pricing
path, restated with seeded synthetic inputs:

* ``c1`` European: 20 semi-annual forwards at 5%, zero displacement, flat
  20% vol, rho = exp(-0.05|dT|), 3 factors, 16,384 paths; caplet strip and
  payer swap struck at 5%.
* ``c2`` Bermudan payer swaption: 40 semi-annual forwards 4%..6%,
  displacement 0.015, abcd (0.05, 0.09, 0.44, 0.11), rho = exp(-0.1|dT|),
  5 factors, 262,144 pricing + 65,536 regression paths, strike 5%, basis
  {1, S, S^2, f1, A, S f1}.
* ``c3`` precision form: 80 quarterly forwards, seeded smooth quadratic
  curve in [3%, 6%], same abcd vol, 10 factors, 2^20 paths, full quadratic
  basis with cross terms (10 functions).
* ``c4`` differentiation form: the c3 model (10 factors, the form's factor
  count is not stated and is taken from c3) with a portfolio of the
  Bermudan payer swaption struck at 5% and a cap strip struck at 5% (a
  caplet on every period, paid whatever the swaption's exercise), 2^20
  paths.
* ``c5`` large form: 120 quarterly forwards, displacement 0.02,
  rho = exp(-0.08|dT|), 15 factors, 2^21 paths, cancellable payer swap,
  12 basis functions.
* ``t1`` target redemption note on the c1 market: the reference's TARN
  test note (total coupon 0.15, strike 0.10, multiplier 2).

The first reset is one accrual period after today (T_0 = tau), evolution
times are the resets T_0..T_{n-1}, and the value at time 0 of one unit of
the T_0 numeraire is P(0, T_0) = 1 / (1 + f_0 T_0).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

PRODUCTS = {"swaption": 0, "cancellable": 1, "european": 2, "tarn": 3, "bermudan_cap": 4}


@dataclass
class Config:
    name: str
    n: int
    tau: float
    F: int
    paths: int
    reg_paths: int
    f0: np.ndarray
    disp: float
    vol: str  # "flat" or "abcd"
    sigma: float = 0.2
    abcd: tuple = (0.05, 0.09, 0.44, 0.11)
    beta: float = 0.1
    L: float = 0.0
    product: str = "swaption"
    strike: float = 0.05
    cap_strike: float = 0.05
    pay_receive: float = 1.0
    basis: str = "cross"
    normalise: bool = True
    scramble_seed: int = 1
    cutoff: float = 10.0
    tarn_total: float = 0.15        # TARN: total coupon
    tarn_multiplier: float = 2.0    # TARN: inverse-floater multiplier
    notes: dict = field(default_factory=dict)

    @property
    def steps(self) -> int:
        return self.n

    @property
    def dims(self) -> int:
        return self.n * self.F


def quadratic_curve(n: int, tau: float, seed: int, lo: float = 0.03, hi: float = 0.06) -> np.ndarray:
    """Seeded smooth initial curve: the quadratic in maturity through three
    uniform draws in [lo, hi] at the first, middle and last reset, clipped
    to [lo, hi]."""
    rng = np.random.default_rng(seed)
    y = rng.uniform(lo, hi, 3)
    t = tau * (np.arange(n) + 1.0)
    x = np.array([t[0], t[n // 2], t[-1]])
    c = np.polyfit(x, y, 2)
    return np.clip(np.polyval(c, t), lo, hi).astype(np.float32)


CURVE_SEED = 2024


def make_config(name: str, **overrides) -> Config:
    name = name.lower()
    if name == "c1":
        cfg = Config("c1", n=20, tau=0.5, F=3, paths=16384, reg_paths=0,
                     f0=np.full(20, 0.05, np.float32), disp=0.0, vol="flat", sigma=0.2,
                     beta=0.05, product="european", strike=0.05, cap_strike=0.05)
    elif name == "c2":
        cfg = Config("c2", n=40, tau=0.5, F=5, paths=262144, reg_paths=65536,
                     f0=np.linspace(0.04, 0.06, 40).astype(np.float32), disp=0.015,
                     vol="abcd", beta=0.1, product="swaption", strike=0.05, basis="c2")
    elif name == "c3":
        cfg = Config("c3", n=80, tau=0.25, F=10, paths=1 << 20, reg_paths=1 << 20,
                     f0=quadratic_curve(80, 0.25, CURVE_SEED), disp=0.015, vol="abcd",
                     beta=0.1, product="swaption", strike=0.05, basis="cross")
    elif name == "c4":
        cfg = Config("c4", n=80, tau=0.25, F=10, paths=1 << 20, reg_paths=1 << 20,
                     f0=quadratic_curve(80, 0.25, CURVE_SEED), disp=0.015, vol="abcd",
                     beta=0.1, product="bermudan_cap", strike=0.05, cap_strike=0.05,
                     basis="cross", notes={"factors": "10, taken from the c3 form"})
    elif name == "c5":
        cfg = Config("c5", n=120, tau=0.25, F=15, paths=1 << 21, reg_paths=1 << 21,
                     f0=quadratic_curve(120, 0.25, CURVE_SEED), disp=0.02, vol="abcd",
                     beta=0.08, product="cancellable", strike=0.05, basis="c5")
    elif name == "t1":
        # the reference's TARN test note (LMM_evolver_test.cu:1404-1412: total
        # coupon 0.15, strike 0.10, multiplier 2, half-year accruals) on the C1
        # market
        cfg = Config("t1", n=20, tau=0.5, F=3, paths=16384, reg_paths=0,
                     f0=np.full(20, 0.05, np.float32), disp=0.0, vol="flat", sigma=0.2,
                     beta=0.05, product="tarn", strike=0.10, tarn_total=0.15,
                     tarn_multiplier=2.0)
    else:
        raise ValueError(f"unknown configuration {name!r}")
    return replace(cfg, **overrides) if overrides else cfg
