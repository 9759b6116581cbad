"""Model and product set-up for the LMM pipeline (host side, numpy).

Builds everything the C ABI consumes as small inputs: accruals, initial
curve, displacements, pseudo-roots (through lmm_abcd_pseudo_roots /
lmm_flat_pseudo_roots), fixed drifts, Sobol direction numbers, scrambler
words and the per-exercise-date Longstaff–Schwartz basis tables.

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
* ``c4`` differentiation form: the c3 model (10 factors) with the Bermudan
  plus a 5% cap strip, 2^20 paths.
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

import ctypes
import os
from dataclasses import dataclass, field, replace
from pathlib import Path

import numpy as np

from ._lib import call

_VP = ctypes.c_void_p


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return _VP(a.ctypes.data)


PRODUCTS = {"swaption": 0, "cancellable": 1, "european": 2, "tarn": 3}


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
                     beta=0.1, product="swaption", strike=0.05, basis="cross",
                     notes={"factors": "10, taken from the c3 form"})
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


# ---------------------------------------------------------------------------
# LS basis tables.  Variables per date: v0 = first forward, v1 = swap rate,
# v2 = annuity (see lmm_pipeline.h).  Tables list monomial exponents.
# ---------------------------------------------------------------------------
def n_variables(step: int, n: int) -> int:
    """actualNumberOfVariables (gold/LS_basis_examples_gold.h:50-60)."""
    if step + 3 <= n:
        return 3
    if step + 2 == n:
        return 2
    if step + 1 == n:
        return 1
    return 0


def _cross(V: int) -> list[tuple]:
    """quadraticPolynomialCrossGenerator order (gold/LS_regression.h:166-240)."""
    z = [0, 0, 0]

    def m(**kw):
        e = list(z)
        for k, v in kw.items():
            e[int(k[1])] += v
        return tuple(e)

    if V == 0:
        return [tuple(z)]
    if V == 1:
        return [tuple(z), m(x0=1), m(x0=2)]
    if V == 2:
        return [tuple(z), m(x0=1), m(x1=1), m(x0=2), (1, 1, 0), m(x1=2)]
    out = [tuple(z)] + [m(**{f"x{i}": 1}) for i in range(V)]
    for i in range(V):
        k = (i + 1) % V
        e = [0, 0, 0]
        e[i] += 1
        e[k] += 1
        out.append(tuple(e))
    out += [m(**{f"x{i}": 2}) for i in range(V)]
    return out


def _quadratic(V: int) -> list[tuple]:
    """quadraticPolynomialGenerator order (gold/LS_regression.h:123-160)."""
    out = [(0, 0, 0)]
    for i in range(V):
        e1 = [0, 0, 0]
        e1[i] = 1
        e2 = [0, 0, 0]
        e2[i] = 2
        out += [tuple(e1), tuple(e2)]
    return out


BASIS_C2 = [(0, 0, 0), (0, 1, 0), (0, 2, 0), (1, 0, 0), (0, 0, 1), (1, 1, 0)]
BASIS_C5 = _cross(3) + [(1, 1, 1), (0, 3, 0)]


def basis_tables(kind: str, nvars: np.ndarray):
    """(monomials [E][16][3] uint8, nbasis [E] int32) for every date."""
    E = len(nvars)
    mono = np.zeros((E, 16, 3), np.uint8)
    nb = np.zeros(E, np.int32)
    for e, V in enumerate(nvars):
        if kind == "cross":
            lst = _cross(int(V))
        elif kind == "quadratic":
            lst = _quadratic(int(V))
        elif kind in ("c2", "c5"):
            full = BASIS_C2 if kind == "c2" else BASIS_C5
            lst = [m for m in full if all(m[j] == 0 for j in range(int(V), 3))]
        else:
            raise ValueError(f"unknown basis {kind!r}")
        mono[e, : len(lst)] = np.array(lst, np.uint8)
        nb[e] = len(lst)
    return mono, nb


# ---------------------------------------------------------------------------
# Sobol direction numbers
# ---------------------------------------------------------------------------
def joe_kuo_table(dims: int):
    """Primitive polynomials and initial direction integers of the published
    Joe–Kuo table shipped with scipy (new-joe-kuo-6.21201)."""
    import scipy

    path = Path(os.path.dirname(scipy.__file__)) / "stats" / "_sobol_direction_numbers.npz"
    z = np.load(path)
    poly = z["poly"][:dims].astype(np.int64)
    vinit = z["vinit"][:dims].astype(np.uint32)
    if poly.size < dims:
        raise ValueError(f"table has only {poly.size} dimensions")
    deg = np.array([int(p).bit_length() - 1 for p in poly], np.uint32)
    a = np.array([(int(p) >> 1) & ((1 << max(int(p).bit_length() - 2, 0)) - 1) for p in poly], np.uint32)
    return deg, a, np.ascontiguousarray(vinit)


def sobol_directions(dims: int) -> np.ndarray:
    deg, a, m = joe_kuo_table(dims)
    out = np.zeros((dims, 32), np.uint32)
    call("lmm_sobol_directions", dims, _p(deg), _p(a), _p(m), m.shape[1], _p(out))
    return out


def scramblers(seed: int, dims: int) -> np.ndarray:
    out = np.zeros(dims, np.uint32)
    call("lmm_mt19937_words", seed, dims, _p(out))
    return out


# ---------------------------------------------------------------------------
# Market bundle
# ---------------------------------------------------------------------------
@dataclass
class Market:
    cfg: Config
    taus: np.ndarray
    disp: np.ndarray
    f0: np.ndarray
    rate_times: np.ndarray
    A64: np.ndarray
    A: np.ndarray
    fixed: np.ndarray
    directions: np.ndarray
    scramblers: np.ndarray
    scramble_dims: int
    ex_steps: np.ndarray
    nvars: np.ndarray
    mono: np.ndarray
    nbasis: np.ndarray

    @property
    def initial_numeraire(self) -> float:
        """P(0, T_0) = 1 / (1 + f_0 T_0)."""
        return 1.0 / (1.0 + float(self.f0[0]) * float(self.rate_times[0]))


def pseudo_roots(cfg: Config, rate_times: np.ndarray) -> np.ndarray:
    n, F = cfg.n, cfg.F
    resets = np.ascontiguousarray(rate_times[:n].astype(np.float64))
    evol = resets.copy()
    out = np.zeros((n, n, F), np.float64)
    if cfg.vol == "abcd":
        a, b, c, d = cfg.abcd
        mult = np.ones(n)
        call("lmm_abcd_pseudo_roots", a, b, c, d, _p(evol), n, _p(resets), n, _p(mult), F,
             cfg.L, cfg.beta, _p(out))
    else:
        vols = np.full(n, cfg.sigma)
        call("lmm_flat_pseudo_roots", _p(resets), n, _p(evol), n, _p(vols), F, cfg.L,
             cfg.beta, _p(out))
    return out


def build_market(cfg: Config, directions: np.ndarray | None = None,
                 scramble_all: bool = True) -> Market:
    n, F = cfg.n, cfg.F
    taus = np.full(n, cfg.tau, np.float32)
    disp = np.full(n, cfg.disp, np.float32)
    f0 = np.ascontiguousarray(cfg.f0.astype(np.float32))
    rate_times = cfg.tau * (np.arange(n + 1) + 1.0)
    A64 = pseudo_roots(cfg, rate_times)
    A = np.ascontiguousarray(A64.astype(np.float32))
    fixed = np.zeros((n, n), np.float32)
    call("lmm_fixed_drifts", _p(A), n, n, F, _p(fixed))
    D = n * F
    dirs = sobol_directions(D) if directions is None else np.ascontiguousarray(directions[:D])
    scr = scramblers(cfg.scramble_seed, D)
    if cfg.product in ("european", "tarn"):
        ex_steps = np.zeros(0, np.int32)
    else:
        ex_steps = np.arange(n, dtype=np.int32)
    nvars = np.array([n_variables(int(s), n) for s in ex_steps], np.int32)
    mono, nb = basis_tables(cfg.basis, nvars) if len(ex_steps) else (
        np.zeros((0, 16, 3), np.uint8), np.zeros(0, np.int32))
    return Market(cfg, taus, disp, f0, rate_times, A64, A, fixed, dirs, scr,
                  D if scramble_all else n, ex_steps, nvars, mono, nb)
