"""Model and product set-up for the LMM pipeline (host side, numpy).

Builds everything the C ABI consumes as small inputs: accruals, initial
curve, displacements, pseudo-roots (through lmm_abcd_pseudo_roots /
lmm_flat_pseudo_roots), fixed drifts, Sobol direction numbers, scrambler
words and the per-exercise-date Longstaff–Schwartz basis tables, for the
benchmark configurations of ``configs``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from ._lib import call
from .configs import CURVE_SEED, PRODUCTS, Config, make_config, quadratic_curve  # noqa: F401

_VP = ctypes.c_void_p


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return _VP(a.ctypes.data)



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
SOBOL_TABLE = "joe-kuo-6.10200"
_TABLE_10200 = Path(__file__).resolve().parent / "data" / "joe_kuo_6_10200.npz"


def joe_kuo_table(dims: int, table: str = SOBOL_TABLE):
    """(degree, interior coefficient bits, initial direction integers) of the
    first `dims` dimensions of a published Joe–Kuo table of primitive
    polynomials.  "joe-kuo-6.10200" (the default) is the table the
    reference compiles in (gold/sobol_primitives.cpp), shipped here for
    2,048 dimensions (128 rates x 16 factors, the library's largest model),
    so the default points are the reference's;
    "new-joe-kuo-6.21201" is the later table shipped with scipy, identical
    on the first 211 dimensions."""
    if table == "joe-kuo-6.10200":
        z = np.load(_TABLE_10200)
        if dims > z["degree"].size:
            raise ValueError(f"table {table} ships {z['degree'].size} dimensions, {dims} asked")
        return (np.ascontiguousarray(z["degree"][:dims]), np.ascontiguousarray(z["a"][:dims]),
                np.ascontiguousarray(z["m"][:dims]))
    if table != "new-joe-kuo-6.21201":
        raise ValueError(f"unknown Sobol table {table!r}")
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


def sobol_directions(dims: int, table: str = SOBOL_TABLE) -> np.ndarray:
    deg, a, m = joe_kuo_table(dims, table)
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
