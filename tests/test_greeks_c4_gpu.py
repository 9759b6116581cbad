"""Pathwise adjoint Greeks of the differentiation form at its stated shape
(GPU): 80 quarterly forwards, 10 factors, the portfolio of the Bermudan
payer swaption and the 5% cap strip, log-rate checkpoints every 8 steps,
2^12 paths.

Two references, both on the adjoint's own Sobol points:

* central differences of the FP64 oracle's frozen-exercise price
  (orc_frozen_payoff_d, each path held at the exercise step the GPU
  recorded): a sample of deltas and per-rate vegas, two random directions
  in the pseudo-root entries and the four abcd vegas.  The first forward
  (5.03%) sits at the caplets' 5% strike, so a bump of 1e-5 straddles a
  caplet kink on some paths, where a central difference averages the two
  slopes; in FP64 a bump of 1e-6 costs nothing in rounding and shrinks that
  bias tenfold, so the deltas and vegas are held to 2e-4 of the largest
  entry at 1e-6 and to 5e-4 at the stated bump of 1e-5;
* bumped re-runs of the plain forward GPU kernel (the fused second pass,
  lmm_pipeline_second_pass, with the same frozen rule), for every delta and
  every per-rate vega (forward-rate bumps of 1e-5; relative bumps of 1e-3
  of the pseudo-root rows, since 1e-5 would move the log-rates by about one
  FP32 unit in the last place, where the re-runs only quantise).  A bump
  can move a path across the exercise
  boundary, which the pathwise method excludes; such a path shows as a
  jump in the second difference of its payoffs (up - 2 base + down, above
  1e-6 where FP32 rounding leaves about 1e-7), and its difference is taken
  from the FP64 frozen-exercise payoff of that one path instead.  The
  comparison is against the adjoint projected on the exact FP32
  perturbation (rounded bumped inputs minus the base), so the rounding of
  the bump itself cancels; the tolerance is five times the FP32 rounding
  noise of the re-runs (measured from the second differences of the paths
  off the boundary) plus 5e-4 of the largest entry.
"""
import ctypes
import os
from dataclasses import replace

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu

H = 1e-5
# relative bump of a pseudo-root row in the forward re-runs: a row moves the
# log-rates by about A z HV per step, which must stay well above FP32's
# resolution of the log-rates (about 2e-7 at log f ~ -3); at 1e-5 it is
# about one unit in the last place, where the re-runs only quantise
HV = 1e-3
P = 1 << 12
K_CKPT = 8


def _orc():
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from conftest import CLib, _ensure_oracle

    return CLib(_ensure_oracle())


class FrozenC4:
    """FP64 frozen-exercise payoffs of the portfolio on the adjoint's paths."""

    def __init__(self, m, offset, exercise_step):
        self.orc = _orc()
        self.m, self.offset = m, offset
        cfg = m.cfg
        E = len(m.ex_steps)
        pos = {int(s): e for e, s in enumerate(m.ex_steps)}
        self.ex_at = np.array([pos.get(int(s), E) for s in exercise_step], np.int32)
        self.sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff],
                           np.float64)
        self.ex_steps = np.ascontiguousarray(m.ex_steps.astype(np.int32))

    def payoffs(self, f0, A, first=0, count=None):
        """Per-path deflated payoffs of paths [first, first + count)."""
        m, cfg = self.m, self.m.cfg
        count = len(self.ex_at) - first if count is None else count
        si = np.array([cfg.n, cfg.F, count, self.offset + first, m.scramble_dims,
                       mk.PRODUCTS[cfg.product], len(m.ex_steps), int(cfg.normalise),
                       os.cpu_count() or 1], np.int32)
        A = np.ascontiguousarray(A, np.float64)
        fixed = np.ascontiguousarray(-0.5 * (A ** 2).sum(-1))
        f0 = np.ascontiguousarray(f0, np.float64)
        disp = m.disp.astype(np.float64)
        pay = np.zeros(count)
        self.orc("orc_frozen_payoff_d", si, self.sd, m.directions, m.scramblers, A, fixed,
                 m.taus.astype(np.float64), disp, f0, np.log(f0 + disp), self.ex_steps,
                 np.ascontiguousarray(self.ex_at[first:first + count]), pay)
        return pay

    def price(self, f0, A):
        return self.payoffs(f0, A).mean() / (1.0 + f0[0] * float(self.m.rate_times[0]))


@pytest.fixture(scope="module")
def c4(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mk.make_config("c4", paths=P, reg_paths=P))
    assert m.cfg.product == "bermudan_cap" and m.cfg.n == 80 and m.cfg.F == 10
    pipe = Pipeline(m)
    rule = pipe.regress(pipe.first_pass(P, 0, "fused"))
    g = pipe.greeks(P, P, rule, checkpoint_every=K_CKPT)
    fz = FrozenC4(m, P, g.exercise_step)
    return m, pipe, rule, g, fz


def test_c4_price_matches_forward_and_oracle(c4):
    m, pipe, rule, g, fz = c4
    pay = pipe.second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    assert abs(g.price - pay.mean() * m.initial_numeraire) < 1e-9 * abs(g.price) + 1e-12
    ref = fz.price(m.f0.astype(np.float64), m.A64)
    assert abs(ref - g.price) * 1e4 < 0.05, (ref, g.price)
    # the cap strip pays on most paths
    assert np.mean(pay > 0.0) > 0.9
    # some paths exercise the swaption, and exercised paths run on for the cap
    assert np.any(g.exercise_step < m.cfg.n)


def _fd_oracle_close(got, fd, rel):
    scale = max(np.max(np.abs(fd)), 1e-12)
    err = np.max(np.abs(np.asarray(got) - np.asarray(fd))) / scale
    assert err < rel, (err, got, fd)


@pytest.mark.parametrize("h,tol", [(1e-6, 2e-4), (H, 5e-4)])
def test_c4_deltas_and_vegas_vs_fp64_fd(c4, h, tol):
    m, pipe, rule, g, fz = c4
    f0 = m.f0.astype(np.float64)
    A = m.A64
    rates = [0, 1, 7, 19, 38, 52, 70, 79]
    fd_delta, fd_vega = [], []
    for r in rates:
        up, dn = f0.copy(), f0.copy()
        up[r] += h
        dn[r] -= h
        fd_delta.append((fz.price(up, A) - fz.price(dn, A)) / (2 * h))
        D = np.zeros_like(A)
        D[:, r, :] = A[:, r, :]
        fd_vega.append((fz.price(f0, A + h * D) - fz.price(f0, A - h * D)) / (2 * h))
    print(f"c4 bump {h:g}: deltas {np.max(np.abs(g.delta[rates] - fd_delta)):.2e}, "
          f"vegas {np.max(np.abs(g.vega_rate[rates] - fd_vega)):.2e} (largest "
          f"{np.max(np.abs(fd_delta)):.3f}, {np.max(np.abs(fd_vega)):.3f})")
    _fd_oracle_close(g.delta[rates], np.array(fd_delta), tol)
    _fd_oracle_close(g.vega_rate[rates], np.array(fd_vega), tol)
    rng = np.random.default_rng(41)
    for _ in range(2):
        D = A * rng.uniform(-1.0, 1.0, A.shape)
        fd = (fz.price(f0, A + h * D) - fz.price(f0, A - h * D)) / (2 * h)
        ad = float(np.sum(g.abar * D))
        assert abs(ad - fd) < tol * abs(fd) + 1e-9, (ad, fd)


def test_c4_abcd_vegas_vs_fp64_fd(c4):
    from useful_code_b200._lib import LIB

    m, pipe, rule, g, fz = c4
    cfg = m.cfg
    a, b, c, d = cfg.abcd
    times = np.ascontiguousarray(m.rate_times[:cfg.n].astype(np.float64))
    mult = np.ones(cfg.n)
    out = np.zeros(4)
    abar = np.ascontiguousarray(g.abar)
    vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert LIB.lmm_abcd_vegas(a, b, c, d, vp(times), cfg.n, vp(times), cfg.n, vp(mult), cfg.F,
                              cfg.L, cfg.beta, vp(abar), 1e-5, vp(out)) == 0
    f0 = m.f0.astype(np.float64)
    fd = []
    for k in range(4):
        h = 1e-5 * max(abs(cfg.abcd[k]), 1e-3)
        prices = []
        for sgn in (1, -1):
            p = list(cfg.abcd)
            p[k] += sgn * h
            prices.append(fz.price(f0, mk.pseudo_roots(replace(cfg, abcd=tuple(p)),
                                                         m.rate_times)))
        fd.append((prices[0] - prices[1]) / (2 * h))
    _fd_oracle_close(out, np.array(fd), 5e-4)


# ---- bumped re-runs of the plain forward kernel ----------------------------
def _forward(m, rule, f0_32, A32):
    """Per-path payoffs of the fused second pass on a market with the given
    FP32 initial curve and pseudo-roots (fixed drifts recomputed from A)."""
    from useful_code_b200._lib import call
    from useful_code_b200.pricer import Pipeline

    n, F = m.cfg.n, m.cfg.F
    A32 = np.ascontiguousarray(A32, np.float32)
    fixed = np.zeros((n, n), np.float32)
    call("lmm_fixed_drifts", A32.ctypes.data_as(ctypes.c_void_p), n, n, F,
         fixed.ctypes.data_as(ctypes.c_void_p))
    mm = replace(m, f0=np.ascontiguousarray(f0_32, np.float32), A=A32, fixed=fixed,
                 A64=A32.astype(np.float64))
    pay = Pipeline(mm).second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    return pay, 1.0 / (1.0 + float(mm.f0[0]) * float(m.rate_times[0]))


def _gpu_fd(m, rule, fz, base, f0_up, f0_dn, A_up, A_dn):
    """(FD of the price from GPU re-runs with frozen-boundary paths taken
    from the FP64 frozen payoffs, noise scale of the estimate, paths
    replaced)."""
    up, p0u = _forward(m, rule, f0_up, A_up)
    dn, p0d = _forward(m, rule, f0_dn, A_dn)
    jump = np.abs(up - 2.0 * base + dn) > 1e-6
    diff = up - dn
    idx = np.flatnonzero(jump)
    for p in idx:
        ou = fz.payoffs(f0_up.astype(np.float64), A_up.astype(np.float64), int(p), 1)[0]
        od = fz.payoffs(f0_dn.astype(np.float64), A_dn.astype(np.float64), int(p), 1)[0]
        diff[p] = ou - od
    # price = P(0,T_0) mean(payoff); P(0,T_0) moves only with f0_0
    mean_up = base.mean() + 0.5 * diff.mean()
    mean_dn = base.mean() - 0.5 * diff.mean()
    fd = p0u * mean_up - p0d * mean_dn
    # FP32 rounding noise of the estimate: for a path off the boundary the
    # second difference up - 2 base + down is rounding alone (curvature is
    # O(h^2)), with three times the variance of up - down's rounding
    second = (up - 2.0 * base + dn)[~jump]
    noise = 0.5 * (p0u + p0d) * np.sqrt(np.mean(second ** 2) / 3.0) / np.sqrt(P)
    return fd, noise, idx.size


def test_c4_bumped_forward_runs_match_adjoint(c4):
    m, pipe, rule, g, fz = c4
    n = m.cfg.n
    f0 = np.ascontiguousarray(m.f0, np.float32)
    A = np.ascontiguousarray(m.A, np.float32)
    base, _ = _forward(m, rule, f0, A)
    replaced = 0
    worst = 0.0
    scale_d = np.max(np.abs(g.delta))
    scale_v = np.max(np.abs(g.vega_rate))
    for r in range(n):
        up, dn = f0.copy(), f0.copy()
        up[r] = np.float32(f0[r] + np.float32(H))
        dn[r] = np.float32(f0[r] - np.float32(H))
        pred = g.delta[r] * (float(up[r]) - float(dn[r]))
        fd, noise, k = _gpu_fd(m, rule, fz, base, up, dn, A, A)
        replaced += k
        err = abs(fd - pred)
        worst = max(worst, err / (float(up[r]) - float(dn[r])) / scale_d)
        assert err < 5.0 * noise + 5e-4 * scale_d * (float(up[r]) - float(dn[r])), \
            ("delta", r, fd, pred, noise)
        Au, Ad = A.copy(), A.copy()
        Au[:, r, :] = (A[:, r, :].astype(np.float64) * (1.0 + HV)).astype(np.float32)
        Ad[:, r, :] = (A[:, r, :].astype(np.float64) * (1.0 - HV)).astype(np.float32)
        pred = float(np.sum(g.abar * (Au.astype(np.float64) - Ad.astype(np.float64))))
        fd, noise, k = _gpu_fd(m, rule, fz, base, f0, f0, Au, Ad)
        replaced += k
        assert abs(fd - pred) < 5.0 * noise + 5e-4 * scale_v * 2 * HV, \
            ("vega", r, fd, pred, noise)
    # the boundary paths are few: the re-runs are the check, not the oracle
    assert replaced < 0.02 * P * 2 * n, replaced
    print(f"c4 bumped forward runs: worst delta error {worst:.2e} of the largest delta, "
          f"{replaced} boundary paths replaced over {2 * n} bumps of {P} paths")
