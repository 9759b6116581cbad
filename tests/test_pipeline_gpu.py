"""Whole pipeline (staged and fused) against the CPU oracle (GPU).

The oracle evolves the same Sobol points path by path (lmm_oracle.cpp,
orc_pipeline_*): in FP32 it checks the kernels' arithmetic, in FP64 it is
the precision reference for prices.  Small configurations keep the oracle
within seconds; full sizes are covered by size-independent properties
(batch additivity, staged == fused).
"""
import ctypes
import os
from dataclasses import replace

import numpy as np
import pytest

from conftest import rel_err
from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu


def var_err(a, b):
    """Error of LS variables (rates, swap rates, annuities): relative, with
    values below 0.01 (displaced rates near zero) compared absolutely on
    that scale.  Two FP32 evaluations of the same path agree to about 2e-5
    on this measure: the swap rate (P_s - P_n) / annuity of a short swap
    loses digits to cancellation and the implementations round
    differently."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 0.01)


def mini(product="swaption", n=12, F=3, basis=None, **kw):
    base = {"swaption": "c2", "cancellable": "c5", "european": "c1", "tarn": "t1",
            "bermudan_cap": "c4"}[product]
    cfg = mk.make_config(base)
    f0 = np.linspace(0.04, 0.06, n).astype(np.float32)
    args = dict(n=n, F=F, f0=f0, paths=4096, reg_paths=4096)
    if basis:
        args["basis"] = basis
    args.update(kw)
    from dataclasses import replace

    return replace(cfg, **args)


def oracle_pipeline(mkt, P, offset, mode, rule=None, double=False):
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    from conftest import CLib, _ensure_oracle

    orc = CLib(_ensure_oracle())
    cfg = mkt.cfg
    R = np.float64 if double else np.float32
    E = len(mkt.ex_steps)
    si = np.array([cfg.n, cfg.F, P, offset, mkt.scramble_dims, mk.PRODUCTS[cfg.product], E,
                   int(cfg.normalise), os.cpu_count() or 1], np.int32)
    sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff, cfg.tarn_total,
                   cfg.tarn_multiplier], np.float64)
    if double:
        A = np.ascontiguousarray(mkt.A64)
        fixed = np.ascontiguousarray(-0.5 * (A ** 2).sum(-1))
    else:
        A = mkt.A
        fixed = mkt.fixed
    tau = mkt.taus.astype(R)
    disp = mkt.disp.astype(R)
    f0 = mkt.f0.astype(R)
    lf0 = np.log(f0 + disp).astype(R)
    vars_ = np.zeros((max(E, 1), 3, P), R)
    ex = np.zeros((max(E, 1), P), R)
    cf = np.zeros((max(E, 1), P), R)
    num = np.zeros((max(E, 1), P), R)
    payoff = np.zeros(P)
    beta = means = sds = None
    if rule is not None:
        beta = np.ascontiguousarray(rule.beta.cpu().numpy())
        if rule.means is not None:
            means = rule.means.cpu().numpy().astype(np.float64)
            sds = rule.sds.cpu().numpy().astype(np.float64)
    ex_steps = np.ascontiguousarray(mkt.ex_steps.astype(np.int32))
    orc("orc_pipeline_d" if double else "orc_pipeline_f", si, sd, mkt.directions, mkt.scramblers,
        A, fixed, tau, disp, f0, lf0, ex_steps, mkt.nvars, mkt.mono, mkt.nbasis, mode, beta,
        means, sds, vars_, ex, cf, num, payoff)
    return vars_, ex, cf, num, payoff


@pytest.fixture(scope="module")
def swaption(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("swaption"))
    return m, Pipeline(m)


def test_first_pass_staged_matches_oracle(swaption):
    m, pipe = swaption
    P = 4096
    ls = pipe.first_pass(P, 0, "staged")
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0)
    assert np.max(var_err(ls.vars.cpu().numpy(), v)) < 5e-5
    assert np.max(rel_err(ls.num.cpu().numpy(), num)) < 2e-5
    assert np.max(np.abs(ls.ex.cpu().numpy() - ex)) < 1e-6
    assert not ls.cf.cpu().numpy().any()


def test_fused_equals_staged(swaption):
    m, pipe = swaption
    P = 4096
    a = pipe.first_pass(P, 0, "staged")
    b = pipe.first_pass(P, 0, "fused")
    assert np.max(var_err(b.vars.cpu().numpy(), a.vars.cpu().numpy())) < 5e-5
    assert np.max(rel_err(b.num.cpu().numpy(), a.num.cpu().numpy())) < 2e-6
    # the fused kernels use the hardware exp/rcp approximations
    assert np.max(np.abs(b.ex.cpu().numpy() - a.ex.cpu().numpy())) < 1e-6


def test_rates_vs_fp64_oracle(swaption):
    """Forward rates (as displaced rates f + d, the lognormal quantity),
    annuities and numeraires of the FP32 fused pass within 2e-5 relative of
    the FP64 oracle on the same Sobol points."""
    m, pipe = swaption
    P = 4096
    b = pipe.first_pass(P, 0, "fused")
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0, double=True)
    got = b.vars.cpu().numpy().astype(np.float64)
    d = float(m.disp[0])
    assert np.max(np.abs(got[:, 0] - v[:, 0]) / (v[:, 0] + d)) < 2e-5
    assert np.max(rel_err(got[:, 2], v[:, 2])) < 2e-5
    assert np.max(rel_err(b.num.cpu().numpy(), num)) < 2e-5


@pytest.mark.parametrize("mode", ["staged", "fused"])
def test_batches_are_additive(swaption, mode):
    m, pipe = swaption
    whole = pipe.first_pass(4096, 7, mode)
    parts = pipe.first_pass(4096, 7, mode, batch=1024)
    for x, y in zip((whole.vars, whole.ex, whole.cf, whole.num),
                    (parts.vars, parts.ex, parts.cf, parts.num)):
        assert np.array_equal(x.cpu().numpy(), y.cpu().numpy())


def test_regression_and_second_pass(swaption):
    m, pipe = swaption
    P = 4096
    ls = pipe.first_pass(P, 0, "fused")
    rule = pipe.regress(ls)
    assert int(rule.status.item()) & 3 == 0
    # second pass: staged and fused apply the same frozen rule
    a = pipe.second_pass(P, P, rule, "staged").cpu().numpy()
    b = pipe.second_pass(P, P, rule, "fused").cpu().numpy()
    flips = np.mean(np.abs(a - b) > 1e-6)
    assert flips < 0.01
    assert abs(a.mean() - b.mean()) < 2e-6
    # against the FP32 oracle path by path
    *_, pay = oracle_pipeline(m, P, P, 1, rule)
    assert np.mean(np.abs(b - pay) > 1e-6) < 0.01
    assert abs(b.mean() - pay.mean()) < 2e-6


def test_price_vs_fp64_oracle(swaption):
    """FP32 pipeline price against the FP64 oracle on the same Sobol points
    (regression and pricing both redone in FP64)."""
    import torch

    from useful_code_b200.pricer import LSResult

    m, pipe = swaption
    P = 4096
    res = pipe.price(P, P, "fused")
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0, double=True)
    from conftest import CLib, _ensure_oracle

    orc = CLib(_ensure_oracle())
    E = len(m.ex_steps)
    beta = np.zeros((E, 16))
    means = np.zeros((E, 3))
    sds = np.zeros((E, 3))
    orc("orc_ls_regress_d", E, P, v, m.nvars, m.mono, m.nbasis, cf, ex, num, 1, beta, means, sds,
        None, restype=ctypes.c_double)
    rule = LSResult(torch.from_numpy(beta), torch.from_numpy(means.astype(np.float32)),
                    torch.from_numpy(sds.astype(np.float32)), None, torch.zeros(1), torch.zeros(1))
    *_, pay = oracle_pipeline(m, P, P, 1, rule, double=True)
    price64 = pay.mean() * m.initial_numeraire
    diff_bp = abs(res["price"] - price64) * 1e4
    print(f"mini swaption: fp32 {res['price']:.8f} fp64 {price64:.8f} diff {diff_bp:.4f} bp")
    assert diff_bp < 0.5


def test_cancellable_swap(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("cancellable", n=12, F=3))
    pipe = Pipeline(m)
    P = 4096
    a = pipe.first_pass(P, 0, "staged")
    b = pipe.first_pass(P, 0, "fused")
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0)
    # variable 1 is the swap rate of the swap starting one period later,
    # (P_{s+1} - P_n) / annuity (the reference's formula): at the last dates
    # it is a one- or two-period swap, P_{s+1} - P_n is about tau f P, and a
    # 1-ulp difference in the discount ratios moves it by 200 ulp at a 1%
    # rate; 1e-4 there, 5e-5 for the other variables
    got, staged = b.vars.cpu().numpy(), a.vars.cpu().numpy()
    assert np.max(var_err(got[:, [0, 2]], v[:, [0, 2]])) < 5e-5
    assert np.max(var_err(got[:, 1], v[:, 1])) < 1e-4
    assert np.max(np.abs(b.cf.cpu().numpy() - cf)) < 1e-6
    assert np.max(np.abs(a.cf.cpu().numpy() - cf)) < 1e-6
    assert np.max(var_err(got[:, [0, 2]], staged[:, [0, 2]])) < 5e-5
    assert np.max(var_err(got[:, 1], staged[:, 1])) < 1e-4
    # one frozen rule, applied by the staged and the fused second pass
    rule = pipe.regress(b)
    pa = pipe.second_pass(P, P, rule, "staged").cpu().numpy()
    pb = pipe.second_pass(P, P, rule, "fused").cpu().numpy()
    assert np.mean(np.abs(pa - pb) > 1e-6) < 0.01
    assert abs(pa.mean() - pb.mean()) < 2e-6
    *_, pay = oracle_pipeline(m, P, P, 1, rule)
    assert abs(pb.mean() - pay.mean()) < 2e-6


def test_european_strip(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("european", n=20, F=3))
    pipe = Pipeline(m)
    P = 8192
    a = pipe.second_pass(P, 0, None, "staged").cpu().numpy()
    b = pipe.second_pass(P, 0, None, "fused").cpu().numpy()
    *_, pay32 = oracle_pipeline(m, P, 0, 1)
    *_, pay64 = oracle_pipeline(m, P, 0, 1, double=True)
    assert np.max(np.abs(a - b)) < 2e-6
    assert np.max(np.abs(b - pay32)) < 2e-6
    assert abs(b.mean() - pay64.mean()) * 1e4 < 0.05


@pytest.mark.parametrize("strike", [0.10, 0.08])
def test_tarn_note(cuda, strike):
    """Target redemption note (reference test note: total 0.15, multiplier
    2) over 20 half-year periods: staged, fused and tensor-core evolutions
    agree with the FP32 oracle path by path and with the FP64 oracle within
    0.05 bp.  Strike 0.08 knocks out later, so more coupons are paid."""
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("tarn", n=20, F=3, strike=strike))
    pipe = Pipeline(m)
    P = 8192
    a = pipe.second_pass(P, 0, None, "staged").cpu().numpy()
    b = pipe.second_pass(P, 0, None, "fused").cpu().numpy()
    c = pipe.second_pass(P, 0, None, "tensor").cpu().numpy()
    *_, pay32 = oracle_pipeline(m, P, 0, 1)
    *_, pay64 = oracle_pipeline(m, P, 0, 1, double=True)
    # a knock-out decided by a coupon within rounding of the target moves
    # the note's remaining flows: compare path by path away from those
    close = np.abs(b - pay32) < 2e-6
    assert np.mean(close) > 0.999
    assert np.mean(np.abs(a - b) < 2e-6) > 0.999
    assert np.mean(np.abs(c - b) < 2e-5) > 0.999
    assert abs(b.mean() - pay64.mean()) * 1e4 < 0.05
    assert abs(c.mean() - pay64.mean()) * 1e4 < 0.05
    assert abs(a.mean() - pay64.mean()) * 1e4 < 0.05
    # the note pays something and knocks out on some but not all paths
    assert b.std() > 0


def test_c3_price_and_rates_vs_fp64_oracle(cuda):
    """The benchmark configuration (80 quarterly rates, 10 factors, cross
    basis) on 2^14 regression + 2^14 pricing paths: the first forward at
    every exercise date within 2e-5 (plain relative where |f| >= 0.005,
    absolute 2e-7 below) of the FP64 oracle,
    and all LS basis variables (forward, swap rate, annuity) within 5e-5
    (relative, values below 0.01 on that scale: the swap rate's
    cancellation); every forward rate of every step is checked in
    test_all_forward_rates_vs_fp64_oracle; the price
    within 0.05 bp of notional of the FP64 oracle under the same rule, and
    the FP64 oracle's own regression within 0.5 bp (see _price_vs_fp64)."""
    from useful_code_b200.pricer import Pipeline

    P = 1 << 14
    m = mk.build_market(mk.make_config("c3", paths=P, reg_paths=P))
    pipe = Pipeline(m)
    ls = pipe.first_pass(P, 0, "fused")
    v, *_ = oracle_pipeline(m, P, 0, 0, double=True)
    got = ls.vars.cpu().numpy().astype(np.float64)
    big = np.abs(v[:, 0]) >= 0.005  # as in the all-rates check: near zero, absolute
    fwd_max = float(np.max(np.abs(got[:, 0] - v[:, 0])[big] / np.abs(v[:, 0])[big]))
    assert np.all(np.abs(got[:, 0] - v[:, 0])[~big] < 2e-5 * 0.01)
    var_max = float(np.max(var_err(got, v)))
    assert fwd_max < 2e-5, fwd_max
    assert var_max < 5e-5, var_max
    price, price64, price64_own = _price_vs_fp64(m, pipe, P, ls)
    diff_bp = abs(price - price64) * 1e4
    rule_bp = abs(price64 - price64_own) * 1e4
    print(f"c3 2^14+2^14: fp32 {price:.8f} fp64 {price64:.8f} diff {diff_bp:.4f} bp; "
          f"fp64 with its own rule {price64_own:.8f} ({rule_bp:.4f} bp); forwards {fwd_max:.2e}, "
          f"LS variables {var_max:.2e}")
    assert diff_bp < 0.05
    assert rule_bp < 0.5


def test_bermudan_cap_portfolio(cuda):
    """The swaption-plus-cap portfolio of the differentiation form on a small
    model: staged and fused second passes against the FP32 oracle path by
    path and the FP64 oracle within 0.05 bp; the portfolio equals the
    swaption (same rule) plus the cap strip (the European strip with no swap
    leg) priced separately on the same points."""
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("bermudan_cap"))
    pipe = Pipeline(m)
    P = 4096
    rule = pipe.regress(pipe.first_pass(P, 0, "fused"))
    a = pipe.second_pass(P, P, rule, "staged").cpu().numpy().astype(np.float64)
    b = pipe.second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    *_, pay32 = oracle_pipeline(m, P, P, 1, rule)
    *_, pay64 = oracle_pipeline(m, P, P, 1, rule, double=True)
    assert np.mean(np.abs(b - pay32) < 2e-6) > 0.999
    assert np.mean(np.abs(a - b) < 2e-6) > 0.999
    assert abs(b.mean() - pay64.mean()) * 1e4 < 0.05
    assert abs(a.mean() - pay64.mean()) * 1e4 < 0.05
    swp = Pipeline(mk.build_market(replace(m.cfg, product="swaption")))
    cap = Pipeline(mk.build_market(replace(m.cfg, product="european", pay_receive=0.0)))
    s1 = swp.second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    s2 = cap.second_pass(P, P, None, "fused").cpu().numpy().astype(np.float64)
    assert np.max(np.abs(b - (s1 + s2))) < 1e-6
    assert s1.mean() > 0 and s2.mean() > 0
    with pytest.raises(Exception):
        pipe.second_pass(P, P, rule, "tensor")


def _price_vs_fp64(m, pipe, P, ls=None):
    """(device price, FP64 price under the device's rule, FP64 price under
    the FP64 oracle's own rule), all at time 0 on P regression + P pricing
    paths.  The device's and the oracle's rules come from regressions on
    the FP32 and FP64 first passes of the same points: their fitted values
    agree to about 1e-7, which still moves the exercise decision of a
    handful of paths lying that close to the boundary; at 2^12-2^14 paths
    that shifts the price by up to about 0.1 bp, a sampling effect of the
    regression that shrinks like 1/sqrt(paths).  The FP32 path arithmetic
    is measured under one rule: the device's price against the FP64 oracle
    pricing the same points with the device's rule."""
    import torch

    from conftest import CLib, _ensure_oracle
    from useful_code_b200.pricer import LSResult

    ls = ls if ls is not None else pipe.first_pass(P, 0, "fused")
    rule = pipe.regress(ls)
    price = float(pipe.mean(pipe.second_pass(P, P, rule, "fused")).item()) * m.initial_numeraire
    *_, pay_dev_rule = oracle_pipeline(m, P, P, 1, rule, double=True)
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0, double=True)
    orc = CLib(_ensure_oracle())
    E = len(m.ex_steps)
    beta = np.zeros((E, 16))
    means = np.zeros((E, 3))
    sds = np.zeros((E, 3))
    orc("orc_ls_regress_d", E, P, v, m.nvars, m.mono, m.nbasis, cf, ex, num, 1, beta, means, sds,
        None, restype=ctypes.c_double)
    rule64 = LSResult(torch.from_numpy(beta), torch.from_numpy(means.astype(np.float32)),
                      torch.from_numpy(sds.astype(np.float32)), None, torch.zeros(1), torch.zeros(1))
    *_, pay64 = oracle_pipeline(m, P, P, 1, rule64, double=True)
    return price, pay_dev_rule.mean() * m.initial_numeraire, pay64.mean() * m.initial_numeraire


def test_c4_portfolio_price_vs_fp64_oracle(cuda):
    """The differentiation form at its stated model shape (80 quarterly
    rates, 10 factors, the swaption-plus-cap portfolio) on 2^13 regression
    + 2^13 pricing paths: the price within 0.05 bp of notional of the FP64
    oracle under the same rule; the FP64 oracle's own regression changes
    the price by less than 0.5 bp (see _price_vs_fp64)."""
    from useful_code_b200.pricer import Pipeline

    P = 1 << 13
    m = mk.build_market(mk.make_config("c4", paths=P, reg_paths=P))
    price, price64, price64_own = _price_vs_fp64(m, Pipeline(m), P)
    diff_bp = abs(price - price64) * 1e4
    rule_bp = abs(price64 - price64_own) * 1e4
    print(f"c4 2^13+2^13: fp32 {price:.8f} fp64 {price64:.8f} diff {diff_bp:.4f} bp; "
          f"fp64 with its own rule {price64_own:.8f} ({rule_bp:.4f} bp)")
    assert diff_bp < 0.05
    assert rule_bp < 0.5


@pytest.mark.parametrize("name,P", [("c2", 4096), ("c3", 2048), ("c5", 1024)])
def test_all_forward_rates_vs_fp64_oracle(cuda, name, P):
    """Every forward rate of every step, at the form's stated model shape:
    the fused pricing arithmetic (lmm_fused_variates, then lmm_evolve_pc_all,
    whose rate step is the pricing kernels') against the FP64 oracle
    evolving the same Sobol points in double.  Plain relative error within
    2e-5 for |f| >= 0.005; below that (displaced rates can pass through
    zero, about 2.5% of the c5 entries) the absolute error within
    2e-5 x 0.01."""
    import torch

    from conftest import CLib, _ensure_oracle
    from useful_code_b200._lib import call
    from useful_code_b200.pricer import Pipeline, dp, stream_handle

    m = mk.build_market(mk.make_config(name, paths=P, reg_paths=P))
    cfg = m.cfg
    n, F = cfg.n, cfg.F
    pipe = Pipeline(m)
    var = torch.empty(n, F, P, device="cuda")
    call("lmm_fused_variates", ctypes.addressof(pipe.model), P, 0, dp(var), stream_handle())
    rates = torch.empty(n, n, P, device="cuda")
    lrates = torch.empty(n, n, P, device="cuda")
    alive = np.arange(n, dtype=np.int32)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    call("lmm_evolve_pc_all", vp(m.f0), vp(m.taus), vp(m.disp), dp(var), 1, dp(pipe.A),
         dp(pipe.fixed), vp(alive), P, F, n, n, cfg.cutoff, dp(rates), dp(lrates), None,
         stream_handle())
    got = rates.cpu().numpy().astype(np.float64)
    orc = CLib(_ensure_oracle())
    si = np.array([n, F, P, 0, m.scramble_dims, 0, 0, 0, os.cpu_count() or 1], np.int32)
    sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff], np.float64)
    A = np.ascontiguousarray(m.A64)
    fixed = np.ascontiguousarray(-0.5 * (A ** 2).sum(-1))
    f0 = m.f0.astype(np.float64)
    disp = m.disp.astype(np.float64)
    ref = np.zeros((n, n, P))
    orc("orc_path_rates_d", si, sd, m.directions, m.scramblers, A, fixed,
        m.taus.astype(np.float64), disp, f0, np.log(f0 + disp), ref)
    mask = np.broadcast_to(np.triu(np.ones((n, n), bool))[:, :, None], (n, n, P))
    g, r = got[mask], ref[mask]
    big = np.abs(r) >= 0.005
    rel = np.abs(g[big] - r[big]) / np.abs(r[big])
    small = np.abs(g[~big] - r[~big])
    print(f"{name} all rates: max rel {rel.max():.2e} (mean {rel.mean():.1e}) over {big.sum()}, "
          f"max abs {small.max() if small.size else 0:.1e} over {small.size} near zero")
    assert rel.max() < 2e-5
    assert small.size == 0 or small.max() < 2e-5 * 0.01


@pytest.mark.parametrize("name,P", [("c2", 1 << 13), ("c5", 1 << 12)])
def test_config_price_vs_oracles(cuda, name, P):
    """The c2 form (40 semi-annual rates, 5 factors, the six-function basis)
    and the c5 form (120 quarterly rates, 15 factors, the cancellable payer
    swap, twelve basis functions) at their stated model shapes on P
    regression + P pricing paths: the fused first pass's LS inputs against
    the FP32 oracle on the same points (two FP32 evaluations drift apart with
    the step count: 5e-5 on var_err's measure over c2's 40 steps, 1e-4 over
    c5's 120); the second pass under the device's
    rule against the FP32 oracle path by path; the price within 0.05 bp of
    notional of the FP64 oracle under the same rule, and the FP64 oracle's
    own regression within 0.5 bp (see _price_vs_fp64)."""
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mk.make_config(name, paths=P, reg_paths=P))
    assert int(m.nbasis.max()) == {"c2": 6, "c5": 12}[name]
    pipe = Pipeline(m)
    ls = pipe.first_pass(P, 0, "fused")
    v32, ex32, cf32, num32, _ = oracle_pipeline(m, P, 0, 0)
    assert np.max(var_err(ls.vars.cpu().numpy(), v32)) < {"c2": 5e-5, "c5": 1e-4}[name]
    assert np.max(rel_err(ls.num.cpu().numpy(), num32)) < 2e-5
    assert np.max(np.abs(ls.ex.cpu().numpy() - ex32)) < 2e-6
    assert np.max(np.abs(ls.cf.cpu().numpy() - cf32)) < 2e-6
    rule = pipe.regress(ls)
    pay = pipe.second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    *_, pay32 = oracle_pipeline(m, P, P, 1, rule)
    assert np.mean(np.abs(pay - pay32) < 2e-6) > 0.999
    price, price64, price64_own = _price_vs_fp64(m, pipe, P, ls)
    assert abs(price - pay.mean() * m.initial_numeraire) < 1e-7
    diff_bp = abs(price - price64) * 1e4
    rule_bp = abs(price64 - price64_own) * 1e4
    print(f"{name} {P}+{P}: fp32 {price:.8f} fp64 {price64:.8f} diff {diff_bp:.4f} bp; "
          f"fp64 with its own rule {price64_own:.8f} ({rule_bp:.4f} bp)")
    assert diff_bp < 0.05
    assert rule_bp < 0.5


def test_c1_stated_shape_vs_oracles(cuda):
    """The c1 form at its stated shape (20 semi-annual rates, flat 5%
    forwards, 3 factors, 20 steps, 16,384 paths, the caplet strip plus the
    payer swap at 5%): fused payoffs path by path against the FP32 oracle on
    the same Sobol points, the staged form against the fused one, and the
    price within 0.05 bp of notional of the FP64 oracle."""
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mk.make_config("c1"))
    cfg = m.cfg
    assert (cfg.n, cfg.F, cfg.paths, cfg.product) == (20, 3, 16384, "european")
    P = cfg.paths
    pipe = Pipeline(m)
    fused = pipe.second_pass(P, 0, None, "fused").cpu().numpy().astype(np.float64)
    staged = pipe.second_pass(P, 0, None, "staged").cpu().numpy().astype(np.float64)
    *_, pay32 = oracle_pipeline(m, P, 0, 1)
    *_, pay64 = oracle_pipeline(m, P, 0, 1, double=True)
    assert np.max(np.abs(fused - pay32)) < 2e-6
    assert np.max(np.abs(staged - fused)) < 2e-6
    diff_bp = abs(fused.mean() - pay64.mean()) * m.initial_numeraire * 1e4
    print(f"c1 {P}: fp32 {fused.mean() * m.initial_numeraire:.8f} "
          f"fp64 {pay64.mean() * m.initial_numeraire:.8f} diff {diff_bp:.5f} bp")
    assert diff_bp < 0.05
