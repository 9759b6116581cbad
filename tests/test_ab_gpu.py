"""Andersen–Broadie upper bound on the GPU (lmm_andersen_broadie,
lmm_ab_duality_gap) against the reference's gold estimator and the CPU
oracle.

The oracle's gap estimator is pinned to the reference's gold in
test_oracle_pinning.py.  Here: the device estimator equals the gold on the
same data; the inner sub-simulations (continuation estimates) equal the
oracle's, which continues the GPU's recorded outer states with the same
Philox normals; the gap of the whole estimate equals the oracle's gap on
the device's decisions, payoffs and continuation estimates; and the bounds
behave as bounds (gap >= 0, lower bound near the second-pass price).
"""
import ctypes
import os

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def dptr(t):
    return VP(t.data_ptr()) if t is not None else None


def test_duality_gap_kernel_matches_gold(cuda, orc, kref):
    import torch

    from useful_code_b200._lib import call
    from useful_code_b200.pricer import call_size

    rng = np.random.default_rng(17)
    steps, paths = 11, 3001
    is_ex = np.array([1, 1, 0, 1, 1, 1, 0, 1, 1, 1, 0], np.int32)
    ex = (rng.random((steps, paths)) < 0.25).astype(np.int32)
    means = rng.normal(0.01, 0.02, (paths, steps))
    pay = np.maximum(rng.normal(0.0, 0.03, (steps, paths)), 0.0)
    ws = torch.empty(call_size("lmm_ab_duality_gap_workspace_bytes", paths), dtype=torch.uint8,
                     device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    d_ex = torch.from_numpy(ex).cuda()
    d_means = torch.from_numpy(means).cuda()
    d_pay = torch.from_numpy(pay).cuda()
    # zero rebate against the reference's gold
    call("lmm_ab_duality_gap", steps, paths, VP(is_ex.ctypes.data), dptr(d_ex), None,
         dptr(d_means), dptr(ws), ws.numel(), dptr(out), None)
    ref = np.zeros(2)
    kref("kref_ab_gap_zero_rebate", steps, paths, ex, means, np.abs(means), is_ex, ref)
    np.testing.assert_allclose(out.cpu().numpy()[:2], ref, rtol=1e-12)
    # non-zero rebate against the oracle's restatement
    call("lmm_ab_duality_gap", steps, paths, VP(is_ex.ctypes.data), dptr(d_ex), dptr(d_pay),
         dptr(d_means), dptr(ws), ws.numel(), dptr(out), None)
    mine = np.zeros(2)
    orc("orc_ab_gap", steps, paths, ex, pay, means, is_ex, mine)
    np.testing.assert_allclose(out.cpu().numpy()[:2], mine, rtol=1e-12)


def _oracle_ab_inner(m, res, ck, ckN, K, inner, seed, e_begin, e_end):
    from conftest import CLib, _ensure_oracle

    orc = CLib(_ensure_oracle())
    cfg = m.cfg
    E = len(m.ex_steps)
    D = res.depth
    si = np.array([cfg.n, cfg.F, K, 0, m.scramble_dims, mk.PRODUCTS[cfg.product], E,
                   int(cfg.normalise), os.cpu_count() or 1], np.int32)
    sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff], np.float64)
    tau = m.taus.astype(np.float32)
    disp = m.disp.astype(np.float32)
    f0 = m.f0.astype(np.float32)
    lf0 = np.log(f0 + disp).astype(np.float32)
    beta = np.ascontiguousarray(res.beta.cpu().numpy().reshape(E, D, 16))
    means = np.ascontiguousarray(res.means.cpu().numpy().astype(np.float64).reshape(E, D, 3))
    sds = np.ascontiguousarray(res.sds.cpu().numpy().astype(np.float64).reshape(E, D, 3))
    cuts = (np.ascontiguousarray(res.cuts.cpu().numpy().reshape(E, D, 2))
            if res.cuts is not None else None)
    Q = np.zeros((E, K))
    se = np.zeros((E, K))
    ex_steps = np.ascontiguousarray(m.ex_steps.astype(np.int32))
    orc("orc_ab_inner_f", si, sd, m.directions, m.scramblers, m.A, m.fixed, tau, disp, f0, lf0,
        ex_steps, m.nvars, m.mono, m.nbasis, D, beta, means, sds, cuts,
        np.ascontiguousarray(ck), np.ascontiguousarray(ckN), K, inner, ctypes.c_uint64(seed),
        e_begin, e_end, Q, se)
    return Q, se


@pytest.fixture(scope="module")
def swaption_rules(cuda):
    from dataclasses import replace

    from useful_code_b200.pricer import Pipeline, Selector

    cfg = replace(mk.make_config("c2"), n=12, F=3,
                  f0=np.linspace(0.04, 0.06, 12).astype(np.float32), paths=1 << 14,
                  reg_paths=1 << 14)
    m = mk.build_market(cfg)
    pipe = Pipeline(m)
    ls = pipe.first_pass(1 << 14, 0, "fused")
    return m, pipe, {1: pipe.regress(ls), 2: pipe.regress_nested(ls, Selector.production(
        2, min_paths=300))}


@pytest.mark.parametrize("depth", [1, 2])
def test_inner_estimates_and_gap_match_oracle(swaption_rules, orc, depth):
    """Mini Bermudan swaption (12 rates, 3 factors), 64 outer x 256 inner
    paths: every continuation estimate of the device equals the oracle's on
    the device's recorded outer states with the same normals (FP32 on both
    sides: a few inner decisions may flip, each moving an estimate by at most
    an exercise value / 256), and the gap equals the oracle's estimator on
    the device's decisions, payoffs and estimates."""
    m, pipe, rules = swaption_rules
    rule = rules[depth]
    K, inner, seed = 64, 256, 987654321
    r = pipe.andersen_broadie(rule, K, 1 << 15, inner, seed=seed, keep=True)
    Qg = r.Q.cpu().numpy()
    E = Qg.shape[0]
    ck = r.ckpt.cpu().numpy()
    ckN = r.ckptN.cpu().numpy()
    Qo, _ = _oracle_ab_inner(m, rule, ck, ckN, K, inner, seed, 0, E)
    diff = np.abs(Qg - Qo)
    assert np.mean(diff < 1e-6) > 0.97, np.sort(diff.ravel())[-10:]
    assert diff.max() < 2e-3
    assert np.abs(Qg[-1]).max() == 0.0
    X = np.ascontiguousarray(r.X.cpu().numpy())
    Z = np.ascontiguousarray(r.Z.cpu().numpy())
    steps = E + 1
    is_ex = np.array([1] * E + [0], np.int32)
    means = np.zeros((K, steps))
    means[:, :E] = Qg.T
    pay = np.zeros((steps, K))
    pay[:E] = Z
    exm = np.zeros((steps, K), np.int32)
    exm[:E] = X
    mine = np.zeros(2)
    orc("orc_ab_gap", steps, K, exm, pay, means, is_ex, mine)
    assert abs(r.gap - mine[0]) < 1e-12 and abs(r.gap_se - mine[1]) < 1e-12
    # lower bound on the outer paths: payoff at each path's first exercise
    first = np.where(X.any(0), X.argmax(0), -1)
    low = np.where(first >= 0, Z[np.maximum(first, 0), np.arange(K)], 0.0)
    assert abs(r.lower - low.mean()) < 1e-12


def test_bounds_bracket_the_price(swaption_rules):
    """The gap is non-negative, the outer lower bound agrees with the
    second-pass price of the same rule within its standard errors, and the
    gap of a reasonable rule is a small fraction of the price."""
    m, pipe, rules = swaption_rules
    rule = rules[1]
    r = pipe.andersen_broadie(rule, 512, 1 << 16, 256, seed=42)
    assert r.gap >= 0.0
    pay = pipe.second_pass(1 << 16, 1 << 17, rule, "fused")
    price = float(pipe.mean(pay).item())
    pay_np = pay.cpu().numpy().astype(np.float64)
    se_price = pay_np.std() / np.sqrt(pay_np.size)
    assert abs(r.lower - price) < 4 * np.hypot(r.lower_se, se_price)
    assert r.gap < 0.05 * price
    print(f"AB mini swaption: lower {r.lower:.6f} +- {r.lower_se:.6f}, gap {r.gap:.6f} "
          f"+- {r.gap_se:.6f}, second pass {price:.6f}")
