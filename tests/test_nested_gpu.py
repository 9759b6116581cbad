"""Nested Longstaff–Schwartz regressions (depth > 1, fraction selector) and
rules with Andersen shifts, on the GPU, against the CPU oracle.

The oracle's restatement (orc_ls_regress_multi_*) is pinned to the
reference's gold nested regression in test_oracle_pinning.py.  Here the
device regression (lmm_ls_regress_nested) runs on the same FP32 inputs as
the oracle's FP32-input restatement: the in-sample price, the cut-offs of
every nested regression, the per-depth moments and the fitted values must
agree; the frozen nested rule (with shifts) applied by the GPU in every
mode must give the oracle's path values.
"""
import ctypes

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def call(name, *args):
    from useful_code_b200._lib import call as c

    return c(name, *args)


def dptr(t):
    return VP(t.data_ptr()) if t is not None else None


def hptr(a):
    return VP(a.ctypes.data)


def gpu_nested(vars32, cf32, ex32, num32, nvars, mono, nb, select, normalise=1):
    import torch

    from useful_code_b200.pricer import LmmLsSelect

    E, _, P = vars32.shape
    D = select[0]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    v, c, x, n = dev(vars32), dev(cf32), dev(ex32), dev(num32)
    from useful_code_b200.pricer import call_size

    ws = torch.empty(call_size("lmm_ls_nested_workspace_bytes", P, E), dtype=torch.uint8,
                     device="cuda")
    beta = torch.zeros(E, D, 16, dtype=torch.float64, device="cuda")
    means = torch.zeros(E, D, 3, device="cuda")
    sds = torch.ones(E, D, 3, device="cuda")
    cuts = torch.zeros(E, D, 2, dtype=torch.float64, device="cuda")
    npaths = torch.zeros(E, D, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    price = torch.zeros(1, dtype=torch.float64, device="cuda")
    sel = LmmLsSelect(*select)
    mono = np.ascontiguousarray(mono.astype(np.uint8))
    nvars = np.ascontiguousarray(nvars.astype(np.int32))
    nb = np.ascontiguousarray(nb.astype(np.int32))
    call("lmm_ls_regress_nested", E, P, dptr(v), hptr(nvars), hptr(mono), hptr(nb), dptr(c),
         dptr(x), dptr(n), normalise, ctypes.addressof(sel), dptr(ws), ws.numel(), dptr(beta),
         dptr(means) if normalise else None, dptr(sds) if normalise else None, dptr(cuts),
         dptr(npaths), dptr(status), dptr(price), None)
    torch.cuda.synchronize()
    return dict(beta=beta.cpu().numpy(), means=means.cpu().numpy().astype(np.float64),
                sds=sds.cpu().numpy().astype(np.float64), cuts=cuts.cpu().numpy(),
                npaths=npaths.cpu().numpy(), status=int(status.item()),
                price=float(price.item()))


def oracle_nested(orc, vars32, cf32, ex32, num32, nvars, mono, nb, select, normalise=1):
    E, _, P = vars32.shape
    D = select[0]
    beta = np.zeros((E, D, 16))
    means = np.zeros((E, D, 3))
    sds = np.ones((E, D, 3))
    cuts = np.zeros((E, D, 2))
    status = np.zeros(1, np.int32)
    opts = np.array([select[1], select[2], select[3], select[4], float(select[5])])
    price = orc("orc_ls_regress_multi_f", E, P, vars32, nvars, mono, nb, cf32, ex32, num32,
                normalise, D, opts, beta, means, sds, cuts, status, restype=ctypes.c_double)
    return dict(beta=beta, means=means, sds=sds, cuts=cuts, status=int(status[0]), price=price)


def fits(res, vars_, mono, nb, e, d):
    """Fitted values of regression (e, d) on all paths."""
    x = (vars_[e].astype(np.float64) - res["means"][e, d][:, None]) / res["sds"][e, d][:, None]
    phi = np.stack([np.prod([x[j] ** int(mono[e, k, j]) for j in range(3)], 0)
                    for k in range(nb[e])])
    return res["beta"][e, d, :nb[e]] @ phi


@pytest.mark.parametrize("depth", [2, 3, 4])
@pytest.mark.parametrize("cross", [0])
def test_nested_regression_one_date_gold_inputs(cuda, gold, orc, depth, cross):
    """Each of the gold LS fixture's first three dates (512 paths, exercise
    values tripled) as a one-date problem, production selector settings
    with 20 paths minimum: coefficients, moments, cut-offs and path counts
    of every nested regression against the oracle on the same FP32 inputs.
    One date at a time, so no exercise decision feeds the next regression:
    over several dates the nested regressions (fitted to the paths nearest
    the exercise boundary) leave estimate and exercise value within FP32
    rounding of each other on some paths, and FP32 / FP64 evaluations take
    different decisions there.  (The fourth date's basis variables f and SR
    coincide in exact arithmetic; the oracle-against-gold pinning covers it
    with the reference's SVD.)  The quadratic basis only: the cross basis's
    ten functions on nested subsets of 21 to 237 of these paths are too
    close to singular for FP32 and FP64 fits to agree to better than about
    1e-3; test_nested_regression_one_date_first_pass covers the cross basis
    on 2^14 paths."""
    nvars_all = gold["ls_nvars"]
    mono_all, nb_all = mk.basis_tables("cross" if cross else "quadratic", nvars_all)
    lf = 0.1 ** (1.0 / (depth - 1))
    select = (depth, lf, lf * 1.01, 2.5, 0.8, 20)
    for e in range(3):
        sl = slice(e, e + 1)
        c32 = lambda k: np.ascontiguousarray(gold[k][sl].astype(np.float32))
        vars32, cf32, ex32, num32 = c32("ls_vars"), c32("ls_cf"), c32("ls_ex3"), c32("ls_num")
        nvars = np.ascontiguousarray(nvars_all[sl])
        mono = np.ascontiguousarray(mono_all[sl])
        nb = np.ascontiguousarray(nb_all[sl])
        g = gpu_nested(vars32, cf32, ex32, num32, nvars, mono, nb, select)
        o = oracle_nested(orc, vars32, cf32, ex32, num32, nvars, mono, nb, select)
        # nested regressions of up to 10 functions on 21 to 237 paths: their
        # FP32 / FP64 fits agree to a few 1e-4 of the values' scale, the
        # cut-offs to 1e-4, and one decision of 512 may flip (about 1e-5)
        check_nested(g, o, vars32, mono, nb, depth, min_paths=20, fit_tol=5e-4, ex32=ex32,
                     cut_rtol=1e-4, price_tol=5e-5)


def check_nested(g, o, vars32, mono, nb, depth, min_paths, fit_tol, ex32, cut_rtol=1e-6,
                 price_tol=1e-6):
    """Parity of two nested regressions; each regression's fitted values are
    compared on the paths it was fitted to (the oracle's selection)."""
    E, _, P = vars32.shape
    assert (g["status"] & ~4) == 0 and o["status"] == 0
    assert abs(g["price"] - o["price"]) < price_tol
    np.testing.assert_allclose(g["cuts"][:, :-1], o["cuts"][:, :-1], rtol=cut_rtol, atol=1e-12)
    for e in range(E):
        assert g["npaths"][e, 0] == P
        member = np.ones(P, bool)
        for d in range(depth):
            if d > 0 and o["cuts"][e, d - 1, 1] == 0.0:
                assert g["npaths"][e, d] == 0
                break
            if d > 0:
                net = fits(o, vars32, mono, nb, e, d - 1) - ex32[e].astype(np.float64)
                member &= np.abs(net) <= o["cuts"][e, d - 1, 1]
                assert g["npaths"][e, d] > min_paths
                assert abs(int(g["npaths"][e, d]) - int(member.sum())) <= 1
            np.testing.assert_allclose(g["means"][e, d], o["means"][e, d], rtol=1e-5, atol=1e-7)
            np.testing.assert_allclose(g["sds"][e, d], o["sds"][e, d], rtol=1e-5)
            fg = fits(g, vars32, mono, nb, e, d)[member]
            fo = fits(o, vars32, mono, nb, e, d)[member]
            scale = max(np.abs(fo).max(), 1e-3)
            assert np.max(np.abs(fg - fo)) < fit_tol * scale, (e, d)


def _pipeline_rule(m, res, E):
    """Oracle rule arrays (FP64) from a GPU nested regression."""
    D = res.depth
    beta = np.ascontiguousarray(res.beta.cpu().numpy().reshape(E, D, 16))
    means = np.ascontiguousarray(res.means.cpu().numpy().astype(np.float64).reshape(E, D, 3))
    sds = np.ascontiguousarray(res.sds.cpu().numpy().astype(np.float64).reshape(E, D, 3))
    cuts = np.ascontiguousarray(res.cuts.cpu().numpy().reshape(E, D, 2))
    shifts = (np.ascontiguousarray(res.shifts.cpu().numpy().astype(np.float64))
              if res.shifts is not None else None)
    return beta, means, sds, cuts, shifts


def oracle_pipeline_rule(m, P, offset, beta, means, sds, cuts, shifts, D, double=False):
    import os

    from conftest import CLib, _ensure_oracle

    orc = CLib(_ensure_oracle())
    cfg = m.cfg
    R = np.float64 if double else np.float32
    E = len(m.ex_steps)
    si = np.array([cfg.n, cfg.F, P, offset, m.scramble_dims, mk.PRODUCTS[cfg.product], E,
                   int(cfg.normalise), os.cpu_count() or 1], np.int32)
    sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff, cfg.tarn_total,
                   cfg.tarn_multiplier], np.float64)
    if double:
        A = np.ascontiguousarray(m.A64)
        fixed = np.ascontiguousarray(-0.5 * (A ** 2).sum(-1))
    else:
        A, fixed = m.A, m.fixed
    tau = m.taus.astype(R)
    disp = m.disp.astype(R)
    f0 = m.f0.astype(R)
    lf0 = np.log(f0 + disp).astype(R)
    vars_ = np.zeros((E, 3, P), R)
    ex = np.zeros((E, P), R)
    cf = np.zeros((E, P), R)
    num = np.zeros((E, P), R)
    payoff = np.zeros(P)
    ex_steps = np.ascontiguousarray(m.ex_steps.astype(np.int32))
    orc("orc_pipeline_rule_d" if double else "orc_pipeline_rule_f", si, sd, m.directions,
        m.scramblers, A, fixed, tau, disp, f0, lf0, ex_steps, m.nvars, m.mono, m.nbasis, 1, beta,
        means, sds, vars_, ex, cf, num, payoff, D, cuts, shifts)
    return payoff


@pytest.fixture(scope="module")
def nested_swaption(cuda):
    from dataclasses import replace

    from useful_code_b200.pricer import Pipeline, Selector

    cfg = mk.make_config("c2")
    cfg = replace(cfg, n=12, F=3, f0=np.linspace(0.04, 0.06, 12).astype(np.float32),
                  paths=1 << 14, reg_paths=1 << 14)
    m = mk.build_market(cfg)
    pipe = Pipeline(m)
    ls = pipe.first_pass(1 << 14, 0, "fused")
    res = pipe.regress_nested(ls, Selector.production(3, min_paths=300))
    return m, pipe, ls, res


@pytest.mark.parametrize("basis", ["cross", "quadratic"])
@pytest.mark.parametrize("depth", [2, 4])
def test_nested_regression_one_date_first_pass(cuda, orc, basis, depth):
    """Cross and quadratic bases on first-pass data (2^14 paths), each of
    four exercise dates as a one-date problem, production selector with 300
    paths minimum: tight parity of every nested regression."""
    from dataclasses import replace

    from useful_code_b200.pricer import Pipeline

    cfg = replace(mk.make_config("c2"), n=12, F=3,
                  f0=np.linspace(0.04, 0.06, 12).astype(np.float32), paths=1 << 14,
                  reg_paths=1 << 14, basis=basis)
    m = mk.build_market(cfg)
    pipe = Pipeline(m)
    ls = pipe.first_pass(1 << 14, 0, "fused")
    arrs = [t.cpu().numpy() for t in (ls.vars, ls.cf, ls.ex, ls.num)]
    lf = 0.1 ** (1.0 / (depth - 1))
    select = (depth, lf, lf * 1.01, 2.5, 0.8, 300)
    for e in (0, 3, 6, 9):
        sl = slice(e, e + 1)
        vars32, cf32, ex32, num32 = (np.ascontiguousarray(a[sl]) for a in arrs)
        nvars = np.ascontiguousarray(m.nvars[sl])
        mono = np.ascontiguousarray(m.mono[sl])
        nb = np.ascontiguousarray(m.nbasis[sl])
        g = gpu_nested(vars32, cf32, ex32, num32, nvars, mono, nb, select)
        o = oracle_nested(orc, vars32, cf32, ex32, num32, nvars, mono, nb, select)
        check_nested(g, o, vars32, mono, nb, depth, min_paths=300, fit_tol=1e-5, ex32=ex32)


@pytest.mark.parametrize("depth", [2, 3, 4])
def test_nested_regression_on_first_pass(nested_swaption, orc, depth):
    """Bermudan swaption (12 semi-annual rates, 3 factors) on 2^14 paths,
    production selector with 300 paths minimum: the device regression
    equals the oracle's on the same first-pass data (price, every cut-off,
    path counts, fits of every regression)."""
    from useful_code_b200.pricer import Selector

    m, pipe, ls, _ = nested_swaption
    E = pipe.E
    res = pipe.regress_nested(ls, Selector.production(depth, min_paths=300))
    vars32 = ls.vars.cpu().numpy()
    cf32, ex32, num32 = (t.cpu().numpy() for t in (ls.cf, ls.ex, ls.num))
    lf = 0.1 ** (1.0 / (depth - 1))
    sel = (depth, lf, lf * 1.01, 2.5, 0.8, 300)
    o = oracle_nested(orc, vars32, cf32, ex32, num32, m.nvars, m.mono, m.nbasis, sel)
    cuts = res.cuts.cpu().numpy()
    assert (int(res.status.item()) & ~4) == 0
    assert abs(float(res.price.item()) - o["price"]) < 2e-6
    np.testing.assert_allclose(cuts[:, :-1], o["cuts"][:, :-1], rtol=1e-5, atol=1e-9)
    npaths = res.npaths.cpu().numpy()
    assert (npaths[:, 0] == 1 << 14).all()
    assert (npaths[:, 1] > 300).sum() >= E // 2  # most dates nest
    g = dict(beta=res.beta.cpu().numpy(), means=res.means.cpu().numpy().astype(np.float64),
             sds=res.sds.cpu().numpy().astype(np.float64))
    for e in range(E):
        for d in range(depth):
            if d > 0 and cuts[e, d - 1, 1] == 0.0:
                continue
            fg = fits(g, vars32, m.mono, m.nbasis, e, d)
            fo = fits(o, vars32, m.mono, m.nbasis, e, d)
            assert np.max(np.abs(fg - fo)) < 1e-5 * max(np.abs(fo).max(), 1e-3), (e, d)


def test_nested_rule_on_stored_paths(nested_swaption, orc):
    """The frozen depth-3 rule applied to the regression paths' stored inputs
    (lmm_ls_apply_rule_nested) equals the oracle's chain on the same inputs
    and reproduces the in-sample estimate of the backward induction."""
    m, pipe, ls, res = nested_swaption
    E = pipe.E
    vars32 = ls.vars.cpu().numpy()
    cf32, ex32, num32 = (t.cpu().numpy() for t in (ls.cf, ls.ex, ls.num))
    # the frozen rule on the regression paths (stored inputs) gives the
    # in-sample estimate of the backward induction (same decisions)
    import torch

    from useful_code_b200.pricer import rule_struct

    P = 1 << 14
    pay = torch.empty(P, device="cuda")
    rs = rule_struct(res)
    call("lmm_ls_apply_rule_nested", E, P, dptr(ls.vars), hptr(pipe._nvars), hptr(pipe._mono),
         hptr(pipe._nbasis), dptr(ls.cf), dptr(ls.ex), dptr(ls.num), ctypes.addressof(rs),
         dptr(pay), None)
    beta, means, sds, cutsd, _ = _pipeline_rule(m, res, E)
    ref = orc("orc_ls_second_pass_multi_d", E, P, vars32.astype(np.float64), m.nvars, m.mono,
              m.nbasis, cf32.astype(np.float64), ex32.astype(np.float64),
              num32.astype(np.float64), res.depth, beta, means, sds, cutsd, None,
              restype=ctypes.c_double)
    assert abs(float(pay.double().mean().item()) - ref) < 2e-6
    assert abs(ref - float(res.price.item())) < 1e-4


@pytest.mark.parametrize("mode", ["staged", "fused", "tensor"])
def test_nested_rule_second_pass(nested_swaption, mode):
    """Fresh paths priced with the frozen depth-3 rule and Andersen shifts
    by every evolution mode, against the FP32 oracle path by path and the
    FP64 oracle within 0.05 bp."""
    import torch

    m, pipe, ls, res = nested_swaption
    E = pipe.E
    P = 1 << 13
    res.shifts = torch.linspace(0.0, 4e-4, E, device="cuda")
    try:
        pay = pipe.second_pass(P, 1 << 14, res, mode).cpu().numpy().astype(np.float64)
        beta, means, sds, cuts, shifts = _pipeline_rule(m, res, E)
    finally:
        res.shifts = None
    p32 = oracle_pipeline_rule(m, P, 1 << 14, beta, means, sds, cuts, shifts, res.depth)
    p64 = oracle_pipeline_rule(m, P, 1 << 14, beta, means, sds, cuts, shifts, res.depth,
                               double=True)
    tol = 2e-5 if mode == "tensor" else 2e-6
    assert np.mean(np.abs(pay - p32) < tol) > 0.995
    assert abs(pay.mean() - p64.mean()) * 1e4 < 0.05
    # the shifts move decisions: without them the value differs
    plain = pipe.second_pass(P, 1 << 14, res, mode).cpu().numpy().astype(np.float64)
    assert np.any(np.abs(plain - pay) > 1e-6)


def test_depth_one_rule_equals_plain_rule(nested_swaption):
    """A nested regression of depth 1 is the plain regression."""
    from useful_code_b200.pricer import Selector

    m, pipe, ls, res = nested_swaption
    one = pipe.regress_nested(ls, Selector(depth=1))
    plain = pipe.regress(ls)
    b1 = one.beta.cpu().numpy()[:, 0, :]
    b0 = plain.beta.cpu().numpy()
    assert abs(float(one.price.item()) - float(plain.price.item())) < 1e-6
    np.testing.assert_allclose(b1, b0, rtol=1e-6, atol=1e-9)


def test_nested_regression_graph_replay(nested_swaption):
    """The nested regression captured as a CUDA graph (its launches carry no
    host synchronisation) and replayed twice gives the direct call's rule
    bit for bit: coefficients, cut-offs, paths per depth, in-sample price."""
    import torch

    from useful_code_b200.pricer import Selector

    m, pipe, ls, res = nested_swaption
    sel = Selector.production(3, min_paths=300)
    graph, out = pipe.regress_nested_graph(ls, sel)
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(out.beta, res.beta) and torch.equal(out.cuts, res.cuts)
        assert torch.equal(out.npaths, res.npaths) and torch.equal(out.price, res.price)
        assert int(out.status.item()) == int(res.status.item())
