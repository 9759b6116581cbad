"""Pathwise adjoint Greeks (lmm_greeks) against central finite differences
(GPU).

The adjoint differentiates the frozen-rule price with each path's exercise
step held fixed.  The reference function is the same price evaluated by the
FP64 oracle on the same Sobol points with the exercise steps the GPU
recorded (orc_frozen_payoff_d), bumped by 1e-5 and differenced centrally:
initial forwards (deltas), row scalings of the pseudo-roots (per-rate
vegas), a random direction in the pseudo-root entries (the whole dV/dA) and
the abcd parameters through the host chain rule (lmm_abcd_vegas).
"""
import ctypes
import os
from dataclasses import replace

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu

H = 1e-5  # bump size of the finite differences


def mini(product="swaption", n=12, F=3, **kw):
    base = {"swaption": "c2", "cancellable": "c5", "european": "c1"}[product]
    cfg = mk.make_config(base)
    f0 = np.linspace(0.04, 0.06, n).astype(np.float32)
    args = dict(n=n, F=F, f0=f0, paths=4096, reg_paths=4096)
    args.update(kw)
    return replace(cfg, **args)


class Frozen:
    """FP64 price of the frozen-exercise payoff, with bumpable f0 and A."""

    def __init__(self, m, P, offset, exercise_step):
        import sys

        sys.path.insert(0, os.path.dirname(__file__))
        from conftest import CLib, _ensure_oracle

        self.orc = CLib(_ensure_oracle())
        self.m, self.P, self.offset = m, P, offset
        cfg = m.cfg
        E = len(m.ex_steps)
        pos = {int(s): e for e, s in enumerate(m.ex_steps)}
        self.ex_at = np.array([pos.get(int(s), E) for s in exercise_step], np.int32)
        self.si = np.array([cfg.n, cfg.F, P, offset, m.scramble_dims, mk.PRODUCTS[cfg.product],
                            E, int(cfg.normalise), os.cpu_count() or 1], np.int32)
        self.sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff], np.float64)

    def price(self, f0=None, A=None):
        m = self.m
        f0 = (m.f0.astype(np.float64) if f0 is None else f0).copy()
        A = np.ascontiguousarray(m.A64 if A is None else A)
        fixed = np.ascontiguousarray(-0.5 * (A ** 2).sum(-1))
        tau = m.taus.astype(np.float64)
        disp = m.disp.astype(np.float64)
        lf0 = np.log(f0 + disp)
        pay = np.zeros(self.P)
        self.orc("orc_frozen_payoff_d", self.si, self.sd, m.directions, m.scramblers, A, fixed,
                 tau, disp, f0, lf0, np.ascontiguousarray(m.ex_steps.astype(np.int32)),
                 self.ex_at, pay)
        return pay.mean() / (1.0 + f0[0] * float(m.rate_times[0]))

    def delta(self, r):
        up = self.m.f0.astype(np.float64).copy()
        dn = up.copy()
        up[r] += H
        dn[r] -= H
        return (self.price(f0=up) - self.price(f0=dn)) / (2 * H)

    def along(self, D):
        A = self.m.A64
        return (self.price(A=A + H * D) - self.price(A=A - H * D)) / (2 * H)


def setup(product, **kw):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini(product, **kw))
    pipe = Pipeline(m)
    P = 4096
    rule = None
    if product != "european":
        rule = pipe.regress(pipe.first_pass(P, 0, "fused"))
    return m, pipe, rule, P


@pytest.fixture(scope="module")
def swaption(cuda):
    m, pipe, rule, P = setup("swaption")
    g = pipe.greeks(P, P, rule, checkpoint_every=4)
    return m, pipe, rule, P, g, Frozen(m, P, P, g.exercise_step)


def close(got, ref, rel):
    got, ref = np.asarray(got), np.asarray(ref)
    scale = max(np.max(np.abs(ref)), 1e-12)
    err = np.max(np.abs(got - ref)) / scale
    assert err < rel, (err, got, ref)


def test_price_matches_second_pass(swaption):
    m, pipe, rule, P, g, fz = swaption
    pay = pipe.second_pass(P, P, rule, "fused").cpu().numpy().astype(np.float64)
    assert abs(g.price - pay.mean() * m.initial_numeraire) < 1e-9 * abs(g.price) + 1e-12
    # the FP64 frozen-exercise price on the same points agrees to FP32 accuracy
    assert abs(fz.price() - g.price) < 2e-6 * abs(g.price) + 1e-9


def test_deltas_vs_fd(swaption):
    m, pipe, rule, P, g, fz = swaption
    fd = np.array([fz.delta(r) for r in range(m.cfg.n)])
    close(g.delta, fd, 2e-4)


def test_rate_vegas_vs_fd(swaption):
    m, pipe, rule, P, g, fz = swaption
    fd = []
    for r in range(m.cfg.n):
        D = np.zeros_like(m.A64)
        D[:, r, :] = m.A64[:, r, :]
        fd.append(fz.along(D))
    close(g.vega_rate, np.array(fd), 2e-4)


def test_abar_random_direction(swaption):
    m, pipe, rule, P, g, fz = swaption
    rng = np.random.default_rng(17)
    for _ in range(2):
        D = m.A64 * rng.uniform(-1.0, 1.0, m.A64.shape)
        fd = fz.along(D)
        ad = float(np.sum(g.abar * D))
        assert abs(ad - fd) < 2e-4 * abs(fd) + 1e-9, (ad, fd)


def test_abcd_vegas_vs_fd(swaption):
    from useful_code_b200._lib import LIB

    m, pipe, rule, P, g, fz = swaption
    cfg = m.cfg
    a, b, c, d = cfg.abcd
    times = np.ascontiguousarray(m.rate_times[:cfg.n].astype(np.float64))
    mult = np.ones(cfg.n)
    out = np.zeros(4)
    abar = np.ascontiguousarray(g.abar)
    vp = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    st = LIB.lmm_abcd_vegas(a, b, c, d, vp(times), cfg.n, vp(times), cfg.n, vp(mult), cfg.F,
                            cfg.L, cfg.beta, vp(abar), 1e-5, vp(out))
    assert st == 0
    fd = []
    for k in range(4):
        h = 1e-5 * max(abs(cfg.abcd[k]), 1e-3)
        prices = []
        for sgn in (1, -1):
            p = list(cfg.abcd)
            p[k] += sgn * h
            A = mk.pseudo_roots(replace(cfg, abcd=tuple(p)), m.rate_times)
            prices.append(fz.price(A=A))
        fd.append((prices[0] - prices[1]) / (2 * h))
    close(out, np.array(fd), 5e-4)


def test_checkpoint_interval_invariance(swaption):
    """Intervals giving twelve, three, two and one checkpoint segments (the
    recompute of later segments runs ahead of the reverse sweep on a stream
    of its own, two segments at most)."""
    m, pipe, rule, P, g, fz = swaption
    for k in (1, 5, 6, m.cfg.n):
        h = pipe.greeks(P, P, rule, checkpoint_every=k)
        np.testing.assert_allclose(h.delta, g.delta, rtol=1e-7, atol=1e-12)
        np.testing.assert_allclose(h.abar, g.abar, rtol=1e-6, atol=1e-12)
        assert h.price == g.price


@pytest.mark.parametrize("product", ["cancellable", "european"])
def test_other_products_deltas(cuda, product):
    m, pipe, rule, P = setup(product)
    g = pipe.greeks(P, P, rule, checkpoint_every=3)
    fz = Frozen(m, P, P, g.exercise_step)
    assert abs(fz.price() - g.price) < 2e-6 * abs(g.price) + 1e-9
    fd = np.array([fz.delta(r) for r in range(m.cfg.n)])
    close(g.delta, fd, 2e-4)
    rng = np.random.default_rng(5)
    D = m.A64 * rng.uniform(-1.0, 1.0, m.A64.shape)
    fdv = fz.along(D)
    assert abs(float(np.sum(g.abar * D)) - fdv) < 2e-4 * abs(fdv) + 1e-9


def test_concurrent_calls_from_two_threads(swaption):
    """lmm_greeks called at the same time from two host threads, each on a
    stream and workspace of its own (each thread then runs on its own pair
    of the library's internal streams), three calls each: every result
    equals the single-threaded call bit for bit."""
    import threading

    import torch

    from useful_code_b200._lib import LIB, call

    m, pipe, rule, P, g, fz = swaption
    n, F = m.cfg.n, m.cfg.F
    m_addr, p_addr = ctypes.addressof(pipe.model), ctypes.addressof(pipe.product)
    nbytes = LIB.lmm_greeks_workspace_bytes(m_addr, p_addr, P, 4)
    dp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    results, errors = [], []

    def work():
        try:
            torch.cuda.set_device(0)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
                price = torch.zeros(1, dtype=torch.float64, device="cuda")
                delta = torch.zeros(n, dtype=torch.float64, device="cuda")
                abar = torch.zeros(n * n * F, dtype=torch.float64, device="cuda")
                status = torch.zeros(1, dtype=torch.int32, device="cuda")
                for _ in range(3):
                    call("lmm_greeks", m_addr, p_addr, P, P, dp(rule.beta), dp(rule.means),
                         dp(rule.sds), float(m.rate_times[0]), 4, dp(ws), ws.numel(),
                         dp(price), dp(delta), dp(abar), None, None, dp(status),
                         ctypes.c_void_p(st.cuda_stream))
            st.synchronize()
            results.append((float(price.item()), delta.cpu().numpy(), abar.cpu().numpy(),
                            int(status.item())))
        except Exception as exc:  # re-raised in the test's thread
            errors.append(exc)

    threads = [threading.Thread(target=work) for _ in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert len(results) == 2
    for price, delta, abar, status in results:
        assert status == 0
        assert price == g.price
        np.testing.assert_array_equal(delta, g.delta)
        np.testing.assert_array_equal(abar, g.abar.reshape(-1))


def test_bad_arguments(swaption):
    from useful_code_b200._lib import LmmError

    m, pipe, rule, P, g, fz = swaption
    with pytest.raises(LmmError):
        pipe.greeks(4094, P, rule)  # not a multiple of 4


@pytest.mark.parametrize("F", [1, 4])
def test_generic_factor_counts(cuda, F):
    """Factor counts without their own kernel instantiation (the generic
    kernels, rows padded for 16 factors): deltas and a random dV/dA
    direction against the FP64 frozen-exercise differences."""
    m, pipe, rule, P = setup("swaption", F=F)
    g = pipe.greeks(P, P, rule, checkpoint_every=5)
    fz = Frozen(m, P, P, g.exercise_step)
    assert abs(fz.price() - g.price) < 2e-6 * abs(g.price) + 1e-9
    fd = np.array([fz.delta(r) for r in range(m.cfg.n)])
    close(g.delta, fd, 2e-4)
    rng = np.random.default_rng(9)
    D = m.A64 * rng.uniform(-1.0, 1.0, m.A64.shape)
    fdv = fz.along(D)
    assert abs(float(np.sum(g.abar * D)) - fdv) < 2e-4 * abs(fdv) + 1e-9


@pytest.mark.parametrize("P", [12, 4100, 8324])
def test_ordered_sweep_ragged_counts(cuda, P):
    """The reverse sweep takes the paths in chunks of 4096 ordered by their
    last step with work, two tiles of 128 positions per thread: path counts
    that leave a short last chunk and a short last tile (12 paths: one
    partial tile; 4100: a chunk of 4 paths; 8324: a chunk of 132, a tile of
    4) against the FP64 frozen-exercise differences, and two calls in a row
    bit-identical (the order and every sum are fixed)."""
    m, pipe, rule, _ = setup("swaption")
    g = pipe.greeks(P, 4096, rule, checkpoint_every=4)
    g2 = pipe.greeks(P, 4096, rule, checkpoint_every=4)
    assert g.price == g2.price
    assert np.array_equal(g.delta, g2.delta) and np.array_equal(g.abar, g2.abar)
    fz = Frozen(m, P, 4096, g.exercise_step)
    assert abs(fz.price() - g.price) < 2e-6 * abs(g.price) + 1e-9
    fd = np.array([fz.delta(r) for r in range(m.cfg.n)])
    close(g.delta, fd, 2e-4)
    rng = np.random.default_rng(P)
    D = m.A64 * rng.uniform(-1.0, 1.0, m.A64.shape)
    fdv = fz.along(D)
    assert abs(float(np.sum(g.abar * D)) - fdv) < 2e-4 * abs(fdv) + 1e-9


@pytest.mark.parametrize("n,F", [(12, 5), (16, 10), (16, 15)])
def test_compiled_factor_counts(cuda, n, F):
    """The factor counts with kernels of their own (5: six CTAs per SM, two
    paths per thread; 10: the bench's shape; 15: one path per thread):
    deltas and a random dV/dA direction against the FP64 frozen-exercise
    differences."""
    m, pipe, rule, P = setup("swaption", n=n, F=F, f0=np.linspace(0.04, 0.06, n).astype(np.float32))
    g = pipe.greeks(P, P, rule, checkpoint_every=5)
    fz = Frozen(m, P, P, g.exercise_step)
    assert abs(fz.price() - g.price) < 2e-6 * abs(g.price) + 1e-9
    fd = np.array([fz.delta(r) for r in range(m.cfg.n)])
    close(g.delta, fd, 2e-4)
    rng = np.random.default_rng(F)
    D = m.A64 * rng.uniform(-1.0, 1.0, m.A64.shape)
    fdv = fz.along(D)
    assert abs(float(np.sum(g.abar * D)) - fdv) < 2e-4 * abs(fdv) + 1e-9
