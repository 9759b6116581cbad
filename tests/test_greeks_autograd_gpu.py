"""The adjoint Greeks behind torch.autograd (GPU; test harness only).

`FrozenRulePrice` is a torch.autograd.Function over the frozen-rule price
V(f0, A) of a pipeline: its forward writes the initial forwards and the
pseudo-roots (and their fixed drifts) into the pipeline's model and calls
lmm_greeks through the C ABI; its backward returns the adjoint's deltas and
dV/dA scaled by the incoming gradient.  The tests drive it with
torch.autograd.grad through composed maps and compare with central
differences of the FP64 frozen-exercise price (test_greeks_gpu.Frozen).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _set_point(pipe, f0, A):
    """Write (f0, A) and A's fixed drifts into the pipeline's model."""
    import torch

    from useful_code_b200._lib import call

    m = pipe.mkt
    n, F = m.cfg.n, m.cfg.F
    pipe._f0[:] = np.asarray(f0, np.float32)
    A32 = np.ascontiguousarray(np.asarray(A, np.float32))
    fixed = np.zeros((n, n), np.float32)
    call("lmm_fixed_drifts", ctypes.c_void_p(A32.ctypes.data), n, n, F,
         ctypes.c_void_p(fixed.ctypes.data))
    pipe.A.copy_(torch.from_numpy(A32))
    pipe.fixed.copy_(torch.from_numpy(fixed))


def _frozen_rule_price_fn():
    import torch

    class FrozenRulePrice(torch.autograd.Function):
        """V(f0, A) under a frozen exercise rule; gradients by lmm_greeks."""

        @staticmethod
        def forward(ctx, f0, A, pipe, rule, paths, offset):
            _set_point(pipe, f0.detach().cpu().numpy(), A.detach().cpu().numpy())
            g = pipe.greeks(paths, offset, rule, checkpoint_every=4)
            ctx.save_for_backward(torch.from_numpy(g.delta), torch.from_numpy(g.abar))
            ctx.shape_A = A.shape
            return torch.tensor(g.price, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad):
            delta, abar = ctx.saved_tensors
            return grad * delta, grad * abar.reshape(ctx.shape_A), None, None, None, None

    return FrozenRulePrice


@pytest.fixture(scope="module")
def harness(cuda):
    from test_greeks_gpu import Frozen, setup

    m, pipe, rule, P = setup("swaption")
    g = pipe.greeks(P, P, rule, checkpoint_every=4)
    fz = Frozen(m, P, P, g.exercise_step)
    # the pipeline's model may share the market's f0 array: keep the base
    base_f0 = m.f0.copy()
    yield m, pipe, rule, P, g, fz
    _set_point(pipe, base_f0, m.A)


def test_autograd_matches_the_adjoint_and_fd(harness):
    """d(V^2)/d(alpha, beta) through f0 = f0 + alpha d and A = A (1 + beta D):
    2 V (delta . d) and 2 V sum(dV/dA A D) from autograd equal the adjoint's
    own numbers and the FP64 central differences along the same directions."""
    import torch

    m, pipe, rule, P, g, fz = harness
    Fn = _frozen_rule_price_fn()
    rng = np.random.default_rng(23)
    d = torch.from_numpy(rng.uniform(-1.0, 1.0, m.cfg.n))
    D = torch.from_numpy(rng.uniform(-1.0, 1.0, m.A64.shape))
    A0 = torch.from_numpy(m.A64)
    f00 = torch.from_numpy(m.f0.astype(np.float64))
    alpha = torch.zeros((), dtype=torch.float64, requires_grad=True)
    beta = torch.zeros((), dtype=torch.float64, requires_grad=True)
    V = Fn.apply(f00 + alpha * d, A0 * (1.0 + beta * D), pipe, rule, P, P)
    ga, gb = torch.autograd.grad(V * V, (alpha, beta))
    v = float(V.detach())
    assert v == g.price
    dn = d.numpy()
    DA = m.A64 * D.numpy()
    assert abs(float(ga) - 2 * v * float(g.delta @ dn)) < 1e-12 * abs(float(ga)) + 1e-15
    assert abs(float(gb) - 2 * v * float(np.sum(g.abar * DA))) < 1e-12 * abs(float(gb)) + 1e-15
    h = 1e-5
    fd_a = (fz.price(f0=m.f0.astype(np.float64) + h * dn) -
            fz.price(f0=m.f0.astype(np.float64) - h * dn)) / (2 * h)
    fd_b = fz.along(DA)
    assert abs(float(ga) / (2 * v) - fd_a) < 2e-4 * abs(fd_a) + 1e-9, (float(ga) / (2 * v), fd_a)
    assert abs(float(gb) / (2 * v) - fd_b) < 2e-4 * abs(fd_b) + 1e-9, (float(gb) / (2 * v), fd_b)


def test_autograd_away_from_the_base_point(harness):
    """The forward evaluated at a moved point (f0 + 1e-4 d, A (1 + 1e-3 D)).
    The rule, not the exercise steps, is frozen, so some paths exercise at
    other steps there and the price is not the base price plus a first-order
    term; with the exercise steps the GPU takes at the moved point, the FP64
    frozen-exercise price there equals the Function's value, and its central
    differences along f0 and A directions equal the gradient autograd
    returns there."""
    import torch

    from test_greeks_gpu import Frozen

    m, pipe, rule, P, g, fz = harness
    Fn = _frozen_rule_price_fn()
    rng = np.random.default_rng(29)
    dn = rng.uniform(-1.0, 1.0, m.cfg.n)
    Dn = rng.uniform(-1.0, 1.0, m.A64.shape)
    f0m = m.f0.astype(np.float64) + 1e-4 * dn
    Am = m.A64 * (1.0 + 1e-3 * Dn)
    f0 = torch.tensor(f0m, requires_grad=True)
    A = torch.tensor(Am, requires_grad=True)
    V = Fn.apply(f0, A, pipe, rule, P, P)
    gf, gA = torch.autograd.grad(V, (f0, A))
    gm = pipe.greeks(P, P, rule, checkpoint_every=4)  # the same (moved) point
    assert gm.price == float(V.detach())
    # the FP64 oracle at the moved point: its inputs are the FP32 values the
    # GPU evaluated
    f0_32 = f0m.astype(np.float32).astype(np.float64)
    A_32 = Am.astype(np.float32).astype(np.float64)
    fzm = Frozen(m, P, P, gm.exercise_step)
    assert abs(fzm.price(f0=f0_32, A=A_32) - gm.price) < 2e-6 * abs(gm.price) + 1e-9
    h = 1e-5
    d2 = rng.uniform(-1.0, 1.0, m.cfg.n)
    fd_f = (fzm.price(f0=f0_32 + h * d2, A=A_32) - fzm.price(f0=f0_32 - h * d2, A=A_32)) / (2 * h)
    ad_f = float(gf.numpy() @ d2)
    assert abs(ad_f - fd_f) < 2e-4 * abs(fd_f) + 1e-9, (ad_f, fd_f)
    D2 = A_32 * rng.uniform(-1.0, 1.0, m.A64.shape)
    fd_A = (fzm.price(f0=f0_32, A=A_32 + h * D2) - fzm.price(f0=f0_32, A=A_32 - h * D2)) / (2 * h)
    ad_A = float(np.sum(gA.numpy() * D2))
    assert abs(ad_A - fd_A) < 2e-4 * abs(fd_A) + 1e-9, (ad_A, fd_A)
