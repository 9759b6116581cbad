"""Segmented second pass (lmm_fused_price) on the GPU: the chain of segment
launches that drops exercised paths and packs the survivors must give
every path the payoff of the one-launch rule pass (lmm_fused_evolve) bit for
bit, for every segment length, ragged path counts, both stopping products
(Bermudan swaption, cancellable swap), nested rules with Andersen shifts,
and a rule under which no path ever exercises (all survive) or every path
exercises at the first date (none survive)."""
import ctypes
from dataclasses import replace

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def dptr(t):
    return VP(t.data_ptr()) if t is not None else None


def _market(product, n=24, F=3, paths=4096):
    base = "c5" if product == "cancellable" else "c3"
    cfg = replace(mk.make_config(base), n=n, F=F, tau=0.25,
                  f0=np.linspace(0.04, 0.06, n).astype(np.float32), paths=paths,
                  reg_paths=paths)
    return mk.build_market(cfg)


def _both(pipe, P, offset, rule, seg_steps):
    """(one-launch payoffs, segmented payoffs) of the same variates."""
    import torch

    from useful_code_b200._lib import call
    from useful_code_b200.pricer import call_size, rule_struct, stream_handle

    cfg = pipe.mkt.cfg
    m_addr = ctypes.addressof(pipe.model)
    p_addr = ctypes.addressof(pipe.product)
    var = torch.empty(cfg.n * cfg.F * P, device="cuda")
    call("lmm_fused_variates", m_addr, P, offset, dptr(var), stream_handle())
    one = torch.full((P,), np.nan, device="cuda")
    seg = torch.full((P,), np.nan, device="cuda")
    rs = rule_struct(rule)
    # one launch: segment length >= rates
    call("lmm_fused_price", m_addr, p_addr, P, dptr(var), ctypes.byref(rs), cfg.n, None, 0,
         dptr(one), stream_handle())
    ws = torch.empty(max(1, call_size("lmm_fused_price_workspace_bytes", m_addr, p_addr, P)),
                     dtype=torch.uint8, device="cuda")
    call("lmm_fused_price", m_addr, p_addr, P, dptr(var), ctypes.byref(rs), seg_steps,
         dptr(ws), ws.numel(), dptr(seg), stream_handle())
    torch.cuda.synchronize()
    return one.cpu().numpy(), seg.cpu().numpy()


@pytest.fixture(scope="module", params=["swaption", "cancellable"])
def priced(request, cuda):
    from useful_code_b200.pricer import Pipeline

    m = _market(request.param)
    pipe = Pipeline(m)
    rule = pipe.regress(pipe.first_pass(4096, 0, "fused"))
    return pipe, rule


@pytest.mark.parametrize("seg_steps", [0, 1, 3, 8, 23])
@pytest.mark.parametrize("P", [1, 127, 129, 1000, 4096])
def test_segmented_equals_one_launch(priced, P, seg_steps):
    pipe, rule = priced
    one, seg = _both(pipe, P, 9000, rule, seg_steps)
    assert np.all(np.isfinite(one))
    np.testing.assert_array_equal(seg, one)


def test_segmented_one_launch_equals_fused_evolve(priced):
    """lmm_fused_price with one segment is lmm_fused_evolve's rule pass."""
    import torch

    from useful_code_b200._lib import call
    from useful_code_b200.pricer import stream_handle

    pipe, rule = priced
    cfg = pipe.mkt.cfg
    P = 1000
    m_addr = ctypes.addressof(pipe.model)
    p_addr = ctypes.addressof(pipe.product)
    var = torch.empty(cfg.n * cfg.F * P, device="cuda")
    call("lmm_fused_variates", m_addr, P, 77, dptr(var), stream_handle())
    ref = torch.empty(P, device="cuda")
    call("lmm_fused_evolve", m_addr, p_addr, P, dptr(var), dptr(rule.beta), dptr(rule.means),
         dptr(rule.sds), P, 0, None, None, None, None, dptr(ref), stream_handle())
    _, seg = _both(pipe, P, 77, rule, 0)
    np.testing.assert_array_equal(seg, ref.cpu().numpy())


def test_segmented_nested_rule_with_shifts(cuda):
    import torch

    from useful_code_b200.pricer import Pipeline, Selector

    m = _market("swaption", n=20, F=5, paths=1 << 14)
    pipe = Pipeline(m)
    rule = pipe.regress_nested(pipe.first_pass(1 << 14, 0, "fused"),
                               Selector.production(3, min_paths=300))
    rng = np.random.default_rng(5)
    rule.shifts = torch.as_tensor(rng.normal(0, 1e-3, pipe.E).astype(np.float32),
                                  device="cuda")
    one, seg = _both(pipe, 3000, 1 << 15, rule, 4)
    np.testing.assert_array_equal(seg, one)


@pytest.mark.parametrize("shift", [1e3, -1e3])
def test_segmented_all_or_no_survivors(cuda, shift):
    """A large positive shift keeps every path alive to the end (payoff 0);
    a large negative one exercises every path at the first date, so no path
    survives the first segment."""
    import torch

    from useful_code_b200.pricer import Pipeline

    m = _market("swaption")
    pipe = Pipeline(m)
    rule = pipe.regress(pipe.first_pass(4096, 0, "fused"))
    rule.shifts = torch.full((pipe.E,), shift, dtype=torch.float32, device="cuda")
    one, seg = _both(pipe, 2000, 5000, rule, 2)
    np.testing.assert_array_equal(seg, one)
    if shift > 0:
        assert np.all(one == 0.0)


def test_pipeline_second_pass_uses_segments(cuda):
    """The fused pipeline second pass (segmented) equals the staged pass
    path by path within FP32 noise, as the one-launch kernel does."""
    from useful_code_b200.pricer import Pipeline

    m = _market("swaption")
    pipe = Pipeline(m)
    rule = pipe.regress(pipe.first_pass(4096, 0, "fused"))
    fused = pipe.second_pass(4096, 4096, rule, "fused").cpu().numpy()
    staged = pipe.second_pass(4096, 4096, rule, "staged").cpu().numpy()
    close = np.abs(fused - staged) < 2e-6
    assert close.mean() > 0.99
