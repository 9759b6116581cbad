"""lmm_ls_regress_static: the regression entry point that allocates nothing.

Some callers cannot hand the library a workspace: their device memory is
owned by an outside pool allocator, or their pricing loop must not allocate
because allocation can synchronise the device.  For them the library keeps
its own fixed-size scratch in a static device array.  This test calls that
entry point through the C ABI twice in a row and checks each result against
lmm_ls_regress run with a caller workspace on the same inputs.  It sits in a
file of its own that pytest collects last, and passes alone in a fresh
process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def test_static_scratch_regression_matches_workspace_version(cuda):
    import torch

    from useful_code_b200 import market as mk
    from useful_code_b200._lib import LIB, LmmError, call
    from useful_code_b200.pricer import Pipeline, dp

    cfg = mk.make_config("c2", n=16, F=3, f0=np.linspace(0.04, 0.06, 16).astype(np.float32))
    mkt = mk.build_market(cfg)
    pipe = Pipeline(mkt)
    P = 20000
    ls = pipe.first_pass(P, 0, "fused")
    E = pipe.E
    h = lambda a: VP(a.ctypes.data)  # noqa: E731

    def outputs():
        return (torch.zeros(E, 16, dtype=torch.float64, device="cuda"),
                torch.zeros(E, 3, device="cuda"), torch.ones(E, 3, device="cuda"),
                torch.zeros(E, 16, 17, dtype=torch.float64, device="cuda"),
                torch.zeros(1, dtype=torch.int32, device="cuda"),
                torch.zeros(1, dtype=torch.float64, device="cuda"))

    # existing entry point with a caller workspace
    ws = torch.empty(int(LIB.lmm_ls_workspace_bytes(P, E)), dtype=torch.uint8, device="cuda")
    b0, m0, s0, g0, st0, p0 = outputs()
    call("lmm_ls_regress", E, P, dp(ls.vars), h(pipe._nvars), h(pipe._mono), h(pipe._nbasis),
         dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(ws), ws.numel(), dp(b0), dp(m0), dp(s0),
         dp(g0), dp(st0), dp(p0), None)
    torch.cuda.synchronize()

    # the static-scratch entry point, twice in a row
    for _ in range(2):
        b1, m1, s1, g1, st1, p1 = outputs()
        call("lmm_ls_regress_static", E, P, dp(ls.vars), h(pipe._nvars), h(pipe._mono),
             h(pipe._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(b1), dp(m1), dp(s1),
             dp(g1), dp(st1), dp(p1), None)
        torch.cuda.synchronize()
        assert int(st1.item()) == int(st0.item())
        assert abs(float(p1.item()) - float(p0.item())) <= 1e-12 * max(1.0, abs(float(p0.item())))
        np.testing.assert_allclose(b1.cpu().numpy(), b0.cpu().numpy(), rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(g1.cpu().numpy(), g0.cpu().numpy(), rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(m1.cpu().numpy(), m0.cpu().numpy(), rtol=1e-7)
        np.testing.assert_allclose(s1.cpu().numpy(), s0.cpu().numpy(), rtol=1e-7)

    # sizes beyond the static scratch are rejected before any device work
    big = 1 << 22
    with pytest.raises(LmmError) as ei:
        call("lmm_ls_regress_static", E, big, dp(ls.vars), h(pipe._nvars), h(pipe._mono),
             h(pipe._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(b1), dp(m1), dp(s1),
             None, dp(st1), dp(p1), None)
    assert "static scratch" in str(ei.value)


def test_static_scratch_at_its_limit(cuda):
    """The largest regression the static scratch holds (the path count at
    which lmm_ls_workspace_bytes reaches LMM_LS_STATIC_SCRATCH_BYTES for the
    test's 16 dates, about two million paths) matches the workspace version;
    one path more is rejected.  At this size the carried path values and the
    per-CTA partials fill the array, so an error in the size arithmetic
    would show here."""
    import torch

    from useful_code_b200 import market as mk
    from useful_code_b200._lib import LIB, LmmError, call
    from useful_code_b200.pricer import Pipeline, dp

    cfg = mk.make_config("c2", n=16, F=3, f0=np.linspace(0.04, 0.06, 16).astype(np.float32))
    pipe = Pipeline(mk.build_market(cfg))
    E = pipe.E
    limit = 8 << 20
    lo, hi = 1, 1 << 26
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if LIB.lmm_ls_workspace_bytes(mid, E) <= limit:
            lo = mid
        else:
            hi = mid
    P = lo
    assert LIB.lmm_ls_workspace_bytes(P, E) <= limit < LIB.lmm_ls_workspace_bytes(P + 1, E)
    ls = pipe.first_pass(P, 0, "fused")
    h = lambda a: VP(a.ctypes.data)  # noqa: E731

    def outputs():
        return (torch.zeros(E, 16, dtype=torch.float64, device="cuda"),
                torch.zeros(E, 3, device="cuda"), torch.ones(E, 3, device="cuda"),
                torch.zeros(1, dtype=torch.int32, device="cuda"),
                torch.zeros(1, dtype=torch.float64, device="cuda"))

    ws = torch.empty(int(LIB.lmm_ls_workspace_bytes(P, E)), dtype=torch.uint8, device="cuda")
    b0, m0, s0, st0, p0 = outputs()
    call("lmm_ls_regress", E, P, dp(ls.vars), h(pipe._nvars), h(pipe._mono), h(pipe._nbasis),
         dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(ws), ws.numel(), dp(b0), dp(m0), dp(s0), None,
         dp(st0), dp(p0), None)
    b1, m1, s1, st1, p1 = outputs()
    call("lmm_ls_regress_static", E, P, dp(ls.vars), h(pipe._nvars), h(pipe._mono),
         h(pipe._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(b1), dp(m1), dp(s1), None,
         dp(st1), dp(p1), None)
    torch.cuda.synchronize()
    assert int(st1.item()) == int(st0.item())
    assert abs(float(p1.item()) - float(p0.item())) <= 1e-12 * max(1.0, abs(float(p0.item())))
    np.testing.assert_allclose(b1.cpu().numpy(), b0.cpu().numpy(), rtol=1e-10, atol=1e-14)
    with pytest.raises(LmmError) as ei:
        call("lmm_ls_regress_static", E, P + 1, dp(ls.vars), h(pipe._nvars), h(pipe._mono),
             h(pipe._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), 1, dp(b1), dp(m1), dp(s1), None,
             dp(st1), dp(p1), None)
    assert "static scratch" in str(ei.value)
