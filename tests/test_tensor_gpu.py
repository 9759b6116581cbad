"""The tensor-core evolution (LMM_MODE_TENSOR: drift and correlation
contractions on tcgen05 in split FP16) against the CUDA-core fused form and
the FP64 oracle (GPU).  The contractions change the order of the sums, not
the model, so rates agree with the FP64 oracle to the same 2e-5 bar and
prices to 0.05 bp."""
import ctypes

import numpy as np
import pytest

from test_pipeline_gpu import mini, oracle_pipeline, var_err
from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu


def device_errors():
    from useful_code_b200._lib import LIB

    f = ctypes.c_uint(0)
    assert LIB.lmm_device_error_flags(1, ctypes.byref(f)) == 0
    return f.value


@pytest.mark.parametrize("product,n,F", [("swaption", 12, 3), ("swaption", 40, 5),
                                         ("cancellable", 12, 3), ("swaption", 80, 10)])
def test_first_pass_matches_fused_and_fp64(cuda, product, n, F):
    from useful_code_b200.pricer import Pipeline

    kw = {}
    if n == 80:
        kw = dict(f0=mk.quadratic_curve(80, 0.25, 2024), tau=0.25)
    m = mk.build_market(mini(product, n=n, F=F, **kw))
    pipe = Pipeline(m)
    P = 4096
    a = pipe.first_pass(P, 0, "fused")
    b = pipe.first_pass(P, 0, "tensor")
    assert device_errors() == 0
    assert np.max(var_err(b.vars.cpu().numpy(), a.vars.cpu().numpy())) < 5e-5
    assert np.max(np.abs(b.num.cpu().numpy() / a.num.cpu().numpy() - 1)) < 2e-6
    v, ex, cf, num, _ = oracle_pipeline(m, P, 0, 0, double=True)
    got = b.vars.cpu().numpy().astype(np.float64)
    d = float(m.disp[0])
    assert np.max(np.abs(got[:, 0] - v[:, 0]) / (v[:, 0] + d)) < 2e-5
    assert np.max(np.abs(b.num.cpu().numpy() / num - 1)) < 2e-5
    assert np.max(np.abs(b.cf.cpu().numpy() - cf)) < 1e-6


def test_second_pass_and_price(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("swaption"))
    pipe = Pipeline(m)
    P = 4096
    rule = pipe.regress(pipe.first_pass(P, 0, "fused"))
    a = pipe.second_pass(P, P, rule, "fused").cpu().numpy()
    b = pipe.second_pass(P, P, rule, "tensor").cpu().numpy()
    assert device_errors() == 0
    assert np.mean(np.abs(a - b) > 1e-6) < 0.01
    assert abs(a.mean() - b.mean()) < 2e-6
    ra = pipe.price(P, P, "fused")["price"]
    rb = pipe.price(P, P, "tensor")["price"]
    assert abs(ra - rb) * 1e4 < 0.05


def test_european_strip(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("european", n=20, F=3))
    pipe = Pipeline(m)
    P = 8192
    a = pipe.second_pass(P, 0, None, "fused").cpu().numpy()
    b = pipe.second_pass(P, 0, None, "tensor").cpu().numpy()
    *_, pay64 = oracle_pipeline(m, P, 0, 1, double=True)
    assert device_errors() == 0
    assert np.max(np.abs(a - b)) < 2e-6
    assert abs(b.mean() - pay64.mean()) * 1e4 < 0.05


def test_batches_are_additive(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini("swaption"))
    pipe = Pipeline(m)
    whole = pipe.first_pass(4096, 7, "tensor")
    parts = pipe.first_pass(4096, 7, "tensor", batch=1024)
    for x, y in zip((whole.vars, whole.ex, whole.cf, whole.num),
                    (parts.vars, parts.ex, parts.cf, parts.num)):
        assert np.array_equal(x.cpu().numpy(), y.cpu().numpy())
