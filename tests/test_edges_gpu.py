"""Edge cases of the pipeline on the GPU against the CPU oracle: path counts
that are not multiples of the kernels' blocks (1, 127, 129, 1000), the
smallest model (2 rates, 1 factor) and the largest (128 rates, 16 factors,
2,048 Sobol dimensions), and a regression with fewer paths than basis
functions (singular Gram: the solve reports the jitter or the failure in
its status and the price stays finite)."""
from dataclasses import replace

import numpy as np
import pytest

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu


def market(base, n, F, paths=4096, **kw):
    cfg = replace(mk.make_config(base), n=n, F=F,
                  f0=np.linspace(0.04, 0.06, n).astype(np.float32), paths=paths,
                  reg_paths=paths, **kw)
    return mk.build_market(cfg)


def var_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 0.01)


@pytest.mark.parametrize("P", [1, 127, 129, 1000])
@pytest.mark.parametrize("mode", ["staged", "fused", "tensor"])
def test_ragged_path_counts(cuda, P, mode):
    """First pass and frozen-rule second pass at ragged path counts: the LS
    inputs equal the FP32 oracle's path by path, and the second-pass payoffs
    too (a few decisions may flip at the FP32 margin)."""
    from test_pipeline_gpu import oracle_pipeline
    from useful_code_b200.pricer import Pipeline

    m = market("c2", 12, 3)
    pipe = Pipeline(m)
    ls = pipe.first_pass(P, 5, mode)
    v, ex, cf, num, _ = oracle_pipeline(m, P, 5, 0)
    tol = 2e-4 if mode == "tensor" else 5e-5
    assert np.max(var_err(ls.vars.cpu().numpy(), v)) < tol
    assert np.max(np.abs(ls.num.cpu().numpy() - num) / num) < tol
    # a rule from a full-size regression, applied to the ragged batch
    rule = pipe.regress(pipe.first_pass(4096, 100000, "fused"))
    pay = pipe.second_pass(P, 7, rule, mode).cpu().numpy()
    *_, pay32 = oracle_pipeline(m, P, 7, 1, rule)
    close = np.abs(pay - pay32) < (2e-5 if mode == "tensor" else 2e-6)
    assert close.mean() >= (0.99 if P >= 100 else 1.0) - 1e-12


@pytest.mark.parametrize("mode", ["staged", "fused", "tensor"])
def test_smallest_model(cuda, mode):
    """Two semi-annual rates, one factor, exercise at both resets."""
    from test_pipeline_gpu import oracle_pipeline
    from useful_code_b200.pricer import Pipeline

    m = market("c2", 2, 1, paths=1024)
    pipe = Pipeline(m)
    ls = pipe.first_pass(1024, 0, mode)
    v, ex, cf, num, _ = oracle_pipeline(m, 1024, 0, 0)
    assert np.max(var_err(ls.vars.cpu().numpy(), v)) < 5e-5
    res = pipe.price(1024, 1024, mode)
    assert np.isfinite(res["price"]) and res["price"] > 0


@pytest.mark.parametrize("mode", ["fused", "tensor"])
def test_largest_model(cuda, mode):
    """128 quarterly rates, 16 factors (the library's maximum): 2,048 Sobol
    dimensions, the fused and tensor-core evolutions against the oracle."""
    from test_pipeline_gpu import oracle_pipeline
    from useful_code_b200.pricer import Pipeline

    m = market("c3", 128, 16, paths=256, tau=0.25)
    pipe = Pipeline(m)
    ls = pipe.first_pass(256, 0, mode)
    v, ex, cf, num, _ = oracle_pipeline(m, 256, 0, 0)
    tol = 2e-4 if mode == "tensor" else 1e-4
    assert np.max(var_err(ls.vars.cpu().numpy(), v)) < tol
    assert np.max(np.abs(ls.num.cpu().numpy() - num) / num) < tol


def test_regression_with_fewer_paths_than_basis_functions(cuda):
    """8 paths for the 10-function cross basis: the normal equations are
    singular; the Cholesky adds jitter or gives up (status bits 4 / 2), and
    the in-sample price stays finite."""
    from useful_code_b200.pricer import Pipeline

    m = market("c3", 12, 3, paths=8)
    pipe = Pipeline(m)
    ls = pipe.first_pass(8, 0, "fused")
    rule = pipe.regress(ls)
    st = int(rule.status.item())
    assert st & (2 | 4), st
    assert np.isfinite(float(rule.price.item()))
    assert np.all(np.isfinite(rule.beta.cpu().numpy()))
