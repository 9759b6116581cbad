"""Sharded regression entry points on the GPU (lmm_ls_moment_sums,
lmm_ls_moments_from_sums, lmm_ls_date_sums, lmm_ls_date_solve,
lmm_ls_final_sum).

With one shard they must reproduce lmm_ls_regress; with the paths split
into two shards whose sums are added between the steps (the all-reduce of
a two-GPU run, done here in one process, one shard after the other, no
kernel waiting on another), the rule must agree with the regression on all
paths up to the FP32 order of summation."""
import numpy as np
import pytest
import torch

from useful_code_b200 import market as mk

pytestmark = pytest.mark.gpu


def mini():
    from dataclasses import replace

    cfg = mk.make_config("c2")
    return replace(cfg, n=12, F=3, f0=np.linspace(0.04, 0.06, 12).astype(np.float32),
                   paths=8192, reg_paths=8192)


@pytest.fixture(scope="module")
def setup(cuda):
    from useful_code_b200.pricer import Pipeline

    m = mk.build_market(mini())
    pipe = Pipeline(m)
    P = 8192
    ls = pipe.first_pass(P, 0, "fused")
    return m, pipe, ls, P


def test_one_shard_equals_regress(setup):
    from useful_code_b200.sharded import regress_sharded

    m, pipe, ls, P = setup
    a = pipe.regress(ls)
    b = regress_sharded(pipe, ls, P)
    torch.cuda.synchronize()
    assert int(b.status.item()) == int(a.status.item())
    np.testing.assert_allclose(b.beta.cpu().numpy(), a.beta.cpu().numpy(), rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal(b.means.cpu().numpy(), a.means.cpu().numpy())
    assert abs(float(b.price) - float(a.price.item())) < 1e-12


def test_two_shards_in_lockstep(setup):
    from useful_code_b200.pricer import LSInputs
    from useful_code_b200.sharded import GpuBackend

    m, pipe, ls, P = setup
    h = P // 2
    parts = [LSInputs(ls.vars[:, :, s].contiguous(), ls.ex[:, s].contiguous(),
                      ls.cf[:, s].contiguous(), ls.num[:, s].contiguous())
             for s in (slice(0, h), slice(h, P))]
    bes = [GpuBackend(pipe, part) for part in parts]
    for be in bes:
        be.begin()
    msum = bes[0].moment_sums() + bes[1].moment_sums()
    for be in bes:
        be.moments_from_sums(msum, P)
    for e in range(pipe.E - 1, -1, -1):
        s = bes[0].date_sums(e) + bes[1].date_sums(e)
        for be in bes:
            be.date_solve(e, s, P)
    price = (bes[0].final_sum() + bes[1].final_sum()) / P
    torch.cuda.synchronize()
    ref = pipe.regress(ls, keep_gram=True)
    # both shards solved the same sums: identical rules
    assert torch.equal(bes[0].beta, bes[1].beta)
    # against the one-GPU regression: same sums in another FP32 grouping
    G = ref.gram.cpu().numpy()
    K = int(pipe._nbasis[0])
    for e in range(pipe.E - 1):
        db = bes[0].beta.cpu().numpy()[e, :K] - ref.beta.cpu().numpy()[e, :K]
        g = G[e, :K, :K]
        fit = np.sqrt(ref.beta.cpu().numpy()[e, :K] @ g @ ref.beta.cpu().numpy()[e, :K])
        assert np.sqrt(max(db @ g @ db, 0.0)) < 1e-3 * fit + 1e-12, e
    assert abs(float(price[0]) - float(ref.price.item())) < 1e-5
