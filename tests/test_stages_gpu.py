"""Stage kernels through the C ABI against the reference's gold fixtures and
the CPU oracle (GPU).  Tolerances follow the reference's own tests:
Sobol/scramble bit-exact, bridge 2e-7 mean relative (Bridge_Test.cu:35),
correlate 1e-6 (correlate_drift_test.cu:34), PC rates 2e-6 mean relative
(LMM_evolver_test.cu:45), LS 1e-4 (LSmulti_test.cu:2304)."""
import ctypes
import math

import numpy as np
import pytest

from conftest import BRIDGE_SHAPES, rel_err

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def _torch():
    import torch

    return torch


# Device copies made inline for a call are kept alive until the test ends:
# a raw pointer to a freed temporary would alias the next allocation.
_KEEP = []


@pytest.fixture(autouse=True)
def _release_device_copies():
    yield
    _KEEP.clear()


def dev(a):
    torch = _torch()
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32)).cuda()
    else:
        t = torch.from_numpy(a).cuda()
    _KEEP.append(t)
    return t


def host(t, dtype=None):
    _torch().cuda.synchronize()
    a = t.cpu().numpy()
    if dtype == np.uint32:
        a = a.view(np.uint32)
    return a


def d(t):
    return VP(t.data_ptr()) if t is not None else None


def h(a):
    return VP(a.ctypes.data) if a is not None else None


def empty(shape, dtype="f4"):
    torch = _torch()
    tmap = {"f4": torch.float32, "u4": torch.int32, "i4": torch.int32, "f8": torch.float64}
    return torch.zeros(shape, dtype=tmap[dtype], device="cuda")


def call(name, *args):
    from useful_code_b200._lib import call as c

    return c(name, *args)


# ---------------------------------------------------------------- Sobol ----
@pytest.mark.parametrize("P,dims,off,key", [(1024, 64, 0, "sobol_p1024_d64_off0"),
                                            (512, 64, 777, "sobol_p512_d64_off777")])
def test_sobol_matches_gold(cuda, gold, ref_dirs, P, dims, off, key):
    dd = dev(ref_dirs[:dims])
    out = empty((dims, P), "u4")
    call("lmm_sobol_ints", P, dims, off, d(dd), d(out), None)
    assert np.array_equal(host(out, np.uint32), gold[key])


@pytest.mark.parametrize("P,dims,off", [(1000, 37, 3), (1, 5, 0), ((1 << 20) + 3, 6, 12345)])
def test_sobol_matches_oracle(cuda, orc, ref_dirs, P, dims, off):
    dd = dev(ref_dirs[:dims])
    out = empty((dims, P), "u4")
    call("lmm_sobol_ints", P, dims, off, d(dd), d(out), None)
    ref = np.zeros((dims, P), np.uint32)
    orc("orc_sobol_ints", P, dims, np.uint32(off), ref_dirs[:dims].copy(), ref)
    assert np.array_equal(host(out, np.uint32), ref)


def test_sobol_offset_additivity(cuda, ref_dirs):
    dd = dev(ref_dirs[:200])
    full = empty((200, 1 << 16), "u4")
    call("lmm_sobol_ints", 1 << 16, 200, 0, d(dd), d(full), None)
    a = empty((200, 1 << 15), "u4")
    b = empty((200, 1 << 15), "u4")
    call("lmm_sobol_ints", 1 << 15, 200, 0, d(dd), d(a), None)
    call("lmm_sobol_ints", 1 << 15, 200, 1 << 15, d(dd), d(b), None)
    assert np.array_equal(np.concatenate([host(a, np.uint32), host(b, np.uint32)], 1),
                          host(full, np.uint32))


def test_scramble_matches_gold(cuda, gold, orc):
    data = dev(gold["scramble_in"])
    scr = dev(gold["scramble_scr"])
    D, P = gold["scramble_in"].shape
    call("lmm_scramble", d(data), d(scr), D, P, None)
    assert np.array_equal(host(data, np.uint32), gold["scramble_out"])
    rng = np.random.default_rng(3)
    x = rng.integers(0, 2**32, (7, 1001), dtype=np.uint64).astype(np.uint32)
    s = rng.integers(0, 2**32, 7, dtype=np.uint64).astype(np.uint32)
    t = dev(x)
    call("lmm_scramble", d(t), d(dev(s)), 5, 1001, None)
    ref = x.copy()
    orc("orc_scramble", ref, s, 5, 1001)
    assert np.array_equal(host(t, np.uint32), ref)


def test_icdf(cuda, gold, orc):
    ints = gold["icdf_in"]
    out = empty(ints.size)
    call("lmm_icdf_shaw_brickman", d(dev(ints)), d(out), ints.size, None)
    got = host(out)
    ref = gold["icdf_sb"]
    fin = np.isfinite(ref)
    assert np.max(np.abs(got[fin] - ref[fin]) / np.maximum(1, np.abs(ref[fin]))) < 2e-6
    assert np.all(np.isfinite(got))
    rng = np.random.default_rng(11)
    x = rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.uint32)
    out2 = empty(x.size)
    call("lmm_icdf_shaw_brickman", d(dev(x)), d(out2), x.size, None)
    o = np.zeros(x.size, np.float32)
    orc("orc_icdf_f", x, o, ctypes.c_long(x.size))
    g = host(out2)
    assert np.max(np.abs(g - o) / np.maximum(1, np.abs(o))) < 2e-6
    # odd length takes the scalar path
    out3 = empty(1001)
    call("lmm_icdf_shaw_brickman", d(dev(x[:1001])), d(out3), 1001, None)
    assert np.array_equal(host(out3), g[:1001])


def test_icdf_tails(cuda, orc):
    rng = np.random.default_rng(12)
    x = np.concatenate([rng.integers(0, 2**32, 1 << 20, dtype=np.uint64),
                        np.arange(0, 4096), 2**32 - 1 - np.arange(0, 4096)]).astype(np.uint32)
    out = empty(x.size)
    call("lmm_icdf_shaw_brickman_tails", d(dev(x)), d(out), x.size, None)
    o = np.zeros(x.size, np.float32)
    orc("orc_icdf_tails_f", x, o, ctypes.c_long(x.size))
    g = host(out)
    assert np.all(np.isfinite(g))
    assert np.max(np.abs(g - o) / np.maximum(1, np.abs(o))) < 2e-6
    out3 = empty(1001)
    call("lmm_icdf_shaw_brickman_tails", d(dev(x[:1001])), d(out3), 1001, None)
    assert np.array_equal(host(out3), g[:1001])


@pytest.mark.parametrize("S,F,P", [(20, 3, 2048), (40, 5, 1000), (80, 10, 1024), (120, 15, 512)])
def test_bridge(cuda, orc, S, F, P):
    rng = np.random.default_rng(S)
    z = rng.standard_normal((F * S, P)).astype(np.float32)
    out = empty((S, F, P))
    call("lmm_bridge_transform", d(dev(z)), d(out), P, S, F, None, None)
    ref = np.zeros((S, F, P), np.float32)
    orc("orc_bridge_f", z, ref, P, S, F, None)
    got = host(out)
    assert np.mean(np.abs(got - ref)) / np.mean(np.abs(ref)) < 2e-7
    assert np.max(np.abs(got - ref)) < 5e-5
    # unit-variance increments
    assert abs(float(np.var(got)) - 1.0) < 0.1


@pytest.mark.parametrize("S,F", BRIDGE_SHAPES)
def test_bridge_matches_reference_newbridge(cuda, gold_bridge, S, F):
    """lmm_bridge_transform against the reference's own newBridge
    (brownian_bridge::transformCPU) on identical normals, at the reference
    test's tolerance (Bridge_Test.cu:35: 2e-7 mean relative)."""
    z = gold_bridge[f"bridge_S{S}_F{F}_in"]
    ref = gold_bridge[f"bridge_S{S}_F{F}_out"]
    P = z.shape[1]
    out = empty((S, F, P))
    call("lmm_bridge_transform", d(dev(z)), d(out), P, S, F, None, None)
    got = host(out)
    assert np.mean(np.abs(got - ref)) / np.mean(np.abs(ref)) < 2e-7
    assert np.max(np.abs(got - ref)) < 2e-5


def test_bridge_matches_reference_permuted_allocation(cuda, gold_bridge):
    z = gold_bridge["bridge_perm_in"]
    alloc = np.ascontiguousarray(gold_bridge["bridge_perm_alloc"], np.int32)
    F, S = alloc.shape
    P = z.shape[1]
    ref = gold_bridge["bridge_perm_out"]
    out = empty((S, F, P))
    call("lmm_bridge_transform", d(dev(z)), d(out), P, S, F, h(alloc), None)
    got = host(out)
    assert np.mean(np.abs(got - ref)) / np.mean(np.abs(ref)) < 2e-7
    assert np.max(np.abs(got - ref)) < 2e-5


def test_correlate_drift(cuda, gold, orc):
    z = gold["lmm_z_spf"]
    S, P, F = z.shape
    n = gold["lmm_tau"].size
    alive = np.zeros(S, np.int32)  # gold writes every rate
    out = empty((S, n, P))
    call("lmm_correlate_drift", d(dev(z)), d(out), d(dev(gold["lmm_A"])), h(alive),
         d(dev(gold["lmm_fixed"])), n * F, F, n, P, S, 0, None)
    assert np.max(np.abs(host(out) - gold["lmm_corr"])) < 1e-6
    zt = np.ascontiguousarray(z.transpose(0, 2, 1))  # [S][F][P]
    out2 = empty((S, n, P))
    call("lmm_correlate_drift", d(dev(zt)), d(out2), d(dev(gold["lmm_A"])), h(alive),
         d(dev(gold["lmm_fixed"])), n * F, F, n, P, S, 1, None)
    assert np.max(np.abs(host(out2) - gold["lmm_corr"])) < 1e-6


def test_pc_staged(cuda, gold):
    corr = gold["lmm_corr"]
    S, n, P = corr.shape
    F = gold["lmm_A"].shape[2]
    r = empty((S, n, P))
    lr = empty((S, n, P))
    call("lmm_evolve_pc_staged", h(gold["lmm_f0"]), h(gold["lmm_tau"]), h(gold["lmm_disp"]),
         d(dev(corr)), d(dev(gold["lmm_A"])), None, P, F, S, n, 10.0, d(r), d(lr), None)
    err = rel_err(host(r), gold["lmm_rates"])
    assert err.mean() < 2e-6 and err.max() < 2e-5
    assert np.max(np.abs(host(lr) - gold["lmm_logrates"])) < 2e-5
    # with the alive indices of the pipeline (rate s resets at step s) the
    # live rates are the same: the expired rates' pseudo-root rows are zero
    alive = np.arange(S, dtype=np.int32)
    r2 = empty((S, n, P))
    lr2 = empty((S, n, P))
    call("lmm_evolve_pc_staged", h(gold["lmm_f0"]), h(gold["lmm_tau"]), h(gold["lmm_disp"]),
         d(dev(corr)), d(dev(gold["lmm_A"])), h(alive), P, F, S, n, 10.0, d(r2), d(lr2), None)
    mask = np.zeros((S, n), bool)
    for st in range(S):
        mask[st, st:] = True
    np.testing.assert_allclose(host(r2)[mask], host(r)[mask], rtol=1e-6, atol=1e-9)


def test_curve_stages(cuda, gold):
    rates = gold["lmm_rates"]
    S, n, P = rates.shape
    alive = np.arange(S, dtype=np.int32)
    tau = gold["lmm_tau"]
    disc = empty((S, n + 1, P))
    call("lmm_discount_ratios", d(dev(rates)), h(tau), h(alive), P, S, n, d(disc), None)
    gd = gold["lmm_disc"]
    m = np.zeros(gd.shape, bool)
    for s in range(S):
        m[s, s:] = True
    assert np.max(rel_err(host(disc), gd)[m]) < 2e-6
    ann = empty((S, n, P))
    call("lmm_coterminal_annuities", d(dev(gd)), h(tau), h(alive), P, S, n, d(ann), None)
    sr = empty((S, n, P))
    call("lmm_coterminal_swap_rates", d(dev(gd)), d(dev(gold["lmm_ann"])), h(alive), P, S, n,
         d(sr), None)
    m2 = m[:, :n]
    assert np.max(rel_err(host(ann), gold["lmm_ann"])[m2]) < 2e-6
    assert np.max(rel_err(host(sr), gold["lmm_sr"])[m2]) < 2e-6
    num = empty((n, P))
    call("lmm_spot_numeraires", d(dev(gd)), P, P, 0, n, d(num), None)
    assert np.max(rel_err(host(num), gold["lmm_num"])) < 2e-6
    # single swap rate vs the coterminal one
    one = empty((S, P))
    call("lmm_swap_rate", d(dev(gd)), h(tau), 3, n, P, 3, 3, S, n, d(one), None)
    assert np.max(rel_err(host(one)[3], gold["lmm_sr"][3, 3])) < 2e-6


def test_extractions(cuda, gold):
    rates = gold["lmm_rates"]
    S, n, P = rates.shape
    idx = np.minimum(np.arange(S) + 1, n - 1).astype(np.int32)
    out = empty((S, P))
    call("lmm_forward_extraction", d(dev(rates)), h(idx), P, S, n, d(out), None)
    assert np.array_equal(host(out), rates[np.arange(S), idx])
    steps = np.array([1, 4, 9], np.int32)
    fw = np.array([2, 5, 11], np.int32)
    out2 = empty((3, P))
    call("lmm_forward_extraction_steps", d(dev(rates)), h(fw), h(steps), 3, P, n, d(out2), None)
    assert np.array_equal(host(out2), rates[steps, fw])
    num = gold["lmm_num"]
    ex = gold["cf_ex_idx"]
    some = empty((ex.size, 2 * P))
    call("lmm_numeraire_extraction", d(dev(num)), d(some), P, 2 * P, P, n, ex.size, h(ex), None)
    assert np.array_equal(host(some)[:, P:], num[ex])


def test_cashflows_discounting_aggregation(cuda, gold):
    disc = gold["lmm_disc"]
    S, _, P = disc.shape
    f1 = empty((S, P))
    f2 = empty((S, P))
    call("lmm_cashflows_swap", d(f1), d(f2), h(gold["cf_aux"]), P, S, d(dev(gold["cf_rate1"])), None)
    assert np.max(np.abs(host(f1) - gold["cf_flows1"])) < 1e-9
    assert np.max(np.abs(host(f2) - gold["cf_flows2"])) < 1e-9
    out = empty((S, P))
    summed = empty(P)
    call("lmm_cashflow_discounting", h(gold["cf_first_mid"]), h(gold["cf_second_mid"]),
         h(gold["cf_theta_mid"]), d(dev(disc)), d(dev(gold["cf_flows2"])), d(dev(gold["lmm_num"])),
         P, S, d(out), d(summed), None)
    assert np.max(np.abs(host(out) - gold["cf_discounted"])) < 2e-7
    assert np.max(np.abs(host(summed) - gold["cf_summed"])) < 2e-6
    gen = np.arange(S, dtype=np.int32)
    part = empty((S, P))
    call("lmm_cashflow_discounting_partial", S, h(gen), h(gold["cf_first"]), h(gold["cf_second"]),
         h(gold["cf_theta"]), h(gold["cf_target"]), d(dev(disc)), d(dev(gold["cf_flows2"])),
         d(dev(gold["lmm_num"])), P, S, d(part), None)
    assert np.max(np.abs(host(part) - gold["cf_partial"])) < 2e-7
    ex = gold["cf_ex_idx"]
    agg = empty((ex.size, P))
    call("lmm_aggregate_flows", d(agg), P, ex.size, d(dev(gold["cf_partial"])), P, 0, S,
         h(gold["cf_step_to_ex"]), int(gold["cf_first_positive"]), None)
    assert np.max(np.abs(host(agg) - gold["cf_aggregated"])) < 1e-6
    cap = empty((S, P))
    zero = empty((S, P))
    aux = np.concatenate([[0.05], np.full(S, 0.5)]).astype(np.float32)
    call("lmm_cashflows_caplet", d(cap), d(zero), h(aux), P, S, d(dev(gold["cf_rate1"])), None)
    ref = 0.5 * np.maximum(gold["cf_rate1"] - np.float32(0.05), 0)
    assert np.max(np.abs(host(cap) - ref)) < 1e-9 and not host(zero).any()


@pytest.mark.parametrize("tag", ["a", "b"])
def test_cashflows_tarn(cuda, gold, tag):
    """TARN flows (cashFlowGeneratorCallerTARN) against the reference's gold
    on the fixture's reset rates, and against the oracle's restatement."""
    rate1 = gold["cf_rate1"]
    S, P = rate1.shape
    f1 = empty((S, P))
    f2 = empty((S, P))
    call("lmm_cashflows_tarn", d(f1), d(f2), h(gold[f"tarn_{tag}_aux"]), P, S, d(dev(rate1)),
         d(dev(rate1)), None)
    assert np.max(np.abs(host(f1) - gold[f"tarn_{tag}_flows1"])) < 1e-7
    assert np.max(np.abs(host(f2) - gold[f"tarn_{tag}_flows2"])) < 1e-7


def test_exercise_values_and_basis(cuda, gold):
    r1, r2, r3 = gold["ex_r1"], gold["ex_r2"], gold["ex_r3"]
    E, P = r2.shape
    out = empty((E, P))
    call("lmm_exercise_values_payer_swaption", 0.05, d(dev(r2)), d(dev(r3)), P, P, 0, E, d(out), None)
    assert np.array_equal(host(out), gold["ex_values"])
    for use_log, key in [(0, "bv_raw"), (1, "bv_log")]:
        bv = empty((E, 3, P))
        call("lmm_basis_variables", use_log, h(gold["bv_shifts"]), d(dev(r1)), d(dev(r2)), d(dev(r3)),
             P, P, 0, E, d(bv), None)
        assert np.max(np.abs(host(bv) - gold[key])) < 1e-6


def test_reductions(cuda):
    from useful_code_b200._lib import LIB

    rng = np.random.default_rng(9)
    x = rng.standard_normal(3_000_017).astype(np.float32)
    part = empty(int(LIB.lmm_reduce_workspace_doubles()), "f8")
    out = empty(1, "f8")
    call("lmm_reduce_sum", d(dev(x)), x.size, d(part), d(out), None)
    assert abs(host(out)[0] - math.fsum(x.astype(np.float64))) < 1e-9
    y = (rng.random(x.size).astype(np.float32) + 0.5)
    call("lmm_reduce_mean_ratio", d(dev(x)), d(dev(y)), x.size, d(part), d(out), None)
    ref = math.fsum((x.astype(np.float64) / y.astype(np.float64))) / x.size
    assert abs(host(out)[0] - ref) < 1e-12
    # deterministic: same result twice
    a = host(out)[0]
    call("lmm_reduce_mean_ratio", d(dev(x)), d(dev(y)), x.size, d(part), d(out), None)
    assert host(out)[0] == a


@pytest.mark.parametrize("ragged", [False, True])
@pytest.mark.parametrize("norm", [1, 0])
def test_ls_regress(cuda, gold, orc, norm, ragged):
    """Device regression against the oracle on the gold LS inputs: all 512
    paths (16-byte staged copies of the path inputs) and the first 509
    (rows not 16-byte aligned: each thread copies its own path's inputs)."""
    from useful_code_b200 import market as mk
    from useful_code_b200._lib import LIB

    keep = 509 if ragged else None
    vars64 = np.ascontiguousarray(gold["ls_vars"][:, :, :keep])
    E, _, P = vars64.shape
    vars32 = vars64.astype(np.float32)
    cf = np.ascontiguousarray(gold["ls_cf"][:, :keep]).astype(np.float32)
    ex = np.ascontiguousarray(gold["ls_ex"][:, :keep]).astype(np.float32)
    num = np.ascontiguousarray(gold["ls_num"][:, :keep]).astype(np.float32)
    nv = gold["ls_nvars"]
    mono, nb = mk.basis_tables("cross", nv)
    ws = empty(int(LIB.lmm_ls_workspace_bytes(P, E)), "i4")
    beta = empty((E, 16), "f8")
    means = empty((E, 3))
    sds = empty((E, 3))
    gram = empty((E, 16, 17), "f8")
    status = empty(1, "i4")
    price = empty(1, "f8")
    call("lmm_ls_regress", E, P, d(dev(vars32)), h(nv), h(mono), h(nb), d(dev(cf)), d(dev(ex)),
         d(dev(num)), norm, d(ws), ws.numel() * 4, d(beta), d(means) if norm else None,
         d(sds) if norm else None, d(gram), d(status), d(price), None)
    b_ref = np.zeros((E, 16))
    m_ref = np.zeros((E, 3))
    s_ref = np.zeros((E, 3))
    g_ref = np.zeros((E, 16, 17))
    p_ref = orc("orc_ls_regress_f", E, P, vars32, nv, mono, nb, cf, ex, num, norm, b_ref, m_ref,
                s_ref, g_ref, restype=ctypes.c_double)
    K = nb[0]
    g = host(gram)[:, :K, : K + 1]
    r = g_ref[:, :K, : K + 1]
    scale = np.max(np.abs(r), axis=2, keepdims=True)
    # basis block: FP32 basis values, FP64 sums
    assert np.max(np.abs(g[:, :, :K] - r[:, :, :K]) / scale) < 5e-6
    # target column: the realised continuation values depend on the later
    # dates' decisions, and a path whose exercise value lies within rounding
    # of its estimate may decide differently in FP32 and FP64, moving the
    # sum by (exercise - realised) / paths
    assert np.max(np.abs(g[:, :, K] - r[:, :, K]) / scale[:, :, 0]) < 1e-3
    assert abs(host(price)[0] - p_ref) < 1e-4
    # fitted continuation values (the regression's output) rather than
    # coefficients, which an ill-conditioned basis leaves loosely determined.
    # On raw (unstandardised) rates the cross basis is too ill-conditioned
    # for FP32 basis values to pin the fit; there the price is the check.
    G = r[:, :, :K]
    for e in range(E - 1 if norm else 0):
        db = host(beta)[e, :K] - b_ref[e, :K]
        fit_diff = np.sqrt(max(db @ G[e] @ db, 0.0))
        fit = np.sqrt(max(b_ref[e, :K] @ G[e] @ b_ref[e, :K], 1e-30))
        assert fit_diff < 1e-2 * fit, (e, fit_diff, fit)
    if norm and not ragged:
        assert abs(host(price)[0] - float(gold["ls_cross1_norm1_price"])) < 1e-4


def test_evolve_pc_all_matches_gold(cuda, gold):
    """lmm_evolve_pc_all (the one-launch evolution with full tensors, the
    reference's LMM_evolver_pc_all_gpu) on the gold fixture's uncorrelated
    normals ([step][path][factor], layout 0) against the reference's gold
    correlate + PC chain: rates within 2e-6 mean relative
    (LMM_evolver_test.cu:45); discount ratios as the gold's."""
    z = gold["lmm_z_spf"]
    S, P, F = z.shape
    n = gold["lmm_tau"].size
    alive = np.arange(S, dtype=np.int32)
    rates = empty((S, n, P))
    lrates = empty((S, n, P))
    disc = empty((S, n + 1, P))
    call("lmm_evolve_pc_all", h(gold["lmm_f0"]), h(gold["lmm_tau"]), h(gold["lmm_disp"]),
         d(dev(z)), 0, d(dev(gold["lmm_A"])), d(dev(gold["lmm_fixed"])), h(alive), P, F, S, n,
         10.0, d(rates), d(lrates), d(disc), None)
    got, gl, gd = host(rates), host(lrates), host(disc)
    mask = np.zeros((S, n), bool)
    for s in range(S):
        mask[s, s:] = True
    err = rel_err(got, gold["lmm_rates"])[mask]
    assert err.mean() < 2e-6 and err.max() < 2e-5, (err.mean(), err.max())
    assert np.max(np.abs(gl - gold["lmm_logrates"])[mask]) < 1e-5
    dmask = np.zeros((S, n + 1), bool)
    for s in range(S):
        dmask[s, s:] = True
    assert np.max(rel_err(gd, gold["lmm_disc"])[dmask]) < 2e-5
    # layout 1 ([step][factor][path]) gives the same tensors
    rates1 = empty((S, n, P))
    call("lmm_evolve_pc_all", h(gold["lmm_f0"]), h(gold["lmm_tau"]), h(gold["lmm_disp"]),
         d(dev(np.ascontiguousarray(z.transpose(0, 2, 1)))), 1, d(dev(gold["lmm_A"])),
         d(dev(gold["lmm_fixed"])), h(alive), P, F, S, n, 10.0, d(rates1), d(lrates), None,
         None)
    assert np.array_equal(host(rates1)[mask], got[mask])
