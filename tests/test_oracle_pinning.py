"""Pin the CPU oracle (oracle/lmm_oracle.cpp) against the reference.

Every stage of the restatement is compared with golden fixtures produced
by the reference's own gold routines (tests/golden/make_golden.py), at the
reference tests' tolerances: Sobol and scramble bit-exact
(Sobol_int_test.cu:196, scramble_test.cu:138-142), correlate+drift 1e-6
(correlate_drift_test.cu:34), PC rates 2e-6 (LMM_evolver_test.cu:45), LS
estimate 1e-4 (LSmulti_test.cu:2304).  CPU only.
"""
import numpy as np
import pytest

from conftest import BRIDGE_SHAPES, rel_err


def test_sobol_bit_exact_and_offsets(orc, gold, ref_dirs):
    out = np.zeros((64, 1024), np.uint32)
    orc("orc_sobol_ints", 1024, 64, np.uint32(0), ref_dirs, out)
    assert np.array_equal(out, gold["sobol_p1024_d64_off0"])
    off = np.zeros((64, 512), np.uint32)
    orc("orc_sobol_ints", 512, 64, np.uint32(777), ref_dirs, off)
    assert np.array_equal(off, gold["sobol_p512_d64_off777"])
    # offset additivity: two half batches reproduce the full batch
    a = np.zeros((64, 512), np.uint32)
    b = np.zeros((64, 512), np.uint32)
    orc("orc_sobol_ints", 512, 64, np.uint32(0), ref_dirs, a)
    orc("orc_sobol_ints", 512, 64, np.uint32(512), ref_dirs, b)
    assert np.array_equal(np.concatenate([a, b], 1), gold["sobol_p1024_d64_off0"])


def test_scramble_exact(orc, gold):
    data = gold["scramble_in"].copy()
    orc("orc_scramble", data, gold["scramble_scr"], data.shape[0], data.shape[1])
    assert np.array_equal(data, gold["scramble_out"])


def test_icdf_shaw_brickman(orc, gold):
    ints = gold["icdf_in"]
    ref = gold["icdf_sb"]
    out = np.zeros(ints.size, np.float32)
    orc("orc_icdf_f", ints, out, ctypes_long(ints.size))
    finite = np.isfinite(ref)
    assert np.max(np.abs(out[finite] - ref[finite])) <= 2e-6 * np.maximum(1, np.abs(ref[finite])).max()
    # points where the reference takes log(0) map to the finite tail here
    assert np.all(np.isfinite(out))
    assert np.all(np.abs(out[~finite]) > 5.0)


def test_icdf_tails_is_accurate(orc):
    """The pipelines' form (tail probability from the integer) stays within
    7e-7 of the exact quantile everywhere; the reference's single-precision
    form loses up to 1e-3 in the outer one percent and more in the far
    tails (the reason the pipelines do not use it)."""
    from scipy.special import ndtri

    rng = np.random.default_rng(3)
    ints = np.concatenate([rng.integers(0, 2**32, 200000, dtype=np.uint64),
                           np.arange(1, 4096), 2**32 - 1 - np.arange(0, 4096),
                           2**31 + np.arange(-4096, 4096)]).astype(np.uint32)
    ref_form = np.zeros(ints.size, np.float32)
    tails = np.zeros(ints.size, np.float32)
    orc("orc_icdf_f", ints, ref_form, ctypes_long(ints.size))
    orc("orc_icdf_tails_f", ints, tails, ctypes_long(ints.size))
    exact = ndtri(ints.astype(np.float64) * 2.0**-32)
    scale = np.maximum(1, np.abs(exact))
    assert np.max(np.abs(tails - exact) / scale) < 7e-7
    assert np.max(np.abs(ref_form - exact) / scale) > 1e-2
    # identical forms where 1 - |2u - 1| is exact in single precision
    mid = np.abs(ints.astype(np.int64) - 2**31) < 2**29
    assert np.max(np.abs(tails[mid] - ref_form[mid]) / scale[mid]) < 5e-7
    # i = 0 is clamped like the reference's path
    z0 = np.zeros(1, np.float32)
    orc("orc_icdf_tails_f", np.zeros(1, np.uint32), z0, ctypes_long(1))
    assert np.isfinite(z0[0]) and z0[0] < -6.0


def ctypes_long(n):
    import ctypes

    return ctypes.c_long(n)


def test_icdf_double_is_accurate(orc):
    from scipy.special import ndtri

    rng = np.random.default_rng(5)
    ints = rng.integers(1 << 8, (1 << 32) - (1 << 8), 20000, dtype=np.uint64).astype(np.uint32)
    out = np.zeros(ints.size)
    orc("orc_icdf_d", ints, out, ctypes_long(ints.size))
    u = ints.astype(np.float64) * 2.0 ** -32
    assert np.max(np.abs(out - ndtri(u))) < 1e-12


@pytest.mark.parametrize("F,S", [(3, 20), (5, 40), (10, 80), (15, 120)])
def test_bridge_allocation(orc, gold, F, S):
    a = np.zeros((F, S), np.int32)
    orc("orc_bridge_allocate_diagonal", F, S, a)
    assert np.array_equal(a, gold[f"alloc_diag_F{F}_S{S}"])


@pytest.mark.parametrize("S,F", BRIDGE_SHAPES)
def test_bridge_matches_reference_newbridge(orc, gold_bridge, S, F):
    """The restated bridge equals the reference's own newBridge host code
    (brownian_bridge::transformCPU, brownian_bridge.cu:401-455, tables
    :639-697, run by tests/golden/make_golden.py) bit for bit in FP32, with
    the diagonal allocation; the FP64 form agrees to FP32 rounding."""
    z = gold_bridge[f"bridge_S{S}_F{F}_in"]
    ref = gold_bridge[f"bridge_S{S}_F{F}_out"]
    P = z.shape[1]
    out = np.zeros((S, F, P), np.float32)
    orc("orc_bridge_f", z, out, P, S, F, None)
    assert np.array_equal(out, ref)
    out64 = np.zeros((S, F, P))
    orc("orc_bridge_d", np.ascontiguousarray(z, np.float64), out64, P, S, F, None)
    assert np.max(np.abs(out64 - ref)) < 1e-5


def test_bridge_matches_reference_permuted_allocation(orc, gold_bridge):
    z = gold_bridge["bridge_perm_in"]
    alloc = np.ascontiguousarray(gold_bridge["bridge_perm_alloc"], np.int32)
    F, S = alloc.shape
    P = z.shape[1]
    out = np.zeros((S, F, P), np.float32)
    orc("orc_bridge_f", z, out, P, S, F, alloc)
    assert np.array_equal(out, gold_bridge["bridge_perm_out"])


@pytest.mark.parametrize("k", [1, 3, 5, 7])
def test_power_of_two_bridge_is_the_newbridge(orc, gold_bridge, k):
    """The reference's power-of-two bridge (BrownianBridge<float>,
    gold/Bridge_gold.h:168-327) is the newBridge construction on 2^k unit
    steps with the identity allocation (same points, order, variates and
    weights): the restated newBridge agrees with it to FP32 rounding."""
    z = gold_bridge[f"pow2_k{k}_in"]
    n, P = z.shape
    out = np.zeros((n, 1, P), np.float32)
    orc("orc_bridge_f", z, out, P, n, 1, np.arange(n, dtype=np.int32))
    ref = gold_bridge[f"pow2_k{k}_out"]
    assert np.max(np.abs(out[:, 0] - ref)) < 2e-5
    assert np.mean(np.abs(out[:, 0] - ref)) / np.mean(np.abs(ref)) < 2e-7


def test_correlate_drift(orc, gold):
    z = gold["lmm_z_spf"]
    S, P, F = z.shape
    n = gold["lmm_tau"].size
    out = np.zeros((S, n, P), np.float32)
    orc("orc_correlate_drift_f", z, out, gold["lmm_A"], n * F, gold["lmm_fixed"], F, n, P, S, 0)
    assert np.max(np.abs(out - gold["lmm_corr"])) < 1e-6


def test_pc_evolution(orc, gold):
    corr = gold["lmm_corr"]
    S, n, P = corr.shape
    F = gold["lmm_A"].shape[2]
    rates = np.zeros_like(corr)
    lrates = np.zeros_like(corr)
    orc("orc_pc_f", gold["lmm_f0"], gold["lmm_tau"], corr, gold["lmm_A"], gold["lmm_disp"],
        P, F, S, n, np.float32(10.0), rates, lrates)
    err = rel_err(rates, gold["lmm_rates"])
    assert err.mean() < 2e-6 and err.max() < 2e-5
    assert np.max(np.abs(lrates - gold["lmm_logrates"])) < 1e-5


def test_curve_stages(orc, gold):
    rates = gold["lmm_rates"]
    S, n, P = rates.shape
    alive = np.arange(n, dtype=np.int32)
    tau = gold["lmm_tau"]
    disc = np.zeros((S, n + 1, P), np.float32)
    orc("orc_discount_ratios_f", rates, tau, alive, P, S, n, disc)
    mask = np.zeros_like(disc, bool)
    for s in range(S):
        mask[s, s:] = True
    assert np.max(np.abs(disc - gold["lmm_disc"])[mask]) < 1e-6
    ann = np.zeros((S, n, P), np.float32)
    orc("orc_annuities_f", gold["lmm_disc"], tau, alive, P, S, n, ann)
    sr = np.zeros((S, n, P), np.float32)
    orc("orc_swap_rates_f", gold["lmm_disc"], gold["lmm_ann"], alive, P, S, n, sr)
    m2 = mask[:, :n]
    assert np.max(rel_err(ann, gold["lmm_ann"])[m2]) < 1e-6
    assert np.max(rel_err(sr, gold["lmm_sr"])[m2]) < 1e-6
    num = np.zeros((n, P), np.float32)
    orc("orc_numeraires_f", gold["lmm_disc"], P, n, num)
    assert np.max(rel_err(num, gold["lmm_num"])) < 1e-6


def test_discounting(orc, gold):
    disc = gold["lmm_disc"]
    S, _, P = disc.shape
    out = np.zeros((S, P), np.float32)
    summed = np.zeros(P, np.float32)
    orc("orc_discounting_f", gold["cf_first_mid"], gold["cf_second_mid"], gold["cf_theta_mid"],
        disc, gold["cf_flows2"], gold["lmm_num"], P, S, out, summed)
    assert np.max(np.abs(out - gold["cf_discounted"])) < 1e-6
    assert np.max(np.abs(summed - gold["cf_summed"])) < 1e-5


def test_payer_swaption_values(orc, gold):
    r2, r3 = gold["ex_r2"], gold["ex_r3"]
    out = np.zeros_like(r2)
    orc("orc_payer_swaption_values_f", np.float32(0.05), r2, r3, r2.shape[1], r2.shape[0], out)
    assert np.array_equal(out, gold["ex_values"])


@pytest.mark.parametrize("cross,norm", [(1, 1), (1, 0), (0, 1)])
def test_ls_regression_matches_gold(orc, gold, cross, norm):
    from useful_code_b200 import market as mk

    vars_ = gold["ls_vars"]
    E, _, P = vars_.shape
    nvars = gold["ls_nvars"]
    mono, nb = mk.basis_tables("cross" if cross else "quadratic", nvars)
    beta = np.zeros((E, 16))
    means = np.zeros((E, 3))
    sds = np.zeros((E, 3))
    import ctypes

    price = orc("orc_ls_regress_d", E, P, vars_, nvars, mono, nb, gold["ls_cf"], gold["ls_ex"],
                gold["ls_num"], norm, beta, means, sds, None, restype=ctypes.c_double)
    key = f"ls_cross{cross}_norm{norm}"
    ncoef = nb[0]
    if not norm:
        # Raw variables: the Gram is ill-conditioned and the reference's SVD
        # drops singular values below 1e-8 of the largest
        # (gold/MultiLS_regression.cpp:173-177), which moves its fit; hold the
        # estimate to the reference's LS tolerance (LS_test.cu:74).
        assert abs(price - float(gold[key + "_price"])) < 1e-4
        return
    assert abs(price - float(gold[key + "_price"])) < 1e-10
    # The last date of the fixture has collinear variables (f = SR, A a
    # function of f): the Gram is singular, the reference's SVD returns the
    # minimum-norm solution and the Cholesky solve another one with the
    # same fit.  Coefficients are compared where the system is regular, the
    # fitted continuation values everywhere.
    np.testing.assert_allclose(beta[:-1, :ncoef], gold[key + "_coef"][:-1], rtol=1e-6, atol=1e-9)
    if norm:
        np.testing.assert_allclose(means, gold[key + "_means"], rtol=1e-12)
        np.testing.assert_allclose(sds, gold[key + "_sds"], rtol=1e-10)
    m = means if norm else np.zeros((E, 3))
    sd = sds if norm else np.ones((E, 3))
    for e in range(E):
        x = (vars_[e] - m[e][:, None]) / sd[e][:, None]
        phi = np.stack([np.prod([x[j] ** int(mono[e, k, j]) for j in range(3)], 0)
                        for k in range(nb[e])])
        fit_mine = beta[e, : nb[e]] @ phi
        fit_ref = gold[key + "_coef"][e, : nb[e]] @ phi
        tol = 1e-7 if e < E - 1 else 1e-5  # singular last date: jitter vs SVD
        assert np.max(np.abs(fit_mine - fit_ref)) < tol


@pytest.mark.parametrize("tag", ["a", "b"])
def test_tarn_flows(orc, gold, tag):
    """TARN flows of the restatement against the reference's gold TARN on
    the gold fixture's reset rates (note b knocks out within a few periods)."""
    aux = gold[f"tarn_{tag}_aux"]
    rate1 = gold["cf_rate1"]
    S, P = rate1.shape
    f1 = np.zeros((S, P), np.float32)
    f2 = np.zeros((S, P), np.float32)
    orc("orc_tarn_flows_f", f1, f2, aux, P, S, rate1, rate1)
    assert np.array_equal(f1, gold[f"tarn_{tag}_flows1"])
    assert np.array_equal(f2, gold[f"tarn_{tag}_flows2"])


@pytest.mark.parametrize("depth", [2, 3, 4])
@pytest.mark.parametrize("cross", [1, 0])
def test_ls_nested_regressions_match_gold(orc, gold, depth, cross):
    """Regression depth 2-4 with the fraction selector against the
    reference's gold (generateRegressionCoefficientsViaLSMultiQuadratic_gold
    and its frozen MultiLSExerciseStrategy second pass, with Andersen
    shifts): in-sample price, cut-offs, per-depth moments and coefficients
    (dates where the Gram is regular), and the second-pass value of the
    oracle's rule and of the gold rule under the oracle's decision chain."""
    import ctypes

    from useful_code_b200 import market as mk

    vars_, cf, ex, num = gold["ls_vars"], gold["ls_cf"], gold["ls_ex3"], gold["ls_num"]
    E, _, P = vars_.shape
    nvars = gold["ls_nvars"]
    mono, nb = mk.basis_tables("cross" if cross else "quadratic", nvars)
    ncoef = int(nb[0])
    lf = 0.1 ** (1.0 / (depth - 1))
    opts = np.array([lf, lf * 1.01, 2.5, 0.8, 20.0])
    beta = np.zeros((E, depth, 16))
    means = np.zeros((E, depth, 3))
    sds = np.zeros((E, depth, 3))
    cuts = np.zeros((E, depth, 2))
    status = np.zeros(1, np.int32)
    price = orc("orc_ls_regress_multi_d", E, P, vars_, nvars, mono, nb, cf, ex, num, 1, depth,
                opts, beta, means, sds, cuts, status, restype=ctypes.c_double)
    key = f"lsd{depth}_cross{cross}"
    assert status[0] == 0
    assert abs(price - float(gold[key + "_price"])) < 1e-10
    lo, hi = gold[key + "_lo"], gold[key + "_hi"]
    # the last depth's cut-offs are never read (the oracle leaves them zero)
    np.testing.assert_allclose(cuts[:, :-1, 0], lo[:, :-1], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(cuts[:, :-1, 1], hi[:, :-1], rtol=1e-6, atol=1e-9)
    used = hi[:, :-1] > 0  # depths regressed: the one after each non-zero cut
    for e in range(E):
        for d in range(depth):
            if d > 0 and not used[e, d - 1]:
                continue
            np.testing.assert_allclose(means[e, d], gold[key + "_means"][e, d], rtol=1e-10)
            np.testing.assert_allclose(sds[e, d], gold[key + "_sds"][e, d], rtol=1e-9)
            if e < E - 1:  # the last date's Gram is singular (f = SR there)
                ref_c = gold[key + "_coef"][e, d]
                np.testing.assert_allclose(beta[e, d, :ncoef], ref_c, rtol=1e-6,
                                           atol=1e-8 * np.abs(ref_c).max())
    shifts = gold["ls_multi_shifts"]
    second = orc("orc_ls_second_pass_multi_d", E, P, vars_, nvars, mono, nb, cf, ex, num, depth,
                 beta, means, sds, cuts, shifts, restype=ctypes.c_double)
    assert abs(second - float(gold[key + "_second"])) < 1e-10
    gb = np.zeros((E, depth, 16))
    gb[:, :, :ncoef] = gold[key + "_coef"]
    gcuts = np.ascontiguousarray(np.stack([lo, hi], -1))
    mixed = orc("orc_ls_second_pass_multi_d", E, P, vars_, nvars, mono, nb, cf, ex, num, depth,
                gb, gold[key + "_means"], gold[key + "_sds"], gcuts, shifts,
                restype=ctypes.c_double)
    assert abs(mixed - float(gold[key + "_second"])) < 1e-12


def test_ab_duality_gap_matches_gold(orc, kref):
    """Andersen–Broadie duality gap: the zero-rebate estimator equals the
    reference's gold (ABDualityGapEstimateZeroRebate) on random exercise
    decisions and continuation estimates; the non-zero-rebate form (restated
    from the root tree, absent from the buildable copy) reduces to it when
    the payoffs are zero and the last step is not an exercise date, and
    responds to payoffs as its formula says on a hand-worked path."""
    rng = np.random.default_rng(11)
    steps, paths = 9, 257
    is_ex = np.array([1, 0, 1, 1, 0, 1, 1, 1, 0], np.int32)
    ex = (rng.random((steps, paths)) < 0.3).astype(np.int32)
    means = rng.normal(0.01, 0.02, (paths, steps))
    sds = np.abs(rng.normal(0, 1e-3, (paths, steps)))
    ref = np.zeros(2)
    kref("kref_ab_gap_zero_rebate", steps, paths, ex, means, sds, is_ex, ref)
    mine = np.zeros(2)
    orc("orc_ab_gap", steps, paths, ex, None, means, is_ex, mine)
    np.testing.assert_allclose(mine, ref, rtol=1e-13, atol=0)
    zero = np.zeros((steps, paths))
    nz = np.zeros(2)
    orc("orc_ab_gap", steps, paths, ex, zero, means, is_ex, nz)
    np.testing.assert_allclose(nz, ref, rtol=1e-13, atol=0)
    # one path by hand: dates 0, 2; exercise at 2; Z = (0.05, 0, 0.04), Q = (0.03, 0, 0.02)
    ex1 = np.array([[0], [0], [1], [0]], np.int32)
    pay1 = np.array([[0.05], [0.0], [0.04], [0.0]])
    q1 = np.array([[0.03, 0.0, 0.02, 0.0]])
    out = np.zeros(2)
    orc("orc_ab_gap", 4, 1, ex1, pay1, q1, np.array([1, 0, 1, 0], np.int32), out)
    # date 0: x = 0.05 - 0.03 = 0.02; date 2: x = 0, balance = 0.02; end: -0.02
    assert abs(out[0] - 0.02) < 1e-15


def test_philox_is_uniform(orc):
    """Philox4x32-10 words of consecutive counters: uniform moments and no
    lag-1 correlation (a smoke check of the restatement; the GPU kernels are
    checked against it word for word)."""
    n = 1 << 16
    ctr = np.zeros((n, 4), np.uint32)
    ctr[:, 0] = np.arange(n, dtype=np.uint32)
    orc("orc_philox4x32_10", ctr, np.uint32(12345), np.uint32(678), n)
    u = (ctr.astype(np.float64) + 0.5) / 2.0**32
    assert abs(u.mean() - 0.5) < 0.003
    assert abs(u.var() - 1 / 12) < 0.002
    flat = u.ravel()
    assert abs(np.corrcoef(flat[:-1], flat[1:])[0, 1]) < 0.01
    assert len(np.unique(ctr[:, 0])) > n - 5
