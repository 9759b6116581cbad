"""Generate the golden fixtures in tests/golden/ from the reference's gold code.

Runs the reference's own CPU routines (oracle/_ref/libkooref.so, built by
``make -C oracle ref`` from the reference sources in place) and the
reference's newBridge host code (oracle/_ref/libkoobridge.so, ``make -C
oracle bridge``) on small seeded
inputs and stores inputs and outputs as .npz fixtures.  Stage-wise: each
stage is fed the previous gold stage's output, as the reference's own tests
do (LMM_evolver_test.cu:2487-2525).  Only this script reads the reference;
the fixtures travel with the repository.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_LIB = ROOT / "oracle" / "_ref" / "libkooref.so"
BRIDGE_LIB = ROOT / "oracle" / "_ref" / "libkoobridge.so"

P = ctypes.c_void_p
D = ctypes.c_double
F_ = ctypes.c_float


def ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return P(a.ctypes.data)


def main() -> int:
    if not REF_LIB.exists():
        print(f"{REF_LIB} missing: run `make -C oracle ref` first", file=sys.stderr)
        return 1
    ref = ctypes.CDLL(str(REF_LIB))
    ref.kref_ls_multi.restype = ctypes.c_double
    ref.kref_ls_multi_depth.restype = ctypes.c_double
    ref.kref_ls_multi_second_pass.restype = ctypes.c_double
    ref.kref_step_to_exercise.restype = ctypes.c_int

    # --- Sobol direction numbers of the reference table (1800 dims) -------
    dims = 1800
    dirs = np.zeros((dims, 32), np.uint32)
    ref.kref_sobol_directions(dims, ptr(dirs))
    np.save(HERE / "sobol_directions_ref1800.npy", dirs)
    # the product's table covers the library's largest model (128 rates x
    # 16 factors)
    write_direction_table(ref, 2048)

    out = {}
    rng = np.random.default_rng(20240611)

    # --- Sobol integers with offset splits (Sobol_int_test.cu:37-200) ------
    n_paths, n_dims = 1024, 64
    sob = np.zeros((n_dims, n_paths), np.uint32)
    ref.kref_sobol_ints_offset(n_paths, n_dims, 0, ptr(dirs), ptr(sob))
    sob_off = np.zeros((n_dims, 512), np.uint32)
    ref.kref_sobol_ints_offset(512, n_dims, 777, ptr(dirs), ptr(sob_off))
    out.update(sobol_p1024_d64_off0=sob, sobol_p512_d64_off777=sob_off)

    # --- scramble with the reference test's scramblers 6i^2+2i+1 -----------
    # (scramble_test.cu:77), data i*n+p
    sd, sp = 32, 256
    data = (np.arange(sd, dtype=np.uint64)[:, None] * sp + np.arange(sp)[None, :]).astype(np.uint32)
    scr = np.array([(6 * i * i + 2 * i + 1) & 0xFFFFFFFF for i in range(sd)], np.uint32)
    scr_out = np.zeros_like(data)
    ref.kref_scramble(ptr(data), ptr(scr_out), ptr(scr), sd, sp)
    out.update(scramble_in=data, scramble_scr=scr, scramble_out=scr_out)

    # --- Shaw–Brickman inverse normal on assorted integers -----------------
    ints = np.concatenate([
        rng.integers(0, 2**32, 4096, dtype=np.uint64).astype(np.uint32),
        np.array([1, 2, 127, 128, 2**31 - 1, 2**31, 2**31 + 1, 2**32 - 256, 2**32 - 257], np.uint32),
    ])
    icdf = np.zeros(ints.size, np.float32)
    ref.kref_icdf_sb(ptr(ints), ptr(icdf), ctypes.c_long(ints.size))
    out.update(icdf_in=ints, icdf_sb=icdf)

    # --- bridge allocation -------------------------------------------------
    for F, S in [(3, 20), (5, 40), (10, 80), (15, 120)]:
        a = np.zeros((F, S), np.int32)
        ref.kref_bridge_allocate_diagonal(F, S, ptr(a))
        out[f"alloc_diag_F{F}_S{S}"] = a

    # --- MT19937 scrambler words -------------------------------------------
    mt = np.zeros(1000, np.uint32)
    ref.kref_mt19937(ctypes.c_ulong(1234), 1000, ptr(mt))
    out["mt19937_seed1234"] = mt

    # --- small LMM case: pseudo-roots, correlate, PC evolve, curve stages ---
    n, F, Pp = 12, 3, 512
    tau = np.full(n, 0.5, np.float32)
    f0 = np.linspace(0.04, 0.06, n).astype(np.float32)
    disp = np.full(n, 0.015, np.float32)
    rate_starts = np.array([0.5 * (i + 1) for i in range(n)])
    A64 = np.zeros((n, n, F))
    ones = np.ones(n)
    ref.kref_abcd_pseudo_roots(D(0.05), D(0.09), D(0.44), D(0.11), ptr(rate_starts), n,
                               ptr(rate_starts), n, ptr(ones), F, D(0.0), D(0.1), ptr(A64))
    A = A64.astype(np.float32)
    fixed = (-0.5 * (A.astype(np.float32) ** 2).sum(-1)).astype(np.float32)
    z = rng.standard_normal((n, Pp, F)).astype(np.float32)  # [S][P][F]
    corr = np.zeros((n, n, Pp), np.float32)
    ref.kref_correlate_drift_f(ptr(z), ptr(corr), ptr(A), n * F, ptr(fixed), F, n, Pp, n)
    rates = np.zeros((n, n, Pp), np.float32)
    lrates = np.zeros_like(rates)
    ref.kref_lmm_pc_f(ptr(f0), ptr(tau), ptr(corr), ptr(A), ptr(disp), Pp, F, n, n, F_(10.0),
                      ptr(rates), ptr(lrates))
    alive = np.arange(n, dtype=np.int32)
    disc = np.zeros((n, n + 1, Pp), np.float32)
    ref.kref_discount_ratios_f(ptr(rates), ptr(tau), ptr(alive), Pp, n, n, ptr(disc))
    ann = np.zeros((n, n, Pp), np.float32)
    ref.kref_annuities_f(ptr(disc), ptr(tau), ptr(alive), Pp, n, n, ptr(ann))
    sr = np.zeros((n, n, Pp), np.float32)
    ref.kref_swap_rates_f(ptr(disc), ptr(ann), ptr(alive), Pp, n, n, ptr(sr))
    num = np.zeros((n, Pp), np.float32)
    ref.kref_numeraires_f(ptr(disc), Pp, Pp, 0, n, ptr(num))
    out.update(lmm_A64=A64, lmm_A=A, lmm_fixed=fixed, lmm_z_spf=z, lmm_tau=tau, lmm_f0=f0,
               lmm_disp=disp, lmm_corr=corr, lmm_rates=rates, lmm_logrates=lrates,
               lmm_disc=disc, lmm_ann=ann, lmm_sr=sr, lmm_num=num)

    # --- cash flows, discounting, indices/weights, aggregation --------------
    rate_times = np.array([0.5 * (i + 1) for i in range(n + 1)], np.float32)
    pay = rate_times[1:].copy()
    first = np.zeros(n, np.int32)
    second = np.zeros(n, np.int32)
    theta = np.zeros(n, np.float32)
    ref.kref_indices_weights_f(ptr(rate_times), n + 1, ptr(pay), n, ptr(first), ptr(second), ptr(theta))
    pay_mid = (rate_times[:-1] + 0.3).astype(np.float32)
    first_m = np.zeros(n, np.int32)
    second_m = np.zeros(n, np.int32)
    theta_m = np.zeros(n, np.float32)
    ref.kref_indices_weights_f(ptr(rate_times), n + 1, ptr(pay_mid), n, ptr(first_m), ptr(second_m), ptr(theta_m))
    rate1 = np.ascontiguousarray(np.stack([rates[s, s] for s in range(n)]))  # [S][P]
    aux = np.concatenate([[0.05, 1.0], np.full(n, 0.5), np.full(n, 0.5)]).astype(np.float32)
    fl1 = np.zeros((n, Pp), np.float32)
    fl2 = np.zeros((n, Pp), np.float32)
    ref.kref_swap_flows_f(ptr(fl1), ptr(fl2), ptr(aux), Pp, n, ptr(rate1))
    dflows = np.zeros((n, Pp), np.float32)
    summed = np.zeros(Pp, np.float32)
    ref.kref_discounting_f(ptr(first_m), ptr(second_m), ptr(theta_m), ptr(disc), ptr(fl2), ptr(num),
                           Pp, n, ptr(dflows), ptr(summed))
    # TARN flows: the reference test's note (total 0.15, strike 0.10, m 2) and
    # one whose coupons reach the total within a few periods (strike 0.20)
    for tag, strike in (("a", 0.10), ("b", 0.20)):
        taux = np.concatenate([[0.15, strike, 2.0], np.full(n, 0.5), np.full(n, 0.5)]).astype(np.float32)
        t1 = np.zeros((n, Pp), np.float32)
        t2 = np.zeros((n, Pp), np.float32)
        ref.kref_tarn_flows_f(ptr(t1), ptr(t2), ptr(taux), Pp, n, ptr(rate1))
        out[f"tarn_{tag}_aux"] = taux
        out[f"tarn_{tag}_flows1"] = t1
        out[f"tarn_{tag}_flows2"] = t2
    gen = np.arange(n, dtype=np.int32)
    ex_idx = np.array([2, 5, 8, 11], np.int32)
    s2e = np.zeros(n, np.int32)
    first_pos = ref.kref_step_to_exercise(ptr(gen), n, ptr(ex_idx), ex_idx.size, ptr(s2e))
    target = np.array([ex_idx[j] if j >= 0 else 0 for j in s2e], np.int32)
    pflows = np.zeros((n, Pp), np.float32)
    ref.kref_discounting_partial_f(n, ptr(gen), ptr(first), ptr(second), ptr(theta), ptr(target),
                                   ptr(disc), ptr(fl2), ptr(num), Pp, n, ptr(pflows))
    agg = np.zeros((ex_idx.size, Pp), np.float32)
    ref.kref_aggregate_f(ptr(agg), Pp, ex_idx.size, ptr(pflows), Pp, 0, n, ptr(s2e))
    out.update(cf_rate_times=rate_times, cf_first=first, cf_second=second, cf_theta=theta,
               cf_pay_mid=pay_mid, cf_first_mid=first_m, cf_second_mid=second_m,
               cf_theta_mid=theta_m, cf_rate1=rate1, cf_aux=aux, cf_flows1=fl1, cf_flows2=fl2,
               cf_discounted=dflows, cf_summed=summed, cf_ex_idx=ex_idx, cf_step_to_ex=s2e,
               cf_first_positive=np.int32(first_pos), cf_target=target, cf_partial=pflows,
               cf_aggregated=agg)

    # --- exercise values and basis variables --------------------------------
    E = ex_idx.size
    r1 = np.ascontiguousarray(np.stack([rates[e, e] for e in ex_idx]))
    r2 = np.ascontiguousarray(np.stack([sr[e, e] for e in ex_idx]))
    r3 = np.ascontiguousarray(np.stack([ann[e, e] for e in ex_idx]))
    exv = np.zeros((E, Pp), np.float32)
    ref.kref_payer_swaption_values_f(F_(0.05), ptr(r2), ptr(r3), Pp, Pp, 0, n, E, ptr(ex_idx), ptr(exv))
    shifts = np.array([0.015, 0.015, 0.0], np.float32)
    bv_raw = np.zeros((E, 3, Pp), np.float32)
    ref.kref_basis_variables_f(0, ptr(shifts), ptr(r1), ptr(r2), ptr(r3), Pp, Pp, 0, n, E, ptr(ex_idx), ptr(bv_raw))
    bv_log = np.zeros((E, 3, Pp), np.float32)
    ref.kref_basis_variables_f(1, ptr(shifts), ptr(r1), ptr(r2), ptr(r3), Pp, Pp, 0, n, E, ptr(ex_idx), ptr(bv_log))
    out.update(ex_r1=r1, ex_r2=r2, ex_r3=r3, ex_values=exv, bv_shifts=shifts, bv_raw=bv_raw,
               bv_log=bv_log)

    # --- Longstaff–Schwartz (depth 1) on gold-generated data ----------------
    numE = np.ascontiguousarray(np.stack([num[e] for e in ex_idx])).astype(np.float64)
    vars64 = bv_raw.astype(np.float64)
    cf64 = agg.astype(np.float64)
    ex64 = exv.astype(np.float64)
    nvars = np.full(E, 3, np.int32)
    for cross, ncoef in [(1, 10), (0, 7)]:
        for norm in (1, 0):
            coef = np.zeros((E, 1, ncoef))
            means = np.zeros((E, 1, 3))
            sds = np.zeros((E, 1, 3))
            price = ref.kref_ls_multi(E, Pp, ptr(vars64), ptr(nvars), ptr(cf64), ptr(ex64), ptr(numE),
                                      cross, norm, ptr(coef), ncoef, ptr(means), ptr(sds))
            key = f"ls_cross{cross}_norm{norm}"
            out[key + "_coef"] = coef[:, 0, :]
            out[key + "_means"] = means[:, 0, :]
            out[key + "_sds"] = sds[:, 0, :]
            out[key + "_price"] = np.float64(price)
    out.update(ls_vars=vars64, ls_cf=cf64, ls_ex=ex64, ls_num=numE, ls_nvars=nvars)

    # --- nested regressions (depth 2-4) with the fraction selector ----------
    # Exercise values tripled so that every date has net continuation values
    # of both signs (the buildable gold copy lacks the one-sign shortcut of
    # the root tree's gold/MultiLS_regression.cpp:212-225).  Selector
    # settings of kooexample/main.cpp:143-178: lower fraction
    # 0.1^(1/(depth-1)), upper = 1.01 x lower, 2.5 sds, multiplier 0.8;
    # at least 20 paths per nested regression (512 paths here).
    ex3 = np.ascontiguousarray(ex64 * 3.0)
    shifts = np.linspace(0.0, 0.002, E)
    out.update(ls_ex3=ex3, ls_multi_shifts=shifts)
    for depth in (2, 3, 4):
        lf = 0.1 ** (1.0 / (depth - 1))
        for cross, ncoef in [(1, 10), (0, 7)]:
            coef = np.zeros((E, depth, ncoef))
            means = np.zeros((E, depth, 3))
            sds = np.zeros((E, depth, 3))
            lo = np.zeros((E, depth))
            hi = np.zeros((E, depth))
            price = ref.kref_ls_multi_depth(E, Pp, ptr(vars64), ptr(nvars), ptr(cf64), ptr(ex3),
                                            ptr(numE), cross, 1, depth, ctypes.c_double(lf),
                                            ctypes.c_double(lf * 1.01), ctypes.c_double(2.5),
                                            ctypes.c_double(0.8), 20, ptr(coef), ncoef, ptr(means),
                                            ptr(sds), ptr(lo), ptr(hi))
            second = ref.kref_ls_multi_second_pass(E, Pp, ptr(vars64), ptr(nvars), ptr(cf64),
                                                   ptr(ex3), ptr(numE), cross, depth, ptr(coef), ncoef,
                                                   ptr(means), ptr(sds), ptr(lo), ptr(hi),
                                                   ptr(shifts))
            key = f"lsd{depth}_cross{cross}"
            out.update({key + "_coef": coef, key + "_means": means, key + "_sds": sds,
                        key + "_lo": lo, key + "_hi": hi, key + "_price": np.float64(price),
                        key + "_second": np.float64(second)})

    np.savez_compressed(HERE / "kooderive_gold_small.npz", **out)
    print("wrote", HERE / "kooderive_gold_small.npz", "and sobol_directions_ref1800.npy")
    return make_bridge_fixtures()


def write_direction_table(ref, dims: int) -> None:
    """The reference's primitive-polynomial table (Joe and Kuo's published
    direction numbers, file joe-kuo-6.10200, compiled into the reference as
    gold/sobol_primitives.cpp) for the first `dims` dimensions: the
    product's default Sobol table (useful_code_b200.market), so the
    product draws the reference's points.  Row d holds the degree, the
    interior coefficient bits and the 17 initial direction integers of
    dimension d (row 0 is the special first dimension)."""
    deg = np.zeros(dims, np.uint32)
    a = np.zeros(dims, np.uint32)
    m = np.zeros((dims, 17), np.uint32)
    d1 = np.zeros(1, np.uint32)
    a1 = np.zeros(1, np.uint32)
    m1 = np.zeros(17, np.uint32)
    for d in range(dims):
        ref.kref_sobol_primitive(d, ptr(d1), ptr(a1), ptr(m1))
        deg[d], a[d], m[d] = d1[0], a1[0], m1
    out = ROOT / "useful_code_b200" / "data" / "joe_kuo_6_10200.npz"
    out.parent.mkdir(exist_ok=True)
    np.savez_compressed(out, degree=deg, a=a, m=m)
    print("wrote", out)


def make_bridge_fixtures() -> int:
    """The reference's newBridge (brownian_bridge::transformCPU,
    brownian_bridge.cu:401-455, tables :639-697) on seeded normals, at the
    (steps, factors) of the five benchmark forms plus ragged shapes, with
    the diagonal allocation and with one explicit permuted allocation."""
    if not BRIDGE_LIB.exists():
        print(f"{BRIDGE_LIB} missing: run `make -C oracle bridge` first", file=sys.stderr)
        return 1
    kb = ctypes.CDLL(str(BRIDGE_LIB))
    rng = np.random.default_rng(20261203)
    out = {}
    P = 8
    for S, F in [(20, 3), (40, 5), (80, 10), (120, 15), (1, 1), (2, 1), (7, 2), (33, 4), (64, 16)]:
        z = rng.standard_normal((F * S, P)).astype(np.float32)
        w = np.zeros((S, F, P), np.float32)
        rc = kb.kref_newbridge_transform(S, F, P, None, ptr(z), ptr(w))
        assert rc == 0, (S, F)
        out[f"bridge_S{S}_F{F}_in"] = z
        out[f"bridge_S{S}_F{F}_out"] = w
    S, F = 12, 3
    alloc = rng.permutation(S * F).astype(np.int32).reshape(F, S)
    z = rng.standard_normal((F * S, P)).astype(np.float32)
    w = np.zeros((S, F, P), np.float32)
    assert kb.kref_newbridge_transform(S, F, P, ptr(alloc), ptr(z), ptr(w)) == 0
    out.update(bridge_perm_alloc=alloc, bridge_perm_in=z, bridge_perm_out=w)
    # the power-of-two bridge (BrownianBridge<float>) and the multi-factor
    # reordering bridge (BrownianBridgeMultiDim<float>, orderings row,
    # column, triangular) of the reference's gold code
    ref = ctypes.CDLL(str(REF_LIB))
    for k in (1, 3, 5, 7):
        n = 1 << k
        z = rng.standard_normal((n, P)).astype(np.float32)
        w = np.zeros((n, P), np.float32)
        ref.kref_bridge_pow2_f(k, P, ptr(z), ptr(w))
        out[f"pow2_k{k}_in"] = z
        out[f"pow2_k{k}_out"] = w
    for k, F in ((3, 3), (4, 5)):
        for ordering in (0, 1, 2):
            N = F << k
            z = rng.standard_normal((N, P)).astype(np.float32)
            w = np.zeros((N, P), np.float32)
            dims = np.zeros(N, np.int32)
            facs = np.zeros(N, np.int32)
            ref.kref_bridge_multi_f(k, F, ordering, P, ptr(z), ptr(w), ptr(dims), ptr(facs))
            tag = f"multi_k{k}_F{F}_o{ordering}"
            out.update({tag + "_in": z, tag + "_out": w, tag + "_dims": dims,
                        tag + "_facs": facs})
    np.savez_compressed(HERE / "kooderive_bridge.npz", **out)
    print("wrote", HERE / "kooderive_bridge.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main())
