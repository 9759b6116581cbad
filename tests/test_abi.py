"""The C-ABI library: exports, argument validation and the host-side
set-up routines (CPU only, no kernel launches)."""
import ctypes
import subprocess

import numpy as np
import pytest

from useful_code_b200 import _lib
from useful_code_b200 import market as mk
from useful_code_b200._lib import LIB, LmmError, call

VP = ctypes.c_void_p
FAKE = VP(0x1000)  # never dereferenced: validation fails before any access


def p(a):
    return VP(a.ctypes.data)


def test_every_declared_symbol_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = set(_lib.parse_headers())
    assert declared, "no declarations parsed"
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    assert {"lmm_sobol_ints", "lmm_pipeline_first_pass", "lmm_ls_regress"} <= declared


def test_reference_names_are_exported():
    """Every routine of include/kooderive_compat.h is exported under the
    reference's name: extern "C" ones unmangled, the C++ ones with the
    reference's parameter types."""
    import re

    text = (_lib.ROOT / "include" / "kooderive_compat.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    names = set(re.findall(r"\b(\w+)\s*\(", text)) - {"defined", "if", "push", "pop"}
    extern_c = set(re.findall(r'extern "C"\s+(?:const\s+)?\w+\**\s+(\w+)\s*\(', text))
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    syms = [line.split()[-1] for line in out.splitlines() if " T " in line]
    dem = subprocess.run(["c++filt"], input="\n".join(syms), capture_output=True, text=True,
                         check=True).stdout.splitlines()
    plain = set(syms)
    cxx = {d.split("(")[0] for d in dem if "(" in d}
    assert len(names) >= 29, sorted(names)
    assert extern_c <= plain, sorted(extern_c - plain)
    assert names - extern_c <= cxx, sorted(names - extern_c - cxx)


def test_status_and_message():
    st = LIB.lmm_sobol_ints(16, 70000, 0, FAKE, FAKE, None)
    assert st == 1
    assert b"65535" in LIB.lmm_last_error_string()
    with pytest.raises(LmmError) as ei:
        call("lmm_bridge_transform", FAKE, FAKE, 64, 0, 3, None, None)
    assert ei.value.status == 1
    with pytest.raises(LmmError):
        call("lmm_bridge_transform", FAKE, FAKE, 64, 20, 17, None, None)
    with pytest.raises(LmmError):
        call("lmm_correlate_drift", FAKE, FAKE, FAKE, None, FAKE, 60, 3, 20, 64, 20, 1, None)
    with pytest.raises(LmmError) as ei:
        call("lmm_sobol_ints", 16, 4, 2**31 - 4, FAKE, FAKE, None)
    assert "2^31" in str(ei.value)


def test_ls_regress_rejects_small_workspace():
    E, P = 4, 1000
    nv = np.full(E, 3, np.int32)
    mono, nb = mk.basis_tables("cross", nv)
    need = LIB.lmm_ls_workspace_bytes(P, E)
    st = LIB.lmm_ls_regress(E, P, FAKE, p(nv), p(mono), p(nb), None, None, FAKE, 1, FAKE,
                            need - 1, FAKE, FAKE, FAKE, None, FAKE, FAKE, None)
    assert st == 1 and b"workspace" in LIB.lmm_last_error_string()


def test_pipeline_rejects_bad_schedules():
    from useful_code_b200.pricer import LmmModel, LmmProduct

    n, F = 8, 2
    taus = np.full(n, 0.5, np.float32)
    disp = np.zeros(n, np.float32)
    f0 = np.full(n, 0.05, np.float32)
    model = LmmModel(n, F, p(taus), p(disp), p(f0), FAKE, FAKE, FAKE, None, 0, 10.0)
    ex = np.array([3, 2], np.int32)  # not increasing
    nv = np.full(2, 3, np.int32)
    mono, nb = mk.basis_tables("cross", nv)
    prod = LmmProduct(0, 0.05, 0.05, 1.0, 2, p(ex), p(nv), p(mono), p(nb), 1)
    st = LIB.lmm_pipeline_first_pass(ctypes.addressof(model), ctypes.addressof(prod), 64, 0, 1,
                                     FAKE, 1 << 30, 64, 0, FAKE, FAKE, FAKE, FAKE, None)
    assert st == 1 and b"exercise" in LIB.lmm_last_error_string()
    assert LIB.lmm_pipeline_workspace_bytes(ctypes.addressof(model), ctypes.addressof(prod), 64, 1) == 0
    # monomial using an absent variable
    ex2 = np.array([2, 7], np.int32)
    nv2 = np.array([3, 1], np.int32)
    mono2, nb2 = mk.basis_tables("cross", np.array([3, 3], np.int32))
    prod2 = LmmProduct(0, 0.05, 0.05, 1.0, 2, p(ex2), p(nv2), p(mono2), p(nb2), 1)
    st = LIB.lmm_pipeline_first_pass(ctypes.addressof(model), ctypes.addressof(prod2), 64, 0, 1,
                                     FAKE, 1 << 30, 64, 0, FAKE, FAKE, FAKE, FAKE, None)
    assert st == 1 and b"absent variable" in LIB.lmm_last_error_string()


def test_host_mt19937_matches_reference(gold):
    out = np.zeros(1000, np.uint32)
    call("lmm_mt19937_words", 1234, 1000, p(out))
    assert np.array_equal(out, gold["mt19937_seed1234"])


def test_host_directions(ref_dirs, orc):
    # The product's default table is the reference's: its directions on all
    # 1,800 shipped dimensions equal the reference's own
    # initSobolDirectionVectors output.
    assert mk.SOBOL_TABLE == "joe-kuo-6.10200"
    assert np.array_equal(mk.sobol_directions(1800), ref_dirs)
    # The scipy Joe–Kuo table agrees with the reference's table on its first
    # 211 dimensions (the tables diverge afterwards).
    deg, a, m = mk.joe_kuo_table(211, "new-joe-kuo-6.21201")
    out = np.zeros((211, 32), np.uint32)
    call("lmm_sobol_directions", 211, p(deg), p(a), p(m), m.shape[1], p(out))
    assert np.array_equal(out, ref_dirs[:211])
    assert not np.array_equal(mk.sobol_directions(400, "new-joe-kuo-6.21201"), ref_dirs[:400])
    # the oracle's independent restatement gives the same numbers on 1800 dims
    deg, a, m = mk.joe_kuo_table(1800, "new-joe-kuo-6.21201")
    mine = np.zeros((1800, 32), np.uint32)
    orcd = np.zeros((1800, 32), np.uint32)
    call("lmm_sobol_directions", 1800, p(deg), p(a), p(m), m.shape[1], p(mine))
    orc("orc_sobol_directions", 1800, deg, a, m, m.shape[1], orcd)
    assert np.array_equal(mine, orcd)


@pytest.mark.parametrize("F,S", [(3, 20), (5, 40), (10, 80), (15, 120)])
def test_host_bridge_allocation(gold, F, S):
    out = np.zeros((F, S), np.int32)
    call("lmm_bridge_allocate_diagonal", F, S, p(out))
    assert np.array_equal(out, gold[f"alloc_diag_F{F}_S{S}"])


def test_host_pseudo_roots_match_reference(gold):
    A_ref = gold["lmm_A64"]
    n, _, F = A_ref.shape
    rs = np.array([0.5 * (i + 1) for i in range(n)])
    out = np.zeros_like(A_ref)
    call("lmm_abcd_pseudo_roots", 0.05, 0.09, 0.44, 0.11, p(rs), n, p(rs), n, p(np.ones(n)), F,
         0.0, 0.1, p(out))
    cov = np.einsum("srf,sqf->srq", out, out)
    cov_ref = np.einsum("srf,sqf->srq", A_ref, A_ref)
    assert np.max(np.abs(cov - cov_ref)) < 1e-15
    # columns agree up to the sign of each eigenvector
    assert np.max(np.abs(np.abs(out) - np.abs(A_ref))) < 1e-12
    assert np.max(np.abs(out[0] - A_ref[0])) < 1e-12


def test_host_fixed_and_spot_drifts(gold, orc):
    A = gold["lmm_A"]
    S, n, F = A.shape
    fixed = np.zeros((S, n), np.float32)
    call("lmm_fixed_drifts", p(A), S, n, F, p(fixed))
    assert np.max(np.abs(fixed - gold["lmm_fixed"])) < 1e-9
    mu = np.zeros(n, np.float32)
    call("lmm_spot_drifts", p(A[0]), p(gold["lmm_f0"]), p(gold["lmm_tau"]), p(gold["lmm_disp"]),
         n, F, p(mu))
    mu_d = np.zeros(n)
    orc("orc_spot_drift_d", A[0].astype(np.float64), gold["lmm_f0"].astype(np.float64),
        gold["lmm_tau"].astype(np.float64), gold["lmm_disp"].astype(np.float64), n, F, mu_d)
    assert np.max(np.abs(mu - mu_d)) < 1e-8


def test_host_cashflow_indices_and_exercise_mapping(gold):
    rt = gold["cf_rate_times"]
    n = rt.size - 1
    for pay, key in [(rt[1:].copy(), ""), (gold["cf_pay_mid"], "_mid")]:
        fi = np.zeros(n, np.int32)
        si = np.zeros(n, np.int32)
        th = np.zeros(n, np.float32)
        call("lmm_cashflow_indices_weights", p(rt), n + 1, p(pay), n, p(fi), p(si), p(th))
        assert np.array_equal(fi, gold["cf_first" + key])
        assert np.array_equal(si, gold["cf_second" + key])
        assert np.array_equal(th, gold["cf_theta" + key])
    gen = np.arange(n, dtype=np.int32)
    ex = gold["cf_ex_idx"]
    out = np.zeros(n, np.int32)
    first = np.zeros(1, np.int32)
    call("lmm_step_to_exercise_indices", p(gen), n, p(ex), ex.size, p(out), p(first))
    assert np.array_equal(out, gold["cf_step_to_ex"])
    assert int(first[0]) == int(gold["cf_first_positive"])


def test_basis_tables_follow_reference_generators():
    mono, nb = mk.basis_tables("cross", np.array([3, 2, 1], np.int32))
    assert list(nb) == [10, 6, 3]
    assert [tuple(x) for x in mono[0, :10]] == [
        (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (0, 1, 1), (1, 0, 1),
        (2, 0, 0), (0, 2, 0), (0, 0, 2)]
    mono, nb = mk.basis_tables("quadratic", np.array([3], np.int32))
    assert [tuple(x) for x in mono[0, :7]] == [
        (0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (0, 2, 0), (0, 0, 1), (0, 0, 2)]
    mono, nb = mk.basis_tables("c2", np.array([3, 2, 1], np.int32))
    assert list(nb) == [6, 5, 2]


def _mini_model_product(kind=0, n=8, F=2, tarn_total=0.15):
    from useful_code_b200.pricer import LmmModel, LmmProduct

    taus = np.full(n, 0.5, np.float32)
    disp = np.zeros(n, np.float32)
    f0 = np.full(n, 0.05, np.float32)
    keep = [taus, disp, f0]
    model = LmmModel(n, F, p(taus), p(disp), p(f0), FAKE, FAKE, FAKE, None, 0, 10.0)
    ex = np.array([2, 5], np.int32)
    nv = np.full(2, 3, np.int32)
    mono, nb = mk.basis_tables("cross", nv)
    keep += [ex, nv, mono, nb]
    prod = LmmProduct(kind, 0.05, 0.05, 1.0, 2, p(ex), p(nv), p(mono), p(nb), 1, tarn_total,
                      2.0)
    return model, prod, keep


def test_nested_regression_rejects_bad_selectors():
    from useful_code_b200.pricer import LmmLsSelect

    E, P = 4, 1000
    nv = np.full(E, 3, np.int32)
    mono, nb = mk.basis_tables("cross", nv)
    need = LIB.lmm_ls_nested_workspace_bytes(P, E)
    assert need > LIB.lmm_ls_workspace_bytes(P, E)

    def run(sel, ws=need):
        return LIB.lmm_ls_regress_nested(E, P, FAKE, p(nv), p(mono), p(nb), None, None, FAKE, 1,
                                         ctypes.addressof(sel), FAKE, ws, FAKE, FAKE, FAKE,
                                         FAKE, None, FAKE, FAKE, None)

    assert run(LmmLsSelect(9, 0.1, 0.101, 2.5, 0.8, 900)) == 1
    assert b"depth" in LIB.lmm_last_error_string()
    assert run(LmmLsSelect(3, 0.2, 0.1, 2.5, 0.8, 900)) == 1  # upper below lower
    assert b"lower_frac" in LIB.lmm_last_error_string()
    assert run(LmmLsSelect(3, 0.1, 0.101, 2.5, 1.2, 900)) == 1  # multiplier >= 1
    assert run(LmmLsSelect(3, 0.1, 0.101, 2.5, 0.8, 900), need - 1) == 1
    assert b"workspace" in LIB.lmm_last_error_string()


def test_rule_second_pass_and_ab_reject_bad_inputs():
    from useful_code_b200.pricer import LmmAbConfig, LmmLsRule

    model, prod, keep = _mini_model_product()
    m, pr = ctypes.addressof(model), ctypes.addressof(prod)
    rule = LmmLsRule(3, 0x1000, None, None, None, None)  # depth 3 without cuts
    st = LIB.lmm_pipeline_second_pass_rule(m, pr, 64, 0, 1, ctypes.addressof(rule), FAKE,
                                           1 << 30, FAKE, None)
    assert st == 1 and b"cut-offs" in LIB.lmm_last_error_string()
    rule = LmmLsRule(0, 0x1000, None, None, None, None)
    st = LIB.lmm_pipeline_second_pass_rule(m, pr, 64, 0, 1, ctypes.addressof(rule), FAKE,
                                           1 << 30, FAKE, None)
    assert st == 1 and b"depth" in LIB.lmm_last_error_string()
    ok = LmmLsRule(1, 0x1000, None, None, None, None)
    bad_inner = LmmAbConfig(64, 0, 100, 1)
    assert LIB.lmm_andersen_broadie_workspace_bytes(m, pr, ctypes.addressof(bad_inner)) == 0
    st = LIB.lmm_andersen_broadie(m, pr, ctypes.addressof(ok), ctypes.addressof(bad_inner),
                                  FAKE, 1 << 30, FAKE, None, None, None, None, None, None)
    assert st == 1 and b"multiple of 128" in LIB.lmm_last_error_string()
    cfg = LmmAbConfig(64, 0, 256, 1)
    assert LIB.lmm_andersen_broadie_workspace_bytes(m, pr, ctypes.addressof(cfg)) > 0
    model2, prod2, keep2 = _mini_model_product(kind=1)  # cancellable swap
    st = LIB.lmm_andersen_broadie(ctypes.addressof(model2), ctypes.addressof(prod2),
                                  ctypes.addressof(ok), ctypes.addressof(cfg), FAKE, 1 << 30,
                                  FAKE, None, None, None, None, None, None)
    assert st == 1 and b"swaption" in LIB.lmm_last_error_string()
    st = LIB.lmm_ab_duality_gap(0, 10, FAKE, FAKE, None, FAKE, FAKE, 1 << 20, FAKE, None)
    assert st == 1


def test_tarn_needs_a_positive_total():
    model, prod, keep = _mini_model_product(kind=3, tarn_total=0.0)
    st = LIB.lmm_pipeline_second_pass(ctypes.addressof(model), ctypes.addressof(prod), 64, 0, 1,
                                      None, None, None, FAKE, 1 << 30, FAKE, None)
    assert st == 1 and b"TARN" in LIB.lmm_last_error_string()


def test_segmented_price_rejects_bad_inputs():
    """lmm_fused_price: a stopping product needs a rule, and the segmented
    chain needs its survivor buffers; one launch (segment >= rates) needs
    none, and products that never stop need no workspace."""
    from useful_code_b200.pricer import LmmLsRule

    model, prod, keep = _mini_model_product()
    m, pr = ctypes.addressof(model), ctypes.addressof(prod)
    need = LIB.lmm_fused_price_workspace_bytes(m, pr, 1000)
    assert need > 1000 * 4
    st = LIB.lmm_fused_price(m, pr, 1000, FAKE, None, 0, FAKE, 1 << 30, FAKE, None)
    assert st == 1 and b"null rule" in LIB.lmm_last_error_string()
    rule = LmmLsRule(1, 0x1000, None, None, None, None)
    # 8 rates: segments of 2 steps need the survivor buffers (the default 8
    # steps would be one launch, which needs none)
    st = LIB.lmm_fused_price(m, pr, 1000, FAKE, ctypes.addressof(rule), 2, FAKE, need // 2,
                             FAKE, None)
    assert st == 1 and b"workspace" in LIB.lmm_last_error_string()
    st = LIB.lmm_fused_price(m, pr, 1000, FAKE, ctypes.addressof(rule), 2, None, 0, FAKE, None)
    assert st == 1 and b"workspace" in LIB.lmm_last_error_string()
    st = LIB.lmm_fused_price(m, pr, 0, FAKE, ctypes.addressof(rule), 0, FAKE, 1 << 30, FAKE,
                             None)
    assert st == 1
    model3, prod3, keep3 = _mini_model_product(kind=2)  # European strip: never stops
    assert LIB.lmm_fused_price_workspace_bytes(ctypes.addressof(model3),
                                               ctypes.addressof(prod3), 1000) == 256
