"""The reference's GPU entry points by their own names (include/
kooderive_compat.h), called through ctypes exactly as a caller compiled
against the reference's headers would call them (GPU).

extern "C" routines are looked up by name; the C++ routines by their
mangled names (nm + c++filt); `const std::vector<int>&` arguments are
passed as libstdc++'s vector layout (begin, end, end of storage).  Each
result is compared with the reference's gold code (fixtures) where it has
one, else with the lmm_* entry point the routine forwards to or a NumPy
restatement of the reference kernel cited beside the test.
"""
import ctypes
import subprocess

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p
F32 = ctypes.c_float


def _torch():
    import torch

    return torch


_KEEP = []


@pytest.fixture(autouse=True)
def _release():
    yield
    _KEEP.clear()


def dev(a):
    torch = _torch()
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
    _KEEP.append(t)
    return t


def zeros(shape, dtype=np.float32):
    torch = _torch()
    t = torch.zeros(shape, dtype={np.float32: torch.float32, np.int32: torch.int32}[dtype],
                    device="cuda")
    _KEEP.append(t)
    return t


def d(t):
    return VP(t.data_ptr())


def host(t, dtype=None):
    _torch().cuda.synchronize()
    a = t.cpu().numpy()
    return a.view(np.uint32) if dtype == np.uint32 else a


class StdVectorInt(ctypes.Structure):
    """libstdc++'s std::vector<int>: pointers to the first element, one
    past the last, and one past the storage."""
    _fields_ = [("begin", VP), ("end", VP), ("cap", VP)]


def stdvec(a):
    a = np.ascontiguousarray(a, np.int32)
    _KEEP.append(a)
    b = a.ctypes.data
    v = StdVectorInt(b, b + 4 * a.size, b + 4 * a.size)
    _KEEP.append(v)
    return ctypes.byref(v)


@pytest.fixture(scope="module")
def lib():
    from useful_code_b200._lib import LIB_PATH

    return ctypes.CDLL(str(LIB_PATH))


@pytest.fixture(scope="module")
def cxx(lib):
    """C++ routine name -> callable (looked up by its mangled symbol)."""
    from useful_code_b200._lib import LIB_PATH

    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    mangled = [ln.split()[-1] for ln in out.splitlines() if ln.split()[-1].startswith("_Z")]
    dem = subprocess.run(["c++filt"], input="\n".join(mangled), capture_output=True, text=True,
                         check=True).stdout.splitlines()
    table = {dm.split("(")[0]: mg for mg, dm in zip(mangled, dem) if "(" in dm}
    return lambda name: getattr(lib, table[name])


# ---------------------------------------------------------------- Sobol ----
def test_sobol_and_scramble(cuda, lib, gold, ref_dirs):
    out = zeros((64, 1024), np.int32)
    lib.sobolGPUInts(1024, 64, ctypes.c_uint(0), d(dev(ref_dirs[:64])), d(out))
    assert np.array_equal(host(out, np.uint32), gold["sobol_p1024_d64_off0"])
    data = dev(gold["scramble_in"])
    D, P = gold["scramble_in"].shape
    lib.scramble_gpu(d(data), d(dev(gold["scramble_scr"])), D, P)
    assert np.array_equal(host(data, np.uint32), gold["scramble_out"])


# -------------------------------------------------------------- bridges ----
@pytest.mark.parametrize("k", [1, 3, 5, 7])
def test_power_of_two_bridge_matches_gold(cuda, lib, gold_bridge, k):
    """brownianBridgeGPU_constant_memory against the reference's
    BrownianBridge<float> (gold/Bridge_gold.h:168-327), 2e-7 mean relative
    (Bridge_Test.cu:35)."""
    z = gold_bridge[f"pow2_k{k}_in"]
    ref = gold_bridge[f"pow2_k{k}_out"]
    P = z.shape[1]
    out = zeros(z.shape)
    lib.brownianBridgeGPU_constant_memory(P, k, d(dev(z)), d(out))
    got = host(out)
    assert np.mean(np.abs(got - ref)) / np.mean(np.abs(ref)) < 2e-7
    assert np.max(np.abs(got - ref)) < 2e-5


@pytest.mark.parametrize("k,F", [(3, 3), (4, 5)])
@pytest.mark.parametrize("ordering", [0, 1, 2])
def test_multi_bridge_reorder_matches_gold(cuda, lib, gold_bridge, k, F, ordering):
    """brownianBridgeMultiGPUReorder moves variate i to (dim(i), fac(i)) of
    BrownianBridgeMultiDim<float> (gold/Bridge_gold.h:334-404); followed by
    the power-of-two bridge over paths x factors vectors it reproduces the
    gold multi-factor bridge."""
    tag = f"multi_k{k}_F{F}_o{ordering}"
    z = gold_bridge[tag + "_in"]
    dims, facs = gold_bridge[tag + "_dims"], gold_bridge[tag + "_facs"]
    n, P = 1 << k, z.shape[1]
    out = zeros((n, P, F))
    lib.brownianBridgeMultiGPUReorder(d(dev(z)), d(out), k, F, P, ordering, ctypes.c_bool(False))
    expect = np.zeros((n, P, F), np.float32)
    for i in range(F * n):
        expect[dims[i], :, facs[i]] = z[i]
    assert np.array_equal(host(out), expect)
    bridged = zeros((n, P * F))
    lib.brownianBridgeGPU_constant_memory(P * F, k, d(out), d(bridged))
    got = host(bridged).reshape(n, P, F).transpose(2, 0, 1).reshape(F * n, P)
    ref = gold_bridge[tag + "_out"]
    assert np.mean(np.abs(got - ref)) / np.mean(np.abs(ref)) < 2e-7


# ------------------------------------------------- correlation, evolution ----
def _lmm(gold):
    z = gold["lmm_z_spf"]
    S, P, F = z.shape
    n = gold["lmm_tau"].size
    return z, S, P, F, n


def test_correlate_and_pc_evolution(cuda, lib, gold):
    z, S, P, F, n = _lmm(gold)
    alive0 = dev(np.zeros(S, np.int32))
    corr = zeros((S, n, P))
    lib.correlated_drift_paths_GPU(d(dev(z)), d(corr), d(dev(gold["lmm_A"])), d(alive0),
                                   d(dev(gold["lmm_fixed"])), n * F, F, n, P, S)
    assert np.max(np.abs(host(corr) - gold["lmm_corr"])) < 1e-6
    rates = zeros((S, n, P))
    lrates = zeros((S, n, P))
    e = zeros((F, P))
    lib.LMM_evolver_pc_gpu(d(dev(gold["lmm_f0"])), d(dev(np.log(gold["lmm_f0"] + gold["lmm_disp"]))),
                           d(dev(gold["lmm_tau"])), d(dev(gold["lmm_corr"])), d(dev(gold["lmm_A"])),
                           d(zeros(n)), d(dev(gold["lmm_disp"])), stdvec(np.zeros(S, np.int32)),
                           P, F, S, n, d(e), d(e), d(rates), d(lrates), ctypes.c_bool(False))
    err = rel_err(host(rates), gold["lmm_rates"])
    assert err.mean() < 2e-6 and err.max() < 2e-5


def test_euler_evolution(cuda, lib, gold):
    """LMM_evolver_euler_gpu against an FP64 restatement of the reference's
    Euler step kernels (LMM_evolver_gpu.cu:835-1010): log f += spot drift
    of the start rates + correlated increment, capped at log 10."""
    z, S, P, F, n = _lmm(gold)
    corr, A = gold["lmm_corr"].astype(np.float64), gold["lmm_A"].astype(np.float64)
    tau, disp = gold["lmm_tau"].astype(np.float64), gold["lmm_disp"].astype(np.float64)
    f = np.repeat(gold["lmm_f0"].astype(np.float64)[:, None], P, 1)
    lf = np.log(f + disp[:, None])
    alive = np.arange(S, dtype=np.int32)
    ref = np.zeros((S, n, P))
    for s in range(S):
        g = (f + disp[:, None]) * tau[:, None] / (1.0 + f * tau[:, None])
        e = np.zeros((F, P))
        for r in range(alive[s], n):
            e += A[s, r][:, None] * g[r]
            lf[r] = np.minimum(lf[r] + A[s, r] @ e + corr[s, r], np.log(10.0))
        f = np.exp(lf) - disp[:, None]
        ref[s] = f
    rates = zeros((S, n, P))
    lrates = zeros((S, n, P))
    e = zeros((F, P))
    lib.LMM_evolver_euler_gpu(d(dev(gold["lmm_f0"])), d(e), d(dev(gold["lmm_tau"])),
                              d(dev(gold["lmm_corr"])), d(dev(gold["lmm_A"])), d(e),
                              d(dev(gold["lmm_disp"])), stdvec(alive), P, F, S, n, d(e), d(rates),
                              d(lrates))
    got = host(rates)
    mask = np.zeros((S, n), bool)
    for s in range(S):
        mask[s, s:] = True
    assert np.max(rel_err(got, ref)[mask]) < 2e-5


def test_pc_all(cuda, lib, gold):
    """LMM_evolver_pc_all_gpu equals lmm_evolve_pc_all (no log-rate cap),
    in both variates layouts, with and without discounts."""
    from useful_code_b200._lib import call

    z, S, P, F, n = _lmm(gold)
    alive = np.arange(S, dtype=np.int32)
    zt = np.ascontiguousarray(z.transpose(0, 2, 1))
    args = (d(dev(gold["lmm_f0"])), d(zeros(n)), d(dev(gold["lmm_tau"])))
    for transposed, doDisc, zz in ((True, True, zt), (False, True, z), (True, False, z)):
        rates, lrates, disc = zeros((S, n, P)), zeros((S, n, P)), zeros((S, n + 1, P))
        e = zeros((F, P))
        lib.LMM_evolver_pc_all_gpu(*args, d(dev(zz)), d(dev(gold["lmm_A"])), d(zeros(n)),
                                   d(dev(gold["lmm_fixed"])), d(dev(gold["lmm_disp"])),
                                   d(dev(alive)), P, F, S, n, d(e), d(e), d(rates), d(lrates),
                                   d(disc), ctypes.c_bool(False), ctypes.c_bool(transposed),
                                   VP(None), 128, ctypes.c_bool(doDisc))
        r2 = zeros((S, n, P))
        call("lmm_evolve_pc_all", gold["lmm_f0"].ctypes.data_as(VP),
             gold["lmm_tau"].ctypes.data_as(VP), gold["lmm_disp"].ctypes.data_as(VP),
             d(dev(zz)), 1 if (transposed and doDisc) else 0, d(dev(gold["lmm_A"])),
             d(dev(gold["lmm_fixed"])), alive.ctypes.data_as(VP), P, F, S, n, 1e30, d(r2),
             d(zeros((S, n, P))), None, None)
        mask = np.zeros((S, n), bool)
        for s in range(S):
            mask[s, s:] = True
        assert np.array_equal(host(rates)[mask], host(r2)[mask])


# ------------------------------------------------------ curve quantities ----
def test_curve_routines(cuda, lib, gold):
    rates = gold["lmm_rates"]
    S, n, P = rates.shape
    alive = np.arange(S, dtype=np.int32)
    tau = dev(gold["lmm_tau"])
    disc = zeros((S, n + 1, P))
    lib.discount_ratios_computation_gpu(d(dev(rates)), d(tau), stdvec(alive), d(dev(alive)), P, S,
                                        n, d(disc), ctypes.c_bool(True))
    mask = np.zeros((S, n + 1), bool)
    for s in range(S):
        mask[s, s:] = True
    assert np.max(np.abs(host(disc) - gold["lmm_disc"])[mask]) < 1e-6
    ann = zeros((S, n, P))
    lib.coterminal_annuity_ratios_computation_gpu(d(dev(gold["lmm_disc"])), d(tau), stdvec(alive),
                                                  P, S, n, d(ann))
    sr = zeros((S, n, P))
    lib.coterminal_swap_rate_computation_gpu(d(dev(gold["lmm_disc"])), d(dev(gold["lmm_ann"])),
                                             stdvec(alive), P, S, n, d(sr))
    m2 = mask[:, :n]
    assert np.max(rel_err(host(ann), gold["lmm_ann"])[m2]) < 1e-6
    assert np.max(rel_err(host(sr), gold["lmm_sr"])[m2]) < 1e-6
    num = zeros((n, P))
    lib.spot_measure_numeraires_computation_gpu(d(dev(gold["lmm_disc"])), d(num), P, n)
    assert np.max(rel_err(host(num), gold["lmm_num"])) < 1e-6
    num2 = zeros((n, 2 * P))
    lib.spot_measure_numeraires_computation_offset_gpu(d(dev(gold["lmm_disc"])), d(num2), P, 2 * P,
                                                       P, n)
    assert np.array_equal(host(num2)[:, P:], host(num))
    # swap rate of rates [2, 7) at step 2, with the lmm_* entry point's result
    from useful_code_b200._lib import call

    out1, out2 = zeros(P), zeros(P)
    lib.swap_rate_computation_gpu(d(dev(gold["lmm_disc"])), d(tau), 2, 7, P, 2, 0, n, d(out1))
    call("lmm_swap_rate", d(dev(gold["lmm_disc"])), gold["lmm_tau"].ctypes.data_as(VP), 2, 7, P,
         2, 0, 3, n, d(out2), None)
    assert np.array_equal(host(out1), host(out2))


def test_extractions(cuda, lib, gold):
    rates = gold["lmm_rates"]
    S, n, P = rates.shape
    idx = np.arange(S, dtype=np.int32)
    sel = zeros((S, P))
    lib.forward_rate_extraction_gpu(d(dev(rates)), stdvec(idx), P, S, n, d(sel))
    assert np.array_equal(host(sel), np.stack([rates[s, s] for s in range(S)]))
    fwd, stp = np.array([3, 5, 7], np.int32), np.array([1, 4, 6], np.int32)
    sel2 = zeros((3, P))
    lib.forward_rate_extraction_selecting_step_gpu(d(dev(rates)), stdvec(fwd), stdvec(stp), P, n,
                                                   d(sel2))
    assert np.array_equal(host(sel2), np.stack([rates[s, f] for f, s in zip(fwd, stp)]))
    num = gold["lmm_num"]
    ex = np.array([2, 5, 8, 11], np.int32)
    some = zeros((4, 2 * P))
    lib.spot_measure_numeraires_extraction_gpu.restype = ctypes.c_double
    t = lib.spot_measure_numeraires_extraction_gpu(d(dev(num)), d(some), P, 2 * P, P, n, 4,
                                                   d(dev(ex)))
    assert t >= 0.0
    assert np.array_equal(host(some)[:, P:], num[ex])


# ------------------------------------------------------------ cash flows ----
def test_cash_flow_routines(cuda, lib, gold):
    r1 = gold["cf_rate1"]
    S, P = r1.shape
    f1, f2 = zeros((S, P)), zeros((S, P))
    null = d(zeros(1))
    lib.cashFlowGeneratorCallerSwap(d(f1), d(f2), d(dev(gold["cf_aux"])), P, S, d(dev(r1)), null,
                                    null, null, null)
    assert np.max(np.abs(host(f1) - gold["cf_flows1"])) < 1e-7
    assert np.max(np.abs(host(f2) - gold["cf_flows2"])) < 1e-7
    t1, t2 = zeros((S, P)), zeros((S, P))
    lib.cashFlowGeneratorCallerTARN(d(t1), d(t2), d(dev(gold["tarn_a_aux"])), P, S, d(dev(r1)),
                                    d(dev(r1)), null, null, null)
    assert np.max(np.abs(host(t1) - gold["tarn_a_flows1"])) < 1e-6
    assert np.max(np.abs(host(t2) - gold["tarn_a_flows2"])) < 1e-6
    dflows, summed = zeros((S, P)), zeros(P)
    lib.cashFlowDiscounting_gpu(d(dev(gold["cf_first_mid"])), d(dev(gold["cf_second_mid"])),
                                d(dev(gold["cf_theta_mid"])), d(dev(gold["lmm_disc"])),
                                d(dev(gold["cf_flows2"])), d(dev(gold["lmm_num"])), P, S,
                                ctypes.c_bool(True), ctypes.c_bool(False), d(dflows), d(summed))
    assert np.max(np.abs(host(dflows) - gold["cf_discounted"])) < 1e-6
    assert np.max(np.abs(host(summed) - gold["cf_summed"])) < 1e-5
    gen = np.arange(S, dtype=np.int32)
    pfl = zeros((S, P))
    lib.cashFlowDiscounting_partial_gpu(S, d(dev(gen)), d(dev(gold["cf_first"])),
                                        d(dev(gold["cf_second"])), d(dev(gold["cf_theta"])),
                                        d(dev(gold["cf_target"])), d(dev(gold["lmm_disc"])),
                                        d(dev(gold["cf_flows2"])), d(dev(gold["lmm_num"])), P, S,
                                        d(pfl))
    assert np.max(np.abs(host(pfl) - gold["cf_partial"])) < 1e-6
    E = gold["cf_ex_idx"].size
    agg = zeros((E, P))
    lib.AggregateFlows_gpu(d(agg), P, E, d(dev(gold["cf_partial"])), P, 0, S,
                           d(dev(gold["cf_step_to_ex"])), int(gold["cf_first_positive"]))
    assert np.max(np.abs(host(agg) - gold["cf_aggregated"])) < 1e-5


# ---------------------------------------------------- Longstaff–Schwartz ----
def test_basis_variables(cuda, lib, gold):
    E, _, P = gold["bv_raw"].shape
    r = [dev(gold[k]) for k in ("ex_r1", "ex_r2", "ex_r3")]
    null = d(zeros(1))
    for use_log, key in ((False, "bv_raw"), (True, "bv_log")):
        out = zeros((E, 3, P))
        lib.adjoinBasisVariablesCaller_gpu(ctypes.c_bool(use_log), null,
                                           d(dev(gold["bv_shifts"])), null, null, d(r[0]),
                                           d(r[1]), d(r[2]), P, P, 0, 12, E,
                                           d(dev(gold["cf_ex_idx"])), null, d(out))
        assert np.max(np.abs(host(out) - gold[key])) < 1e-6


def _basis_np(x, cross):
    V = x.shape[0]
    rows = [np.ones_like(x[0])]
    if not cross:
        for i in range(V):
            rows += [x[i], x[i] * x[i]]
        return np.stack(rows)
    rows += [x[i] for i in range(V)]
    if V == 1:
        rows.append(x[0] * x[0])
    elif V == 2:
        rows += [x[0] * x[0], x[0] * x[1], x[1] * x[1]]
    else:
        rows += [x[i] * x[(i + 1) % V] for i in range(V)] + [x[i] * x[i] for i in range(V)]
    return np.stack(rows)


@pytest.mark.parametrize("cross", [False, True])
@pytest.mark.parametrize("V", [1, 2, 3])
def test_ls_step_routines(cuda, lib, cxx, cross, V):
    """expandBasisFunctions_quadratic_gpu, continuation_net_value_evaluation_
    gpu, oneStepUpdateLS_multi_gpu and updateDeflationOfContinuationValues_
    gpu against NumPy restatements of the reference kernels (LS_gpu.h:92-232,
    LS_gpu.cu:57-99, 251-265, 312-402)."""
    rng = np.random.default_rng(V + 10 * cross)
    P, E, maxv, e = 1000, 4, 3, 2
    vars_ = rng.standard_normal((E, maxv, P)).astype(np.float32)
    phi_ref = _basis_np(vars_[e, :V], cross)
    K = phi_ref.shape[0]
    phi = zeros((K, P))
    cxx("expandBasisFunctions_quadratic_gpu")(P, d(dev(vars_)), e, maxv, V, ctypes.c_bool(cross),
                                              d(phi))
    assert np.array_equal(host(phi), phi_ref)
    w = rng.standard_normal(K).astype(np.float32) * 0.1
    exv = rng.uniform(0, 0.2, P).astype(np.float32)
    out = zeros(P)
    fn = cxx("continuation_net_value_evaluation_gpu")
    fn.restype = ctypes.c_double
    fn(P, e, d(phi), K, d(dev(w)), d(dev(exv)), F32(0.01), d(out))
    ref = np.float32(0.01) + (w[:, None].astype(np.float64) * phi_ref).sum(0) - exv
    assert np.max(np.abs(host(out) - ref)) < 1e-5
    # exercise update with a depth chain of 3 (row size 16)
    depth, row = 3, 16
    wts = (rng.standard_normal((E, depth, row)) * 0.05).astype(np.float32)
    lo = np.array([-0.02, -0.01, 0.0], np.float32)
    hi = np.array([0.02, 0.01, 0.0], np.float32)
    exall = rng.uniform(0, 0.1, (E, P)).astype(np.float32)
    cont0 = rng.uniform(0, 0.1, P).astype(np.float32)
    cont, est, exs = dev(cont0.copy()), zeros(P), zeros(P, np.int32)
    fn = cxx("oneStepUpdateLS_multi_gpu")
    fn.restype = ctypes.c_double
    fn(P, e, d(phi), K, row, depth, d(dev(wts)), d(dev(lo)), d(dev(hi)), d(cont), d(zeros(1)),
       d(dev(exall)), F32(0.0), d(est), d(exs))
    c_ref, x_ref = cont0.copy(), np.zeros(P, np.int32)
    for p in range(P):
        for k in range(depth):
            es = float((wts[e, k, :K].astype(np.float64) * phi_ref[:, p]).sum())
            net = es - float(exall[e, p])
            if k == depth - 1 or net < lo[k] or net > hi[k]:
                break
        x_ref[p] = 1 if net < 0 else -1
        if net < 0:
            c_ref[p] = exall[e, p]
    got_x = host(exs)
    assert np.mean(got_x == x_ref) > 0.995  # FP32 sums at the cut boundaries
    assert np.array_equal(host(cont)[got_x == x_ref], c_ref[got_x == x_ref])
    nums = rng.uniform(1.0, 1.5, (E, P)).astype(np.float32)
    vals = dev(cont0.copy())
    fn = cxx("updateDeflationOfContinuationValues_gpu")
    fn.restype = ctypes.c_double
    fn(d(vals), d(dev(nums)), P, 3, 1)
    np.testing.assert_allclose(host(vals), cont0 * (nums[3] / nums[1]), rtol=2e-7)


# ------------------------------------------------------------ reductions ----
def _pairwise8(x):
    x = x.reshape(-1, 8)
    a = (x[:, 0] + x[:, 1]) + (x[:, 2] + x[:, 3])
    b = (x[:, 4] + x[:, 5]) + (x[:, 6] + x[:, 7])
    return (a + b).astype(np.float32)


def test_partial_reductions(cuda, cxx):
    x = np.random.default_rng(4).standard_normal(8 ** 4).astype(np.float32)
    ws = zeros(x.size)
    fn = cxx("PartialReduce_using8s_gpu")
    fn.restype = VP
    ptr = fn(d(dev(x)), d(ws), x.size, 256, 1)
    lvl = x
    while lvl.size > 1:
        lvl = _pairwise8(lvl)
    off = (ptr - ws.data_ptr()) // 4
    assert 0 <= off < ws.numel()
    assert host(ws)[off] == lvl[0]
    x16 = np.random.default_rng(5).standard_normal(16 ** 3).astype(np.float32)
    ws16 = zeros(x16.size)
    fn16 = cxx("PartialReduce_using16s_gpu")
    fn16.restype = VP
    ptr16 = fn16(d(dev(x16)), d(ws16), x16.size, 256)
    lvl = x16
    while lvl.size > 1:
        h = lvl.reshape(-1, 16)
        lvl = (_pairwise8(h[:, :8].ravel()) + _pairwise8(h[:, 8:].ravel())).astype(np.float32)
    assert host(ws16)[(ptr16 - ws16.data_ptr()) // 4] == lvl[0]


@pytest.mark.parametrize("group", [8, 16])
@pytest.mark.parametrize("offset", [0, 1])
def test_partial_reduce_levels(cuda, group, offset):
    """lmm_partial_reduce on a ragged count (each level drops the remainder
    that does not fill a group) from a 16-byte aligned start and from one
    float further on (the 16-byte-load kernel and the one-value-per-load
    kernel; later levels start wherever the previous level ended): every
    level written to the workspace equals the reference's pairwise FP32
    sums bit for bit."""
    from useful_code_b200._lib import call

    n = 100_003
    x = np.random.default_rng(7 + group).standard_normal(n + offset).astype(np.float32)
    dx = dev(x)
    ws = zeros(n)
    result = VP()
    call("lmm_partial_reduce", VP(dx.data_ptr() + 4 * offset), d(ws), n, group, 1,
         ctypes.byref(result), None)
    levels, lvl = [], x[offset:]
    while lvl.size > 1 and lvl.size >= group:
        h = lvl[: (lvl.size // group) * group]
        if group == 8:
            lvl = _pairwise8(h)
        else:
            h = h.reshape(-1, 16)
            lvl = (_pairwise8(h[:, :8].ravel()) + _pairwise8(h[:, 8:].ravel())).astype(np.float32)
        levels.append(lvl)
    got = host(ws)
    pos = 0
    for ref in levels:
        np.testing.assert_array_equal(got[pos:pos + ref.size], ref)
        pos += ref.size
    assert (result.value - ws.data_ptr()) // 4 == pos - levels[-1].size


@pytest.mark.parametrize("rows,cols,paths", [(10, 10, 4096), (7, 3, 10000), (16, 1, 65536)])
def test_outer_products(cuda, cxx, rows, cols, paths):
    """reduceOuterProduct_gpu (general and symmetric) and
    reduceOuterProductSymmetric_gpu against an FP64 NumPy product, 2e-6
    relative to the largest entry."""
    rng = np.random.default_rng(rows * cols)
    a = rng.standard_normal((rows, paths)).astype(np.float32)
    b = rng.standard_normal((cols, paths)).astype(np.float32)
    threads = 128
    ws = zeros(threads * max(rows, cols) ** 2)
    out = zeros((rows, cols))
    cxx("reduceOuterProduct_gpu")(paths, rows, cols, ctypes.c_bool(False), threads, threads,
                                  d(dev(a)), d(dev(b)), d(out), d(ws))
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    assert np.max(np.abs(host(out) - ref)) < 2e-6 * np.max(np.abs(ref))
    sym = zeros((rows, rows))
    cxx("reduceOuterProductSymmetric_gpu")(paths, rows, threads, threads, d(dev(a)), d(sym),
                                           d(ws))
    refs = a.astype(np.float64) @ a.astype(np.float64).T
    assert np.max(np.abs(host(sym) - refs)) < 2e-6 * np.max(np.abs(refs))
    sym2 = zeros((rows, rows))
    cxx("reduceOuterProduct_gpu")(paths, rows, cols, ctypes.c_bool(True), threads, threads,
                                  d(dev(a)), d(dev(b)), d(sym2), d(ws))
    assert np.array_equal(host(sym2), host(sym))
