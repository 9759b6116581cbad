#!/usr/bin/env python
"""Bermudan LMM Monte Carlo throughput on B200.

One step = one two-pass Longstaff–Schwartz pricing of the precision-form
Bermudan payer swaption (config c3: 80 quarterly forwards, 10 factors, 80
steps, 2^20 regression paths + 2^20 independent pricing paths, FP32 path
arithmetic, FP64 regression solve and reductions): Sobol -> scramble ->
inverse normal -> bridge -> PC evolution -> basis/exercise values -> LS
regression -> second pass with the frozen rule -> price.  ``value`` is
simulated paths (regression + pricing) per second, device-timed with all
inputs resident in HBM, for the fused form; the plain FP32 staged form is
timed beside it.  Inputs (the variates buffer, 3.4 GB, and the LS inputs,
2 GB per pass) are larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Bermudan LMM paths/s: fused mixed-prec vs plain FP32; Greeks/price time ratio"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c3")
    ap.add_argument("--staged-steps", type=int, default=3,
                    help="timed steps of the plain FP32 staged form (after one warm-up step)")
    ap.add_argument("--staged-batch", type=int, default=1 << 19,
                    help="paths per batch of the staged form (its workspace holds full "
                         "[step][rate][path] tensors: about 84 GB at 2^19 for c3)")
    ap.add_argument("--cpu-sample", type=int, default=1 << 15,
                    help="paths per pass of the cpu_baseline leg")
    ap.add_argument("--ref-sample", type=int, default=1 << 15,
                    help="paths per pass of each --impl reference step (the cpu_baseline "
                         "leg's sample, so the two report the same workload)")
    ap.add_argument("--paths", type=int, default=None,
                    help="override the pricing paths (small cases for profiling)")
    ap.add_argument("--reg-paths", type=int, default=None,
                    help="override the regression paths (small cases for profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--greeks-steps", type=int, default=2,
                    help="timed lmm_greeks calls on the pricing paths (0 skips)")
    ap.add_argument("--checkpoint-every", type=int, default=8)
    ap.add_argument("--nested-depth", type=int, default=4,
                    help="regression depth of the nested-regression timing (0 skips)")
    ap.add_argument("--ab-outer", type=int, default=512,
                    help="outer paths of the Andersen-Broadie timing (0 skips)")
    ap.add_argument("--ab-inner", type=int, default=512,
                    help="inner paths per (outer path, exercise date)")
    ap.add_argument("--segment-steps", type=int, default=0,
                    help="steps per launch of the segmented second pass (0: library default; "
                         ">= rates: one launch)")
    ap.add_argument("--evolve", default="fused", choices=["tensor", "fused"],
                    help="evolution kernel: tensor-core contractions or CUDA cores")
    ap.add_argument("--stage-paths", type=int, default=1 << 19,
                    help="paths of the staged cash-flow, discounting and reduction timings "
                         "(0 skips; one GPU only)")
    return ap.parse_args()


# ------------------------------------------------- staged stage timings -----
def hbm_peak() -> tuple[float, str]:
    """Measured copy bandwidth (GB/s) of this pool's B200s, else the fallback."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        v = json.loads(f.read_text()).get("hbm_gbs")
        if v:
            return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def stage_timings(P: int, n: int, call, LIB, stream_handle, dp) -> dict:
    """Device time of each staged cash-flow, discounting, aggregation, basis,
    exercise-value, numeraire and reduction entry point on c3-shaped
    synthetic inputs (n steps = n exercise dates = n rates, P paths), with
    its algorithmic bytes (each input element read once, each output written
    once) and the fraction of the HBM copy bandwidth."""
    import numpy as np
    import torch

    S = E = n
    g = torch.Generator(device="cuda").manual_seed(11)

    def unif(shape, lo, hi):
        return torch.rand(shape, generator=g, device="cuda") * (hi - lo) + lo

    rate1, rate2, rate3 = unif((S, P), 0.02, 0.08), unif((S, P), 0.02, 0.08), unif((S, P), 1, 5)
    flows = unif((S, P), -0.01, 0.01)
    num = unif((S, P), 1.0, 2.0)
    disc = unif((S, n + 1, P), 0.5, 1.0)
    f1, f2, out = (torch.empty((S, P), device="cuda") for _ in range(3))
    summed = torch.empty(P, device="cuda")
    agg = torch.zeros((E, P), device="cuda")
    bv = torch.empty((E, 3, P), device="cuda")
    nums = torch.empty((n, P), device="cuda")
    work = torch.empty(S * P // 7 + 64, device="cuda")
    part = torch.empty(int(LIB.lmm_reduce_workspace_doubles()), dtype=torch.float64,
                       device="cuda")
    res = torch.empty(1, dtype=torch.float64, device="cuda")

    keep = []  # host tables stay alive during the timed calls

    def tab(a, dt):
        arr = np.ascontiguousarray(a, dtype=dt)
        keep.append(arr)
        return arr.ctypes.data_as(ctypes.c_void_p)

    steps_i = np.arange(S)
    first = tab(np.minimum(steps_i + 1, n), np.int32)
    second = tab(np.minimum(steps_i + 2, n), np.int32)
    theta = tab(np.full(S, 0.5), np.float32)
    gen = tab(steps_i, np.int32)
    target = tab(np.maximum(steps_i - 1, 0), np.int32)
    prec = tab(steps_i, np.int32)
    swap_aux = tab(np.concatenate([[0.05, 1.0], np.full(2 * S, 0.25)]), np.float32)
    tarn_aux = tab(np.concatenate([[0.3, 0.08, 1.0], np.full(2 * S, 0.25)]), np.float32)
    shifts = tab(np.array([0.0, 0.0, 1.0]), np.float32)
    st = stream_handle()
    result_ptr = ctypes.c_void_p()  # the level that holds the partial sums
    N = S * P
    B = 4  # bytes per element
    stages = {
        "cashflows_swap (flows_kernel)": (
            lambda: call("lmm_cashflows_swap", dp(f1), dp(f2), swap_aux, P, S, dp(rate1), st),
            3 * S * P * B),
        "cashflows_tarn (tarn_kernel)": (
            lambda: call("lmm_cashflows_tarn", dp(f1), dp(f2), tarn_aux, P, S, dp(rate1),
                         dp(rate2), st), 4 * S * P * B),
        "cashflow_discounting (discounting_kernel)": (
            lambda: call("lmm_cashflow_discounting", first, second, theta, dp(disc), dp(flows),
                         dp(num), P, S, dp(out), dp(summed), st), (6 * S * P + P) * B),
        "cashflow_discounting_partial": (
            lambda: call("lmm_cashflow_discounting_partial", S, gen, first, second, theta,
                         target, dp(disc), dp(flows), dp(num), P, S, dp(out), st),
            7 * S * P * B),
        "aggregate_flows (aggregate_kernel)": (
            lambda: call("lmm_aggregate_flows", dp(agg), P, E, dp(flows), P, 0, S, prec, 0, st),
            (S + 2 * E) * P * B),
        "basis_variables, log (basis_variables_kernel)": (
            lambda: call("lmm_basis_variables", 1, shifts, dp(rate1), dp(rate2), dp(rate3), P, P,
                         0, E, dp(bv), st), 6 * E * P * B),
        "exercise_values_payer_swaption": (
            lambda: call("lmm_exercise_values_payer_swaption", 0.05, dp(rate1), dp(rate3), P, P,
                         0, E, dp(out), st), 3 * E * P * B),
        "spot_numeraires (numeraires_kernel)": (
            lambda: call("lmm_spot_numeraires", dp(disc), P, P, 0, n, dp(nums), st),
            (3 * n - 2) * P * B),
        "reduce_mean_ratio (reduce_partial/final)": (
            lambda: call("lmm_reduce_mean_ratio", dp(flows), dp(num), N, dp(part), dp(res), st),
            2 * N * B),
        "partial_reduce, groups of 8 (partial_reduce_kernel)": (
            lambda: call("lmm_partial_reduce", dp(flows), dp(work), N, 8, 1,
                         ctypes.addressof(result_ptr), st), (N * 9 // 7) * B),
    }
    peak, source = hbm_peak()
    result = {"paths": P, "steps": S, "peak_gbs": peak, "peak_source": source, "kernels": {}}
    for name, (fn, nbytes) in stages.items():
        fn()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(3):
            fn()
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / 3
        gbs = nbytes / (ms / 1e3) / 1e9
        result["kernels"][name] = {"ms": ms, "bytes": nbytes, "gbs": gbs, "frac": gbs / peak}
    del disc
    return result


# --------------------------------------------------------------- clocks -----
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[0]) for r in self.rows if num(r[0])]
        mx = [num(r[1]) for r in self.rows if num(r[1])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ------------------------------------------------------------- CPU legs -----
REF_SO = ROOT / "oracle" / "_ref" / "libkooref.so"


def _configs():
    """The benchmark configurations (useful_code_b200/configs.py, numpy only),
    loaded by file path: the reference arm never imports the package, whose
    import loads the CUDA library."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_lmm_configs",
                                                  ROOT / "useful_code_b200" / "configs.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up by name
    spec.loader.exec_module(mod)
    return mod


def reference_inputs(cfg, ref, scramble_dims: int) -> dict:
    """The workload's model inputs from the reference's own gold set-up code:
    pseudo-roots by ABCDLBetaPseudoRoots (gold/volstructs_gold.cpp:311-360)
    or FlatVolPseudoRootsOfCovariances (:177-255), scrambler words by
    MersenneTwisterUniformRng::nextInt32 (gold/Mersenne_gold.h:42-60), fixed
    drifts -1/2 |A_s[r]|^2 in FP32 as the reference's example forms them
    (kooexample/bermudanIRDPricer.cu:403-417)."""
    import numpy as np

    D = ctypes.c_double
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    n, F = cfg.n, cfg.F
    rate_times = cfg.tau * (np.arange(n + 1) + 1.0)
    resets = np.ascontiguousarray(rate_times[:n])
    A64 = np.zeros((n, n, F))
    if cfg.vol == "abcd":
        a, b, c, d = cfg.abcd
        ref.kref_abcd_pseudo_roots(D(a), D(b), D(c), D(d), vp(resets), n, vp(resets), n,
                                   vp(np.ones(n)), F, D(cfg.L), D(cfg.beta), vp(A64))
    else:
        rt = np.ascontiguousarray(rate_times)  # n + 1 rate times: n rates
        ref.kref_flat_pseudo_roots(vp(rt), n + 1, vp(resets), n, vp(np.full(n, cfg.sigma)), F,
                                   D(cfg.L), D(cfg.beta), vp(A64))
    A = np.ascontiguousarray(A64.astype(np.float32))
    fixed = np.ascontiguousarray((np.float32(-0.5) * (A * A).sum(-1, dtype=np.float32)))
    scr = np.zeros(scramble_dims, np.uint32)
    ref.kref_mt19937(ctypes.c_ulong(cfg.scramble_seed), scramble_dims, vp(scr))
    return {"taus": np.full(n, cfg.tau, np.float32), "disp": np.full(n, cfg.disp, np.float32),
            "f0": np.ascontiguousarray(cfg.f0, np.float32), "A": A, "fixed": fixed, "scr": scr,
            "P0": 1.0 / (1.0 + float(cfg.f0[0]) * float(rate_times[0]))}


def cpu_reference(cfg_name: str, sample: int, threads: int) -> dict:
    """Time the reference's own gold CPU code (oracle/_ref/libkooref.so,
    compiled from the reference sources) on `sample` regression + `sample`
    pricing paths of the workload: LMMEvolutionRoutineGold, the curve
    stages, basis and exercise values, the gold LS regression and the gold
    second pass, chunks of 256 paths spread over `threads` threads.  The
    model inputs come from the reference's gold set-up routines too, so
    nothing of this repository's library is loaded.  Falls back to the CPU
    restatement when the gold library is absent or the product is not the
    swaption with the reference's cross basis."""
    import numpy as np

    cfg = _configs().make_config(cfg_name)
    if not REF_SO.exists() or cfg.product != "swaption" or cfg.basis != "cross":
        return cpu_sample(cfg_name, sample, threads)
    n, F = cfg.n, cfg.F
    p2 = 0
    while (1 << p2) < n:
        p2 += 1
    ref = ctypes.CDLL(str(REF_SO))
    ref.kref_bermudan_swaption.restype = ctypes.c_double
    mkt = reference_inputs(cfg, ref, (1 << p2) * F)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    ins = ctypes.c_double()
    sec = ctypes.c_double()
    price = ref.kref_bermudan_swaption(
        n, F, vp(mkt["taus"]), vp(mkt["disp"]), vp(mkt["f0"]), vp(mkt["A"]), vp(mkt["fixed"]),
        vp(mkt["scr"]), ctypes.c_float(cfg.strike), sample, sample, 0, sample, threads, 256,
        int(cfg.normalise), ctypes.byref(ins), ctypes.byref(sec))
    return {"value": 2 * sample / sec.value, "unit": "paths/s", "cores": threads,
            "kind": "reference",
            "sample": f"{cfg_name}: {sample} regression + {sample} pricing paths through the "
                      f"reference's gold routines (ABCDLBetaPseudoRoots, MersenneTwister "
                      f"scramblers, LMMEvolutionRoutineGold ... "
                      f"SecondPassPriceLSAMultiUsingAggregatedFlows_gold), {threads} threads",
            "seconds": sec.value, "price": price * mkt["P0"]}


def cpu_sample(cfg_name: str, sample: int, threads: int) -> dict:
    """Time the CPU restatement of the path (first pass, regression, second
    pass) on `sample` regression + `sample` pricing paths."""
    import numpy as np

    from useful_code_b200 import market as mk

    so = ROOT / "oracle" / "liblmm_oracle.so"
    if not so.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True,
                       capture_output=True)
    orc = ctypes.CDLL(str(so))
    orc.orc_ls_regress_f.restype = ctypes.c_double
    cfg = mk.make_config(cfg_name)
    mkt = mk.build_market(cfg)
    n, F, E = cfg.n, cfg.F, len(mkt.ex_steps)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data) if a is not None else None  # noqa: E731
    sd = np.array([cfg.strike, cfg.pay_receive, cfg.cap_strike, cfg.cutoff], np.float64)
    lf0 = np.log(mkt.f0 + mkt.disp).astype(np.float32)
    ex_steps = np.ascontiguousarray(mkt.ex_steps.astype(np.int32))
    E1 = max(E, 1)
    v = np.zeros((E1, 3, sample), np.float32)
    ex = np.zeros((E1, sample), np.float32)
    cf = np.zeros((E1, sample), np.float32)
    num = np.zeros((E1, sample), np.float32)
    pay = np.zeros(sample)
    beta = np.zeros((E1, 16))
    means = np.zeros((E1, 3))
    sds = np.ones((E1, 3))
    prod = mk.PRODUCTS[cfg.product]

    def run(offset, mode):
        si = np.array([n, F, sample, offset, mkt.scramble_dims, prod, E, int(cfg.normalise),
                       threads], np.int32)
        orc.orc_pipeline_f(vp(si), vp(sd), vp(mkt.directions), vp(mkt.scramblers), vp(mkt.A),
                           vp(mkt.fixed), vp(mkt.taus), vp(mkt.disp), vp(mkt.f0), vp(lf0),
                           vp(ex_steps), vp(mkt.nvars), vp(mkt.mono), vp(mkt.nbasis),
                           ctypes.c_int(mode), vp(beta), vp(means), vp(sds), vp(v), vp(ex),
                           vp(cf), vp(num), vp(pay))

    t0 = time.perf_counter()
    if cfg.product != "european":
        run(0, 0)
        orc.orc_ls_regress_f(E, sample, vp(v), vp(mkt.nvars), vp(mkt.mono), vp(mkt.nbasis),
                             vp(cf), vp(ex), vp(num), int(cfg.normalise), vp(beta), vp(means),
                             vp(sds), None)
    run(sample, 1)
    dt = time.perf_counter() - t0
    paths = 2 * sample if cfg.product != "european" else sample
    return {"value": paths / dt, "unit": "paths/s", "cores": threads, "kind": "port",
            "sample": f"{cfg_name}: {sample} regression + {sample} pricing paths, full path "
                      f"(oracle/lmm_oracle.cpp restatement, FP32)", "seconds": dt,
            "price": float(pay.mean()) * mkt.initial_numeraire}


def run_reference(args) -> int:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference(args.config, args.ref_sample, threads)
        if i >= args.warmup:
            vals.append(r)
    value = statistics.median(x["value"] for x in vals)
    ms = 1e3 * statistics.median(x["seconds"] for x in vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "paths/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args.config)},
            "cpu_baseline": {k: vals[-1][k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    line["cpu_baseline"]["value"] = value
    print(json.dumps(line))
    return 0


def workload_name(cfg: str) -> str:
    return {"c3": "bermudan-swaption-80q-10f-2^20reg+2^20price",
            "c2": "bermudan-swaption-40s-5f-65536reg+262144price",
            "c1": "european-caplets+swap-20s-3f-16384",
            "c5": "cancellable-swap-120q-15f-2^21reg+2^21price"}.get(cfg, cfg)


# ------------------------------------------------------------- GPU arm -----
def run_b200(args) -> int:
    import numpy as np
    import torch
    import torch.distributed as dist

    from useful_code_b200 import market as mk
    from useful_code_b200._lib import LIB, call
    from useful_code_b200.pricer import Pipeline, dp, rule_struct, stream_handle
    from useful_code_b200.sharded import regress_sharded

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    over = {}
    if args.paths:
        over["paths"] = args.paths
    if args.reg_paths:
        over["reg_paths"] = args.reg_paths
    cfg = mk.make_config(args.config, **over)
    mkt = mk.build_market(cfg)
    pipe = Pipeline(mkt)
    Preg, P = cfg.reg_paths, cfg.paths
    n, F, E = cfg.n, cfg.F, pipe.E
    euro = cfg.product == "european"
    # disjoint Sobol ranges per rank (weak scaling): [reg | price] per rank
    base = rank * (Preg + P)
    off_reg, off_price = base, base + Preg
    # regression and pricing variates in separate buffers: the pricing
    # variates are generated on a low-priority side stream while the first
    # pass and the regression run on the high-priority main stream
    var = torch.empty(n * F * Preg, device="cuda") if not euro else None
    var2 = torch.empty(n * F * P, device="cuda")
    ls = pipe.alloc_inputs(Preg) if not euro else None
    pay = torch.empty(P, device="cuda")
    m_addr = ctypes.addressof(pipe.model)
    p_addr = ctypes.addressof(pipe.product)
    tensor = args.evolve == "tensor"
    tc_ws = torch.empty(max(1, LIB.lmm_tensor_evolve_workspace_bytes(m_addr)), dtype=torch.uint8,
                        device="cuda")

    seg_ws = torch.empty(max(1, LIB.lmm_fused_price_workspace_bytes(m_addr, p_addr, P)),
                         dtype=torch.uint8, device="cuda")

    def evolve(z, paths, beta, means, sds, total, vars_, ex_, cf_, num_, payoff, s):
        if tensor:
            call("lmm_tensor_evolve", m_addr, p_addr, paths, dp(z), beta, means, sds, total, 0,
                 vars_, ex_, cf_, num_, payoff, dp(tc_ws), tc_ws.numel(), s)
        else:
            call("lmm_fused_evolve", m_addr, p_addr, paths, dp(z), beta, means, sds, total, 0,
                 vars_, ex_, cf_, num_, payoff, s)

    def price_pass(paths, rule, payoff, s):
        """Second pass: the segmented rule pass (exercised paths dropped
        between segments) on the CUDA cores, the one-launch tensor form."""
        if tensor:
            evolve(var2, paths, dp(rule.beta) if rule else None,
                   dp(rule.means) if rule else None, dp(rule.sds) if rule else None, paths, None,
                   None, None, None, payoff, s)
            return
        rs = rule_struct(rule) if rule else None
        call("lmm_fused_price", m_addr, p_addr, paths, dp(var2),
             ctypes.byref(rs) if rs else None, args.segment_steps, dp(seg_ws), seg_ws.numel(),
             payoff, s)
    ev = {k: [] for k in ("first", "second", "variates")}

    lo_prio, hi_prio = torch.cuda.Stream.priority_range()
    main = torch.cuda.Stream(priority=hi_prio)
    side = torch.cuda.Stream(priority=lo_prio)

    def step(record: bool):
        """One pricing step on the current (main) stream; the pricing
        variates run on the side stream, joined before the second pass."""
        s = stream_handle()
        rule = None
        if not euro:
            side.wait_stream(torch.cuda.current_stream())
            call("lmm_fused_variates", m_addr, P, off_price, dp(var2),
                 ctypes.c_void_p(side.cuda_stream))
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record()
            call("lmm_fused_variates", m_addr, Preg, off_reg, dp(var), s)
            ev1.record()
            if record:
                ev["variates"].append((ev0, ev1))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            evolve(var, Preg, None, None, None, Preg, dp(ls.vars), dp(ls.ex), dp(ls.cf),
                   dp(ls.num), None, s)
            e1.record()
            if record:
                ev["first"].append((e0, e1))
            # one rule for all ranks: per-date sums all-reduced (NCCL)
            rule = (regress_sharded(pipe, ls, world * Preg, dist.all_reduce) if world > 1
                    else pipe.regress(ls))
            torch.cuda.current_stream().wait_stream(side)
        else:
            call("lmm_fused_variates", m_addr, P, off_price, dp(var2), s)
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record()
        price_pass(P, rule, dp(pay), s)
        e3.record()
        if record:
            ev["second"].append((e2, e3))
        return pipe.mean(pay)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clk = ClockSampler(local).__enter__()  # sampling spans warm-up and timing
    with torch.cuda.stream(main):
        for _ in range(args.warmup):
            step(False)
    torch.cuda.synchronize()
    barrier()
    launches0 = LIB.lmm_launch_count()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    n_before = len(clk.rows)
    torch.cuda.synchronize()
    with torch.cuda.stream(main):
        start.record()
        for _ in range(args.steps):
            price_t = step(True)
        end.record()
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    if len(clk.rows) - n_before >= 3:
        clk.rows = clk.rows[n_before:]  # keep the samples of the timed region
    barrier()
    launches = LIB.lmm_launch_count() - launches0
    ms = max_over_ranks(start.elapsed_time(end) / args.steps)
    price = float(price_t.item()) * mkt.initial_numeraire
    if world > 1:
        t = torch.tensor([price], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        price = float(t.item()) / world
    paths_per_step = (0 if euro else Preg) + P
    value = world * paths_per_step / (ms / 1e3)

    # fused evolution kernel (dominant): average launch time of each pass
    def avg(pairs):
        return statistics.mean(a.elapsed_time(b) for a, b in pairs) if pairs else None

    t_first, t_second = avg(ev["first"]), avg(ev["second"])
    t_var = avg(ev["variates"])  # the first pass's variates (Preg paths)
    R = n * (n + 1) // 2
    flops_path = R * (10 * F + 12)
    clocks = clk.summary()
    sm_mhz = clocks["sm_mhz"] or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    dom_t = t_first if t_first is not None else t_second
    dom_paths = Preg if t_first is not None else P
    achieved = dom_paths * flops_path / (dom_t / 1e3) / 1e12
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        per_path = json.loads(tf.read_text()).get(f"fused_evolve_{args.config}_bytes_per_path")
        if per_path is not None and t_first is not None:
            traffic = per_path * Preg
    kname = "tc_evolve_kernel" if tensor else "fused_evolve_kernel"
    roofline = {"bound": "fp32", "kernel": f"{kname} (first pass)",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": traffic,
                "peak_source": "nominal FP32 FMA rate, 148 SMs x 128 lanes x 2 at the median "
                               "sampled SM clock (no measured FP32 peak in MEASURED_PEAKS.json)",
                "flops_per_launch": dom_paths * flops_path,
                "ms_per_launch": dom_t, "second_pass_ms": t_second}

    # ---- plain FP32 staged form of the same step -------------------------
    staged = None
    if args.staged_steps > 0:
        # its own LS-input and payoff buffers (the fused step's stay as they
        # are for the sections below); the warm-up step allocates the batch
        # workspace, so the timed steps allocate nothing
        ls_st = pipe.alloc_inputs(Preg) if not euro else None
        pay_st = torch.empty(P, device="cuda")

        def staged_step():
            rule_st = None
            if not euro:
                pipe.first_pass(Preg, off_reg, "staged", batch=args.staged_batch, out=ls_st)
                rule_st = pipe.regress(ls_st)
            pipe.second_pass(P, off_price, rule_st, "staged", batch=args.staged_batch,
                             out=pay_st)
            return pipe.mean(pay_st)

        with torch.cuda.stream(main):
            staged_step()
        torch.cuda.synchronize()
        barrier()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(main):
            s0.record()
            for _ in range(args.staged_steps):
                price_st = staged_step()
            s1.record()
        torch.cuda.synchronize()
        sms = max_over_ranks(s0.elapsed_time(s1) / args.staged_steps)
        staged = {"ms_per_step": sms, "value": world * paths_per_step / (sms / 1e3),
                  "steps": args.staged_steps, "warmup": 1, "batch_paths": args.staged_batch,
                  "speedup_fused_vs_staged": sms / ms,
                  "price": float(price_st.item()) * mkt.initial_numeraire}
        del ls_st, pay_st
        pipe._ws.clear()
        torch.cuda.empty_cache()

    # ---- pathwise adjoint Greeks on the pricing paths ------------------------
    greeks = None
    if args.greeks_steps > 0:
        rule = None if euro else pipe.regress(ls)
        gbytes = LIB.lmm_greeks_workspace_bytes(m_addr, p_addr, P, args.checkpoint_every)
        gws = torch.empty(gbytes, dtype=torch.uint8, device="cuda")
        g_price = torch.zeros(1, dtype=torch.float64, device="cuda")
        g_delta = torch.zeros(n, dtype=torch.float64, device="cuda")
        g_abar = torch.zeros(n * n * F, dtype=torch.float64, device="cuda")
        g_vega = torch.zeros(n, dtype=torch.float64, device="cuda")
        g_st = torch.zeros(1, dtype=torch.int32, device="cuda")

        def greeks_call():
            call("lmm_greeks", m_addr, p_addr, P, off_price, dp(rule.beta) if rule else None,
                 dp(rule.means) if rule else None, dp(rule.sds) if rule else None,
                 float(mkt.rate_times[0]), args.checkpoint_every, dp(gws), gws.numel(),
                 dp(g_price), dp(g_delta), dp(g_abar), dp(g_vega), None, dp(g_st),
                 stream_handle())

        greeks_call()  # warm-up
        torch.cuda.synchronize()
        barrier()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        gl0 = LIB.lmm_launch_count()
        g0.record()
        for _ in range(args.greeks_steps):
            greeks_call()
        g1.record()
        torch.cuda.synchronize()
        gms = max_over_ranks(g0.elapsed_time(g1) / args.greeks_steps)
        one_pass = (t_second or 0.0)
        # the frozen-rule pricing pass as a caller runs it on fresh paths:
        # its variates (timed on the first pass, scaled to P paths) + the pass
        with_var = one_pass + (t_var * P / Preg if t_var else 0.0)
        greeks = {"ms": gms, "paths": P, "checkpoint_every": args.checkpoint_every,
                  "price": float(g_price.item()), "status": int(g_st.item()),
                  "launches_per_call": (LIB.lmm_launch_count() - gl0) // args.greeks_steps,
                  "ratio_to_pricing_step": gms / ms,
                  "ratio_to_second_pass_kernel": gms / one_pass if one_pass else None,
                  "ratio_to_second_pass_with_variates": gms / with_var if with_var else None,
                  "outputs": "price, delta[rates], dV/dA[steps][rates][factors], "
                             "vega per rate (row scaling)",
                  "workspace_gb": gbytes / 1e9}
        del gws
        torch.cuda.empty_cache()

    # ---- nested regressions (depth > 1) on the regression paths --------------
    nested = None
    if args.nested_depth > 1 and not euro and world == 1:
        from useful_code_b200.pricer import Selector

        sel = Selector.production(args.nested_depth)

        def timed(fn, reps=3):
            fn()
            torch.cuda.synchronize()
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            l0 = LIB.lmm_launch_count()
            t0.record()
            for _ in range(reps):
                out = fn()
            t1.record()
            torch.cuda.synchronize()
            return out, t0.elapsed_time(t1) / reps, (LIB.lmm_launch_count() - l0) // reps

        plain, plain_ms, _ = timed(lambda: pipe.regress(ls))
        rule_n, nest_ms, nest_launches = timed(lambda: pipe.regress_nested(ls, sel))
        # the same regression replayed from a CUDA graph (no host launch work)
        graph_n, _ = pipe.regress_nested_graph(ls, sel)
        _, graph_ms, _ = timed(lambda: graph_n.replay())
        del graph_n
        pay_n, pass_ms, _ = timed(lambda: pipe.second_pass(P, off_price, rule_n, "fused"))
        pay_1 = pipe.second_pass(P, off_price, plain, "fused")
        npaths = rule_n.npaths.cpu().numpy()
        nested = {"depth": args.nested_depth,
                  "selector": {"lower_frac": sel.lower_frac, "upper_frac": sel.upper_frac,
                               "sds": sel.sds, "multiplier": sel.multiplier,
                               "min_paths": sel.min_paths},
                  "regression_paths": Preg, "regress_ms": nest_ms,
                  "regress_graph_ms": graph_ms,
                  "depth1_regress_ms": plain_ms, "launches_per_regression": nest_launches,
                  "second_pass_ms": pass_ms,
                  "price": float(pipe.mean(pay_n).item()) * mkt.initial_numeraire,
                  "price_depth1": float(pipe.mean(pay_1).item()) * mkt.initial_numeraire,
                  "insample": float(rule_n.price.item()) * mkt.initial_numeraire,
                  "dates_nested": int((npaths[:, 1] > 0).sum()),
                  "mean_paths_per_depth": [float(x) for x in npaths.mean(0)],
                  "status": int(rule_n.status.item())}
        del rule_n, pay_n, pay_1
        torch.cuda.empty_cache()

    # ---- Andersen-Broadie upper bound of the depth-1 rule ---------------------
    ab = None
    if args.ab_outer > 0 and cfg.product == "swaption" and world == 1:
        rule1 = pipe.regress(ls)
        K, I = args.ab_outer, args.ab_inner
        pipe.andersen_broadie(rule1, K, off_price + P, I)  # warm-up
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        al0 = LIB.lmm_launch_count()
        a0.record()
        r_ab = pipe.andersen_broadie(rule1, K, off_price + P, I)
        a1.record()
        torch.cuda.synchronize()
        ab_ms = a0.elapsed_time(a1)
        ex_steps = [int(x) for x in mkt.ex_steps]
        # inner rate-steps: from each date but the last, steps s0..n-1 with
        # rates s..n-1 each
        rate_steps = sum(sum(n - t for t in range(sx + 1, n)) for sx in ex_steps[:-1])
        flops = float(rate_steps) * (10 * F + 12) * K * I
        inner_paths = (len(ex_steps) - 1) * K * I
        scale = mkt.initial_numeraire
        ab = {"outer_paths": K, "inner_paths": I, "ms": ab_ms,
              "launches": LIB.lmm_launch_count() - al0,
              "inner_paths_total": inner_paths,
              "inner_paths_per_s": inner_paths / (ab_ms / 1e3),
              "inner_fp32_tflops": flops / (ab_ms / 1e3) / 1e12,
              "lower": r_ab.lower * scale, "lower_se": r_ab.lower_se * scale,
              "gap": r_ab.gap * scale, "gap_se": r_ab.gap_se * scale,
              "upper": r_ab.upper * scale, "rule": "depth 1"}
        del r_ab
        torch.cuda.empty_cache()

    # ---- the staged cash-flow, discounting and reduction stages ---------------
    stages = None
    if args.stage_paths > 0 and world == 1:
        stages = stage_timings(args.stage_paths, n, call, LIB, stream_handle, dp)
        torch.cuda.empty_cache()

    # ---- end to end through the public API with host buffers ---------------
    host_in = {"A": mkt.A, "fixed": mkt.fixed, "dirs": mkt.directions.view(np.int32),
               "scr": mkt.scramblers.view(np.int32)}
    pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host_in.items()}
    targets = {"A": pipe.A, "fixed": pipe.fixed, "dirs": pipe.dirs, "scr": pipe.scr}
    out_host = torch.empty(1, dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pinned.values())
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        barrier()
        e2e0 = torch.cuda.Event(enable_timing=True)
        e2e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(main):
            e2e0.record()
            for _ in range(args.steps):
                for k in pinned:
                    targets[k].copy_(pinned[k], non_blocking=True)
                res = step(False)
                out_host.copy_(res, non_blocking=True)
            e2e1.record()
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e2e0.elapsed_time(e2e1) / args.steps)
        e2e = {"value": world * paths_per_step / (e2e_ms / 1e3), "unit": "paths/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8, "ms_per_step": e2e_ms}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        cpu = cpu_reference(args.config, args.cpu_sample, os.cpu_count() or 1)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded curve, abcd vols, Sobol points of the reference's "
                    "Joe-Kuo 6.10200 table, MT19937 scramblers)",
            "config": {"workload": workload_name(args.config), "rates": n, "factors": F,
                       "steps": n, "regression_paths": 0 if euro else Preg, "pricing_paths": P,
                       "basis": cfg.basis, "mode": args.evolve,
                       "l2": "inputs larger than L2 (3.4 GB variates, 2 GB LS inputs per pass)",
                       "parallelism": f"dp{world} (disjoint Sobol ranges; LS sums "
                                      "all-reduced per date)" if world > 1 else
                                      "dp1 (disjoint Sobol ranges)"},
            "price": price, "staged": staged, "greeks": greeks, "nested": nested, "ab": ab,
            "stages": stages,
            "roofline": roofline,
            "clocks": clocks,
            "e2e": e2e, "gpu_launches": launches, "cpu_baseline": cpu}
    print(json.dumps(line))
    return 0


def main() -> int:
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
