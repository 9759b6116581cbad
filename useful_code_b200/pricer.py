"""Pricing pipelines over the C ABI (include/lmm_pipeline.h).

``Pipeline`` uploads a ``market.Market`` to the GPU once and then runs,
on torch's current CUDA stream, the first pass (Longstaff–Schwartz inputs),
the device-resident regression (lmm_ls_regress) and the second pass
(frozen-rule pricing), in the plain FP32 staged form or the fused form.
Device memory comes from torch; the library itself allocates nothing.
The structure mirrors BermudanMultiLSPricerExample
(kooexample/bermudanIRDPricer.cu:94-1561): batches of paths with disjoint
Sobol offsets, regression over all first-pass paths, then independent
second-pass paths.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import market as mk
from ._lib import call

_VP = ctypes.c_void_p
MODES = {"staged": 0, "fused": 1, "tensor": 2}


class LmmModel(ctypes.Structure):
    _fields_ = [
        ("rates", ctypes.c_int),
        ("factors", ctypes.c_int),
        ("h_taus", _VP),
        ("h_displacements", _VP),
        ("h_initial_rates", _VP),
        ("d_A", _VP),
        ("d_fixed_drifts", _VP),
        ("d_directions", _VP),
        ("d_scramblers", _VP),
        ("scramble_dims", ctypes.c_int),
        ("cutoff", ctypes.c_float),
    ]


class LmmProduct(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("strike", ctypes.c_float),
        ("cap_strike", ctypes.c_float),
        ("pay_receive", ctypes.c_float),
        ("n_exercise", ctypes.c_int),
        ("h_exercise_steps", _VP),
        ("h_nvars", _VP),
        ("h_monomials", _VP),
        ("h_nbasis", _VP),
        ("normalise", ctypes.c_int),
        ("tarn_total", ctypes.c_float),
        ("tarn_multiplier", ctypes.c_float),
    ]


def _hp(a: np.ndarray):
    return _VP(a.ctypes.data) if a is not None and a.size else None


def dp(t: torch.Tensor | None):
    return _VP(t.data_ptr()) if t is not None else None


def stream_handle() -> _VP:
    return _VP(torch.cuda.current_stream().cuda_stream)


@dataclass
class LSInputs:
    vars: torch.Tensor  # [E][3][P]
    ex: torch.Tensor  # [E][P]
    cf: torch.Tensor  # [E][P]
    num: torch.Tensor  # [E][P]


@dataclass
class LSResult:
    beta: torch.Tensor  # [E][16] float64 ([E][depth][16] for nested rules)
    means: torch.Tensor | None
    sds: torch.Tensor | None
    gram: torch.Tensor | None
    status: torch.Tensor
    price: torch.Tensor  # scalar float64, units of the T_0 numeraire
    depth: int = 1
    cuts: torch.Tensor | None = None    # [E][depth][2] float64 (nested)
    npaths: torch.Tensor | None = None  # [E][depth] paths per regression
    shifts: torch.Tensor | None = None  # [E] float32 Andersen shifts


class LmmLsSelect(ctypes.Structure):
    """lmm_ls_select (include/lmm_c.h)."""
    _fields_ = [
        ("depth", ctypes.c_int),
        ("lower_frac", ctypes.c_double),
        ("upper_frac", ctypes.c_double),
        ("sds", ctypes.c_double),
        ("multiplier", ctypes.c_double),
        ("min_paths", ctypes.c_int),
    ]


class LmmLsRule(ctypes.Structure):
    """lmm_ls_rule (include/lmm_c.h)."""
    _fields_ = [
        ("depth", ctypes.c_int),
        ("d_beta", ctypes.c_void_p),
        ("d_means", ctypes.c_void_p),
        ("d_sds", ctypes.c_void_p),
        ("d_cuts", ctypes.c_void_p),
        ("d_shifts", ctypes.c_void_p),
    ]


@dataclass
class Selector:
    """Nested-regression settings (the reference's RegressionSelectorFraction
    with regression depth, kooexample/bermudanIRDPricer.cu:94-131)."""
    depth: int = 1
    lower_frac: float = 0.1
    upper_frac: float = 0.101
    sds: float = 2.5
    multiplier: float = 0.8
    min_paths: int = 900

    @staticmethod
    def production(depth: int, min_paths: int = 900) -> "Selector":
        """The reference's production sweep (kooexample/main.cpp:143-178):
        lower fraction 0.1^(1/(depth-1)), upper = 1.01 x lower, 2.5 sds,
        multiplier 0.8, 900 paths."""
        lf = 0.1 ** (1.0 / (depth - 1)) if depth > 1 else 0.1
        return Selector(depth, lf, lf * 1.01, 2.5, 0.8, min_paths)


class LmmAbConfig(ctypes.Structure):
    """lmm_ab_config (include/lmm_pipeline.h)."""
    _fields_ = [
        ("outer_paths", ctypes.c_int),
        ("outer_offset", ctypes.c_uint32),
        ("inner_paths", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
    ]


@dataclass
class ABResult:
    """Andersen–Broadie estimate (units of the numeraire at T_0): lower = the
    rule's value on the outer paths, gap = duality gap, upper = lower + gap;
    per-path arrays when kept."""
    lower: float
    lower_se: float
    gap: float
    gap_se: float
    Q: torch.Tensor | None = None
    X: torch.Tensor | None = None
    Z: torch.Tensor | None = None
    ckpt: torch.Tensor | None = None
    ckptN: torch.Tensor | None = None

    @property
    def upper(self) -> float:
        return self.lower + self.gap


def rule_struct(rule: LSResult) -> LmmLsRule:
    return LmmLsRule(rule.depth, dp(rule.beta), dp(rule.means), dp(rule.sds), dp(rule.cuts),
                     dp(rule.shifts))


class Pipeline:
    def __init__(self, mkt: mk.Market, device: str = "cuda"):
        self.mkt = mkt
        cfg = mkt.cfg
        self.device = torch.device(device)
        dev = self.device
        self.A = torch.from_numpy(mkt.A).to(dev)
        self.fixed = torch.from_numpy(mkt.fixed).to(dev)
        self.dirs = torch.from_numpy(mkt.directions.astype(np.int32)).to(dev)
        self.scr = torch.from_numpy(mkt.scramblers.astype(np.int32)).to(dev)
        # host arrays referenced by the descriptors must stay alive
        self._taus = np.ascontiguousarray(mkt.taus)
        self._disp = np.ascontiguousarray(mkt.disp)
        self._f0 = np.ascontiguousarray(mkt.f0)
        self._ex = np.ascontiguousarray(mkt.ex_steps.astype(np.int32))
        self._nvars = np.ascontiguousarray(mkt.nvars.astype(np.int32))
        self._mono = np.ascontiguousarray(mkt.mono.astype(np.uint8))
        self._nbasis = np.ascontiguousarray(mkt.nbasis.astype(np.int32))
        self.model = LmmModel(cfg.n, cfg.F, _hp(self._taus), _hp(self._disp), _hp(self._f0),
                              dp(self.A), dp(self.fixed), dp(self.dirs), dp(self.scr),
                              mkt.scramble_dims, cfg.cutoff)
        self.product = LmmProduct(mk.PRODUCTS[cfg.product], cfg.strike, cfg.cap_strike,
                                  cfg.pay_receive, len(self._ex), _hp(self._ex),
                                  _hp(self._nvars), _hp(self._mono), _hp(self._nbasis),
                                  int(cfg.normalise), cfg.tarn_total, cfg.tarn_multiplier)
        self.E = len(self._ex)
        self._ws = {}
        self._greeks_ws = {}

    # -- workspace -----------------------------------------------------------
    def workspace(self, paths: int, mode: str) -> torch.Tensor:
        nbytes = call_size("lmm_pipeline_workspace_bytes", ctypes.addressof(self.model),
                           ctypes.addressof(self.product), paths, MODES[mode])
        key = (mode, paths)
        ws = self._ws.get(key)
        if ws is None or ws.numel() < nbytes:
            ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws[key] = ws
        return ws

    # -- passes ----------------------------------------------------------------
    def alloc_inputs(self, total: int) -> LSInputs:
        E, dev = self.E, self.device
        return LSInputs(torch.empty(E, 3, total, device=dev), torch.empty(E, total, device=dev),
                        torch.empty(E, total, device=dev), torch.empty(E, total, device=dev))

    def first_pass(self, paths: int, path_offset: int = 0, mode: str = "fused",
                   batch: int | None = None, out: LSInputs | None = None) -> LSInputs:
        batch = batch or paths
        out = out or self.alloc_inputs(paths)
        for col in range(0, paths, batch):
            b = min(batch, paths - col)
            ws = self.workspace(b, mode)
            call("lmm_pipeline_first_pass", ctypes.addressof(self.model),
                 ctypes.addressof(self.product), b, path_offset + col, MODES[mode], dp(ws),
                 ws.numel(), paths, col, dp(out.vars), dp(out.ex), dp(out.cf), dp(out.num),
                 stream_handle())
        return out

    def regress(self, ls: LSInputs, keep_gram: bool = False) -> LSResult:
        E, P, dev = self.E, ls.num.shape[1], self.device
        ws = torch.empty(call_size("lmm_ls_workspace_bytes", P, E), dtype=torch.uint8, device=dev)
        beta = torch.zeros(E, 16, dtype=torch.float64, device=dev)
        norm = bool(self.product.normalise)
        means = torch.zeros(E, 3, device=dev) if norm else None
        sds = torch.ones(E, 3, device=dev) if norm else None
        gram = torch.zeros(E, 16, 17, dtype=torch.float64, device=dev) if keep_gram else None
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        price = torch.zeros(1, dtype=torch.float64, device=dev)
        call("lmm_ls_regress", E, P, dp(ls.vars), _hp(self._nvars), _hp(self._mono),
             _hp(self._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), int(norm), dp(ws), ws.numel(),
             dp(beta), dp(means), dp(sds), dp(gram), dp(status), dp(price), stream_handle())
        return LSResult(beta, means, sds, gram, status, price)

    def regress_nested(self, ls: LSInputs, select: Selector) -> LSResult:
        """Regression with nested regressions and path selection
        (lmm_ls_regress_nested)."""
        E, P, dev, D = self.E, ls.num.shape[1], self.device, select.depth
        ws = torch.empty(call_size("lmm_ls_nested_workspace_bytes", P, E), dtype=torch.uint8,
                         device=dev)
        beta = torch.zeros(E, D, 16, dtype=torch.float64, device=dev)
        norm = bool(self.product.normalise)
        means = torch.zeros(E, D, 3, device=dev) if norm else None
        sds = torch.ones(E, D, 3, device=dev) if norm else None
        cuts = torch.zeros(E, D, 2, dtype=torch.float64, device=dev)
        npaths = torch.zeros(E, D, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        price = torch.zeros(1, dtype=torch.float64, device=dev)
        sel = LmmLsSelect(D, select.lower_frac, select.upper_frac, select.sds, select.multiplier,
                          select.min_paths)
        call("lmm_ls_regress_nested", E, P, dp(ls.vars), _hp(self._nvars), _hp(self._mono),
             _hp(self._nbasis), dp(ls.cf), dp(ls.ex), dp(ls.num), int(norm),
             ctypes.addressof(sel), dp(ws), ws.numel(), dp(beta), dp(means), dp(sds), dp(cuts),
             dp(npaths), dp(status), dp(price), stream_handle())
        return LSResult(beta, means, sds, None, status, price, D, cuts, npaths)

    def regress_nested_graph(self, ls: LSInputs, select: Selector):
        """lmm_ls_regress_nested on these inputs captured as a CUDA graph.

        The entry point issues a fixed sequence of launches (about 2,300 at
        80 dates and depth 4) with no host synchronisation, so it captures
        whole; ``graph.replay()`` recomputes the rule from the current
        contents of ``ls`` into the returned result's buffers, without the
        host's launch work.  Returns (graph, result)."""
        side = torch.cuda.Stream(device=self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.regress_nested(ls, select)  # sets kernel attributes outside the capture
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, capture_error_mode="thread_local"):
            result = self.regress_nested(ls, select)
        torch.cuda.synchronize(self.device)
        return graph, result

    def second_pass(self, paths: int, path_offset: int, rule: LSResult | None,
                    mode: str = "fused", batch: int | None = None,
                    out: torch.Tensor | None = None) -> torch.Tensor:
        batch = batch or paths
        out = out if out is not None else torch.empty(paths, device=self.device)
        nested = rule is not None and (rule.depth > 1 or rule.shifts is not None)
        rs = rule_struct(rule) if nested else None
        for col in range(0, paths, batch):
            b = min(batch, paths - col)
            ws = self.workspace(b, mode)
            if nested:
                call("lmm_pipeline_second_pass_rule", ctypes.addressof(self.model),
                     ctypes.addressof(self.product), b, path_offset + col, MODES[mode],
                     ctypes.addressof(rs), dp(ws), ws.numel(), dp(out[col:col + b]),
                     stream_handle())
                continue
            call("lmm_pipeline_second_pass", ctypes.addressof(self.model),
                 ctypes.addressof(self.product), b, path_offset + col, MODES[mode],
                 dp(rule.beta) if rule else None, dp(rule.means) if rule else None,
                 dp(rule.sds) if rule else None, dp(ws), ws.numel(), dp(out[col:col + b]),
                 stream_handle())
        return out

    def andersen_broadie(self, rule: LSResult, outer_paths: int, outer_offset: int,
                         inner_paths: int, seed: int = 20240601,
                         keep: bool = False) -> ABResult:
        """Andersen–Broadie duality gap of a frozen rule (lmm_andersen_broadie)."""
        cfg = LmmAbConfig(outer_paths, outer_offset, inner_paths, seed)
        nbytes = call_size("lmm_andersen_broadie_workspace_bytes", ctypes.addressof(self.model),
                           ctypes.addressof(self.product), ctypes.addressof(cfg))
        dev, E, K, n = self.device, self.E, outer_paths, self.mkt.cfg.n
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        out = torch.zeros(4, dtype=torch.float64, device=dev)
        Q = X = Z = ck = ckN = None
        if keep:
            Q = torch.zeros(E, K, dtype=torch.float64, device=dev)
            X = torch.zeros(E, K, dtype=torch.int32, device=dev)
            Z = torch.zeros(E, K, dtype=torch.float64, device=dev)
            ck = torch.zeros(n, n, K, device=dev)
            ckN = torch.zeros(n, K, device=dev)
        rs = rule_struct(rule)
        call("lmm_andersen_broadie", ctypes.addressof(self.model), ctypes.addressof(self.product),
             ctypes.addressof(rs), ctypes.addressof(cfg), dp(ws), ws.numel(), dp(out), dp(Q),
             dp(X), dp(Z), dp(ck), dp(ckN), stream_handle())
        o = out.cpu().numpy()
        return ABResult(float(o[2]), float(o[3]), float(o[0]), float(o[1]), Q, X, Z, ck, ckN)

    def greeks(self, paths: int, path_offset: int, rule: LSResult | None,
               checkpoint_every: int = 8) -> Greeks:
        """Pathwise adjoint Greeks of the frozen-rule price over paths
        [path_offset, path_offset + paths) (lmm_greeks)."""
        return _greeks(self, paths, path_offset, rule, checkpoint_every)

    def mean(self, x: torch.Tensor) -> torch.Tensor:
        part = torch.empty(call_size("lmm_reduce_workspace_doubles"), dtype=torch.float64,
                           device=self.device)
        res = torch.empty(1, dtype=torch.float64, device=self.device)
        call("lmm_reduce_mean_ratio", dp(x), None, x.numel(), dp(part), dp(res), stream_handle())
        return res

    def price(self, reg_paths: int, paths: int, mode: str = "fused", reg_offset: int = 0,
              price_offset: int | None = None, batch: int | None = None,
              select: Selector | None = None, shifts: np.ndarray | None = None) -> dict:
        """Full two-pass Bermudan (or one-pass European) price at time 0;
        `select` asks for nested regressions, `shifts` for per-date Andersen
        shifts in the second pass."""
        price_offset = reg_paths + reg_offset if price_offset is None else price_offset
        scale = self.mkt.initial_numeraire
        if self.mkt.cfg.product in ("european", "tarn"):
            pay = self.second_pass(paths, price_offset, None, mode, batch)
            return {"price": float(self.mean(pay).item()) * scale}
        ls = self.first_pass(reg_paths, reg_offset, mode, batch)
        rule = self.regress_nested(ls, select) if select is not None else self.regress(ls)
        if shifts is not None:
            rule.shifts = torch.as_tensor(np.asarray(shifts, np.float32), device=self.device)
        pay = self.second_pass(paths, price_offset, rule, mode, batch)
        return {"price": float(self.mean(pay).item()) * scale,
                "insample": float(rule.price.item()) * scale,
                "ls_status": int(rule.status.item())}


@dataclass
class Greeks:
    price: float           # frozen-rule price at time 0
    delta: np.ndarray      # [rates] dV/df0_r
    abar: np.ndarray       # [steps][rates][factors] dV/dA
    vega_rate: np.ndarray  # [rates] dV/dk_r, A_s[r] -> k_r A_s[r]
    exercise_step: np.ndarray  # [paths] exercise step of each path (rates = never)


def _greeks(pipe: "Pipeline", paths: int, path_offset: int, rule: LSResult | None,
            checkpoint_every: int = 8) -> Greeks:
    cfg = pipe.mkt.cfg
    n, F = cfg.n, cfg.F
    nbytes = call_size("lmm_greeks_workspace_bytes", ctypes.addressof(pipe.model),
                       ctypes.addressof(pipe.product), paths, checkpoint_every)
    dev = pipe.device
    ws = pipe._greeks_ws.get(paths)
    if ws is None or ws.numel() < nbytes:
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        pipe._greeks_ws = {paths: ws}
    price = torch.zeros(1, dtype=torch.float64, device=dev)
    delta = torch.zeros(n, dtype=torch.float64, device=dev)
    abar = torch.zeros(n, n, F, dtype=torch.float64, device=dev)
    vega = torch.zeros(n, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    ex_step = torch.zeros(paths, dtype=torch.int32, device=dev)
    call("lmm_greeks", ctypes.addressof(pipe.model), ctypes.addressof(pipe.product), paths,
         path_offset, dp(rule.beta) if rule else None, dp(rule.means) if rule else None,
         dp(rule.sds) if rule else None, float(pipe.mkt.rate_times[0]), checkpoint_every,
         dp(ws), ws.numel(), dp(price), dp(delta), dp(abar), dp(vega), dp(ex_step),
         dp(status), stream_handle())
    torch.cuda.synchronize(dev)
    if int(status.item()) != 0:
        raise RuntimeError(f"lmm_greeks: device status {int(status.item())}")
    return Greeks(float(price.item()), delta.cpu().numpy(), abar.cpu().numpy(),
                  vega.cpu().numpy(), ex_step.cpu().numpy())


def call_size(name: str, *args) -> int:
    from ._lib import LIB

    return int(getattr(LIB, name)(*args))
