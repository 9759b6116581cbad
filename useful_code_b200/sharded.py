"""Longstaff–Schwartz regression with the paths split over GPUs.

One process per GPU holds a disjoint range of regression paths.  Per
exercise date (backward) each GPU forms the unscaled sums of its paths (the
Gram of the basis and its product with the target), the sums are added over
the GPUs with one all-reduce, and every GPU solves the same normal
equations, so every GPU applies the same exercise rule.  The moments that
standardise the basis variables and the in-sample price are summed the same
way.  This is the per-date structure of the reference's regression
(generateMultiRegressionCoefficientsViaLS_gpu, LS_main_cula.h:565-837) with
the sums over paths extended across GPUs.

``backward`` is the protocol, written against a backend with five
operations; ``GpuBackend`` binds them to the C ABI (lmm_ls_moment_sums,
lmm_ls_moments_from_sums, lmm_ls_date_sums, lmm_ls_date_solve,
lmm_ls_final_sum).  ``allreduce`` sums a float64 tensor in place over the
processes (torch.distributed.all_reduce; the identity on one GPU).
"""
from __future__ import annotations

import ctypes
from typing import Callable

import torch

from ._lib import call
from .pricer import LSInputs, LSResult, Pipeline, dp, stream_handle


def n_sums(nbasis: int) -> int:
    """Doubles in one date's sums: pairs (i, j), j <= i <= K, slot K the target."""
    return (nbasis + 1) * (nbasis + 2) // 2


def backward(backend, E: int, nbasis, normalise: bool, total_paths: int,
             allreduce: Callable[[torch.Tensor], None]):
    """Run the regression; returns what backend.result() returns."""
    backend.begin()
    if normalise:
        m = backend.moment_sums()
        allreduce(m)
        backend.moments_from_sums(m, total_paths)
    for e in range(E - 1, -1, -1):
        sums = backend.date_sums(e)
        allreduce(sums)
        backend.date_solve(e, sums, total_paths)
    price = backend.final_sum()
    allreduce(price)
    return backend.result(price / total_paths)


class GpuBackend:
    """The backend over the C ABI for one GPU's share of the paths."""

    def __init__(self, pipe: Pipeline, ls: LSInputs):
        self.pipe, self.ls = pipe, ls
        self.E = pipe.E
        self.P = ls.num.shape[1]
        dev = pipe.device
        nbytes = int(pipe_ls_workspace(self.P, self.E))
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.beta = torch.zeros(self.E, 16, dtype=torch.float64, device=dev)
        norm = bool(pipe.mkt.cfg.normalise)
        self.means = torch.zeros(self.E, 3, device=dev) if norm else None
        self.sds = torch.ones(self.E, 3, device=dev) if norm else None
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.gram = torch.zeros(self.E, 16, 17, dtype=torch.float64, device=dev)

    def begin(self):
        self.status.zero_()

    def _tables(self):
        p = self.pipe
        return (ctypes.c_void_p(p._nvars.ctypes.data), ctypes.c_void_p(p._mono.ctypes.data),
                ctypes.c_void_p(p._nbasis.ctypes.data))

    def moment_sums(self) -> torch.Tensor:
        out = torch.zeros(self.E, 6, dtype=torch.float64, device=self.pipe.device)
        call("lmm_ls_moment_sums", self.E, self.P, dp(self.ls.vars), dp(self.ws),
             self.ws.numel(), dp(out), stream_handle())
        return out

    def moments_from_sums(self, sums: torch.Tensor, total: int):
        call("lmm_ls_moments_from_sums", self.E, float(total), dp(sums), dp(self.means),
             dp(self.sds), stream_handle())

    def date_sums(self, e: int) -> torch.Tensor:
        k = int(self.pipe._nbasis[e])
        out = torch.zeros(n_sums(k), dtype=torch.float64, device=self.pipe.device)
        nv, mono, nb = self._tables()
        call("lmm_ls_date_sums", e, self.E, self.P, dp(self.ls.vars), nv, mono, nb,
             dp(self.ls.cf), dp(self.ls.ex), dp(self.ls.num), dp(self.means), dp(self.sds),
             dp(self.beta), dp(self.ws), self.ws.numel(), dp(out), stream_handle())
        return out

    def date_solve(self, e: int, sums: torch.Tensor, total: int):
        call("lmm_ls_date_solve", e, int(self.pipe._nbasis[e]), dp(sums), float(total),
             dp(self.beta), dp(self.gram), dp(self.status), stream_handle())

    def final_sum(self) -> torch.Tensor:
        out = torch.zeros(1, dtype=torch.float64, device=self.pipe.device)
        nv, mono, nb = self._tables()
        call("lmm_ls_final_sum", self.E, self.P, dp(self.ls.vars), nv, mono, nb,
             dp(self.ls.cf), dp(self.ls.ex), dp(self.ls.num), dp(self.means), dp(self.sds),
             dp(self.beta), dp(self.ws), self.ws.numel(), dp(out), stream_handle())
        return out

    def result(self, price: torch.Tensor) -> LSResult:
        return LSResult(self.beta, self.means, self.sds, self.gram, self.status, price[0])


def pipe_ls_workspace(paths: int, n_exercise: int) -> int:
    from ._lib import LIB

    return LIB.lmm_ls_workspace_bytes(paths, n_exercise)


def regress_sharded(pipe: Pipeline, ls: LSInputs, total_paths: int,
                    allreduce: Callable[[torch.Tensor], None] | None = None) -> LSResult:
    """Regression over the union of every process's paths; ``ls`` holds this
    process's share, ``total_paths`` the sum of the shares."""
    if allreduce is None:
        def allreduce(t):
            return None
    be = GpuBackend(pipe, ls)
    return backward(be, pipe.E, pipe._nbasis, bool(pipe.mkt.cfg.normalise), total_paths,
                    allreduce)
