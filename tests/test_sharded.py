"""The sharded regression protocol (useful_code_b200.sharded.backward) over
two processes with the gloo backend on the CPU.

Each rank holds half of the paths of the reference's gold LS fixture and
runs the protocol with a NumPy FP64 backend that performs the same five
operations as the GPU entry points (per-rank moment sums, per-date sums of
the basis Gram and target after the next date's decision, solve from the
all-reduced sums, final in-sample sum).  The result must equal the FP64
oracle's regression on all paths in one process (orc_ls_regress_d)."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch

HERE = os.path.dirname(__file__)


class NumpyBackend:
    def __init__(self, vars_, cf, ex, num, nvars, mono, nbasis, normalise):
        self.v, self.cf, self.ex, self.num = vars_, cf, ex, num
        self.nvars, self.mono, self.nb = nvars, mono, nbasis
        self.E, _, self.P = vars_.shape
        self.norm = normalise
        self.beta = np.zeros((self.E, 16))
        self.means = np.zeros((self.E, 3))
        self.sds = np.ones((self.E, 3))
        self.y = np.zeros(self.P)

    def begin(self):
        self.y[:] = 0.0

    def _phi(self, e):
        V, K = int(self.nvars[e]), int(self.nb[e])
        x = np.zeros((3, self.P))
        for v in range(V):
            x[v] = (self.v[e, v] - self.means[e, v]) / self.sds[e, v]
        phi = np.ones((K, self.P))
        for k in range(K):
            for v in range(3):
                phi[k] *= x[v] ** int(self.mono[e, k, v])
        return phi

    def moment_sums(self):
        s = np.zeros((self.E, 6))
        for e in range(self.E):
            for v in range(3):
                s[e, 2 * v] = self.v[e, v].sum()
                s[e, 2 * v + 1] = (self.v[e, v] ** 2).sum()
        return torch.from_numpy(s)

    def moments_from_sums(self, sums, total):
        s = sums.numpy()
        for e in range(self.E):
            for v in range(3):
                m = s[e, 2 * v] / total
                var = s[e, 2 * v + 1] / total - m * m
                sd = np.sqrt(var) if var > 0 else 0.0
                self.means[e, v] = m
                self.sds[e, v] = sd if sd > 0 else 1.0

    def _decide(self, e, deflate):
        K = int(self.nb[e])
        est = self.beta[e, :K] @ self._phi(e)
        exv = self.ex[e]
        self.y = np.where(exv > est, exv, self.y + self.cf[e])
        if deflate:
            self.y = self.y * self.num[e - 1] / self.num[e]

    def date_sums(self, e):
        if e + 1 < self.E:
            self._decide(e + 1, True)
        K = int(self.nb[e])
        slots = np.vstack([self._phi(e), (self.cf[e] + self.y)[None]])
        out = np.zeros((K + 1) * (K + 2) // 2)
        for i in range(K + 1):
            for j in range(i + 1):
                out[i * (i + 1) // 2 + j] = np.dot(slots[i], slots[j])
        return torch.from_numpy(out)

    def date_solve(self, e, sums, total):
        K = int(self.nb[e])
        s = sums.numpy() / total
        G = np.zeros((K, K))
        for i in range(K):
            for j in range(i + 1):
                G[i, j] = G[j, i] = s[i * (i + 1) // 2 + j]
        b = np.array([s[K * (K + 1) // 2 + i] for i in range(K)])
        self.beta[e, :K] = np.linalg.solve(G, b)

    def final_sum(self):
        self._decide(0, False)
        return torch.tensor([np.sum(self.y / self.num[0])], dtype=torch.float64)

    def result(self, price):
        return self.beta.copy(), float(price[0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, data, out_path):
    import torch.distributed as dist

    from useful_code_b200.sharded import backward

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v, cf, ex, num, nvars, mono, nb = data
        P = v.shape[2]
        lo, hi = rank * P // world, (rank + 1) * P // world
        be = NumpyBackend(v[:, :, lo:hi], cf[:, lo:hi], ex[:, lo:hi], num[:, lo:hi],
                          nvars, mono, nb, True)
        beta, price = backward(be, v.shape[0], nb, True, P,
                               lambda t: dist.all_reduce(t))
        if rank == 0:
            np.savez(out_path, beta=beta, price=price)
    finally:
        dist.destroy_process_group()


def test_two_process_regression_equals_one(gold, orc, tmp_path):
    import torch.multiprocessing as mp

    from useful_code_b200 import market as mk

    v = gold["ls_vars"].astype(np.float64)
    cf = gold["ls_cf"].astype(np.float64)
    ex = gold["ls_ex"].astype(np.float64)
    num = gold["ls_num"].astype(np.float64)
    nvars = gold["ls_nvars"]
    mono, nb = mk.basis_tables("cross", nvars)
    E, _, P = v.shape
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_rank, args=(2, _free_port(), (v, cf, ex, num, nvars, mono, nb), out),
                       nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    b_ref = np.zeros((E, 16))
    p_ref = orc("orc_ls_regress_d", E, P, v, nvars, mono, nb, cf, ex, num, 1, b_ref,
                np.zeros((E, 3)), np.zeros((E, 3)), None, restype=ctypes.c_double)
    assert abs(float(got["price"]) - p_ref) < 1e-12
    K = nb[0]
    # the last date's basis is singular in the fixture (collinear variables):
    # compare the well-posed dates
    np.testing.assert_allclose(got["beta"][:-1, :K], b_ref[:-1, :K], rtol=1e-8, atol=1e-10)
