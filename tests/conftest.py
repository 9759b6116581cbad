"""Shared fixtures: the golden fixtures, the CPU oracle and GPU helpers.

The oracle (oracle/liblmm_oracle.so, the CPU restatement) and the
reference's gold library (oracle/_ref/libkooref.so, when it was built in
this container) are test infrastructure: only tests load them.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
ORACLE_SO = ROOT / "oracle" / "liblmm_oracle.so"
REF_SO = ROOT / "oracle" / "_ref" / "libkooref.so"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle() -> Path:
    src = ROOT / "oracle" / "lmm_oracle.cpp"
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True,
                       capture_output=True)
    return ORACLE_SO


class CLib:
    """ctypes wrapper converting numpy arrays / numbers on the fly."""

    def __init__(self, path: Path):
        self.lib = ctypes.CDLL(str(path))

    @staticmethod
    def _conv(a):
        if isinstance(a, np.ndarray):
            assert a.flags["C_CONTIGUOUS"]
            return ctypes.c_void_p(a.ctypes.data)
        if a is None:
            return ctypes.c_void_p(None)
        if isinstance(a, (bool, np.bool_)):
            return ctypes.c_int(int(a))
        if isinstance(a, (int, np.integer)) and not isinstance(a, np.uint32):
            return ctypes.c_int(int(a))
        if isinstance(a, np.uint32):
            return ctypes.c_uint32(int(a))
        if isinstance(a, np.float32):
            return ctypes.c_float(float(a))
        if isinstance(a, float):
            return ctypes.c_double(a)
        return a

    def __call__(self, name, *args, restype=None):
        fn = getattr(self.lib, name)
        fn.restype = restype
        return fn(*[self._conv(a) for a in args])


@pytest.fixture(scope="session")
def gold():
    # materialise once: NpzFile returns a new array on every access, and a
    # raw pointer into such a temporary would dangle
    with np.load(GOLDEN / "kooderive_gold_small.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def gold_bridge():
    """The reference's newBridge (brownian_bridge::transformCPU) outputs."""
    with np.load(GOLDEN / "kooderive_bridge.npz") as z:
        return {k: z[k] for k in z.files}


BRIDGE_SHAPES = [(20, 3), (40, 5), (80, 10), (120, 15), (1, 1), (2, 1), (7, 2), (33, 4), (64, 16)]


@pytest.fixture(scope="session")
def ref_dirs():
    return np.load(GOLDEN / "sobol_directions_ref1800.npy")


@pytest.fixture(scope="session")
def orc():
    return CLib(_ensure_oracle())


@pytest.fixture(scope="session")
def kref():
    if not REF_SO.exists():
        pytest.skip("reference gold library not built (needs the reference tree)")
    return CLib(REF_SO)


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")


def rel_err(a, b, floor=1e-12):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)
