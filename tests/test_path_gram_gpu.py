"""Tensor-core path contraction (lmm_path_gram, split-TF32 tcgen05) against
an FP64 NumPy product (GPU)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
VP = ctypes.c_void_p


@pytest.mark.parametrize("m,n,paths,same,ld_pad", [
    (11, 11, 100003, True, 1),     # LS Gram: 10 basis functions + target, odd path count
    (80, 80, 65536, False, 0),     # adjoint-sized outer products
    (80, 10, 4097, False, 3),      # rectangular, one path past a chunk
    (128, 128, 8192, True, 0),     # full tile
])
def test_path_gram_matches_fp64(cuda, m, n, paths, same, ld_pad):
    import torch

    from useful_code_b200._lib import LIB, call

    rng = np.random.default_rng(m * 1000 + n)
    ld = ((paths + 3) // 4) * 4 + 4 * ld_pad
    X = np.zeros((m, ld), np.float32)
    X[:, :paths] = (rng.standard_normal((m, paths)) * rng.uniform(0.01, 3.0, (m, 1)))
    if same:
        Y = X
    else:
        Y = np.zeros((n, ld), np.float32)
        Y[:, :paths] = rng.standard_normal((n, paths)) + 0.5
    dX = torch.from_numpy(X).cuda()
    dY = dX if same else torch.from_numpy(Y).cuda()
    G = torch.zeros(m, n, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(LIB.lmm_path_gram_workspace_bytes(m, n, paths)), dtype=torch.uint8,
                     device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    scale = 1.0 / paths
    call("lmm_path_gram", m, n, paths, VP(dX.data_ptr()), ld, VP(dY.data_ptr()), ld, scale,
         VP(G.data_ptr()), VP(ws.data_ptr()), ws.numel(), VP(st.data_ptr()), None)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = (X[:, :paths].astype(np.float64) @ Y[:, :paths].astype(np.float64).T) * scale
    got = G.cpu().numpy()
    dx = np.sqrt(np.einsum("ij,ij->i", X[:, :paths].astype(np.float64), X[:, :paths]) * scale)
    dy = np.sqrt(np.einsum("ij,ij->i", Y[:, :paths].astype(np.float64), Y[:, :paths]) * scale)
    err = np.abs(got - ref) / np.outer(dx, dy)
    assert err.max() < 2e-6, err.max()


def test_bounded_wait_times_out_and_frees_tensor_memory(cuda):
    """A wait on an mbarrier that nothing signals runs out after its limit,
    reports it in the status word and frees the tensor memory it holds; the
    context stays usable (a contraction right after is exact)."""
    import time

    import torch

    from useful_code_b200._lib import LIB, SIGNATURES, call

    assert SIGNATURES["lmm_tensor_wait_selftest"][1][0] is ctypes.c_ulonglong
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    call("lmm_tensor_wait_selftest", 2_000_000, VP(st.data_ptr()), None)  # 2 ms
    torch.cuda.synchronize()
    assert int(st.item()) == 1
    assert time.perf_counter() - t0 < 5.0
    m, paths = 11, 4096
    X = np.random.default_rng(1).standard_normal((m, paths)).astype(np.float32)
    dX = torch.from_numpy(X).cuda()
    G = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(LIB.lmm_path_gram_workspace_bytes(m, m, paths)), dtype=torch.uint8,
                     device="cuda")
    st.zero_()
    call("lmm_path_gram", m, m, paths, VP(dX.data_ptr()), paths, VP(dX.data_ptr()), paths, 1.0,
         VP(G.data_ptr()), VP(ws.data_ptr()), ws.numel(), VP(st.data_ptr()), None)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = X.astype(np.float64) @ X.astype(np.float64).T
    assert np.max(np.abs(G.cpu().numpy() - ref)) < 2e-6 * np.max(np.abs(ref))
