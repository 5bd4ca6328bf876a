"""Tensor-core (tcgen05) batched Gram matrices, G = M M^T per 16-row matrix, against FP64."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gram(sb, M):
    import torch
    L = sb.lib()
    L.snapi_batched_gram.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    nmat, _, K = M.shape
    dM = torch.from_numpy(np.ascontiguousarray(M, np.float32)).cuda()
    dG = torch.full((nmat, 16, 16), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = L.snapi_batched_gram(nmat, K, dM.data_ptr(), dG.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    return dG.cpu().numpy()


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


@pytest.mark.parametrize("nmat,K", [(8, 64), (20, 804), (3, 8)])
def test_gram_matches_fp64(sb, nmat, K):
    rng = np.random.default_rng(nmat + K)
    # rows of very different magnitude, as scaled Jacobian rows are, and a zero row
    M = rng.standard_normal((nmat, 16, K)) * (10.0 ** rng.uniform(-3, 3, (nmat, 16, 1)))
    M[:, 15] = 0.0
    M = M.astype(np.float32)
    G = _gram(sb, M)
    ref = np.einsum("mik,mjk->mij", M.astype(np.float64), M.astype(np.float64))
    # 3xTF32 split with FP32 accumulation: ~1e-6 of each row pair's own scale
    scale = np.sqrt(np.einsum("mii->mi", ref))
    tol = 1e-5 * scale[:, :, None] * scale[:, None, :] + 1e-30
    assert np.all(np.isfinite(G))
    assert np.all(np.abs(G - ref) <= tol), np.max(np.abs(G - ref) / tol)
