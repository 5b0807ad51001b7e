"""The tcgen05 BF16x3 GEMM against an FP64 matmul (through the C ABI test hook).

Tolerance: the 3-term split keeps ~16 mantissa bits per product, so results
match FP64 to ~1e-5 relative; the bar here is 2e-4 of the largest entry.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(mode, A, B, alpha=None, zeta=2):
    import torch

    from librascal_b200 import _native as N
    dev = torch.device("cuda")
    At = torch.as_tensor(A, dtype=torch.float32, device=dev).contiguous()
    Bt = torch.as_tensor(B, dtype=torch.float32, device=dev).contiguous()
    M, K = At.shape
    Nn = Bt.shape[0]
    C = torch.zeros((M, Nn), dtype=torch.float32, device=dev)
    e = torch.zeros(M, dtype=torch.float32, device=dev)
    al = torch.as_tensor(alpha if alpha is not None else np.zeros(Nn), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    N.check(N.lib().rgpu_debug_gemm_bf16x3(mode, M, Nn, K, At.data_ptr(), Bt.data_ptr(), al.data_ptr(), zeta,
                                           C.data_ptr(), e.data_ptr(), None))
    torch.cuda.synchronize()
    return C.cpu().numpy().astype(np.float64), e.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (1, 4, 8), (300, 500, 6720), (1000, 2000, 640),
                                   (257, 260, 130), (64, 1024, 448)])
def test_plain_gemm(M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.random((M, K)) / np.sqrt(K)
    B = rng.normal(size=(N, K))
    C, _ = run(0, A, B)
    ref = np.float32(A).astype(np.float64) @ np.float32(B).astype(np.float64).T
    assert np.abs(C - ref).max() <= 2e-4 * np.abs(ref).max()


@pytest.mark.parametrize("zeta", [1, 2, 3])
def test_gap_epilogue(zeta):
    rng = np.random.default_rng(zeta)
    M, N, K = 333, 777, 1344
    A = rng.random((M, K))
    A /= np.linalg.norm(A, axis=1, keepdims=True)
    B = rng.random((N, K))
    B /= np.linalg.norm(B, axis=1, keepdims=True)
    alpha = rng.normal(size=N)
    W, e = run(1, A, B, alpha, zeta)
    k = np.float32(A).astype(np.float64) @ np.float32(B).astype(np.float64).T
    al = np.float32(alpha).astype(np.float64)
    W_ref = al * zeta * k ** (zeta - 1)
    e_ref = (al * k ** zeta).sum(axis=1)
    assert np.abs(W - W_ref).max() <= 2e-4 * np.abs(W_ref).max()
    assert np.abs(e - e_ref).max() <= 2e-4 * np.abs(e_ref).max()
