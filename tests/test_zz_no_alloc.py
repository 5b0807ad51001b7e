"""rgpu_gap_energies_noalloc (static scratch, no device allocation) against
the allocating GEMM entry point rgpu_debug_gemm_bf16x3 (mode 1) and an FP64
matmul.

Both entry points run the same tcgen05 BF16x3 GEMM and epilogue, so their
energies agree to FP32 summation order (bar: 1e-6 of the largest energy);
against FP64 the bar is the GEMM test's 2e-4 of the largest energy. Kept in
its own file, collected last, so it also runs after every other GPU test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.random((M, K))
    A /= np.linalg.norm(A, axis=1, keepdims=True)
    B = rng.random((N, K))
    B /= np.linalg.norm(B, axis=1, keepdims=True)
    return A, B, rng.normal(size=N)


def _energies(A, B, alpha, zeta, noalloc):
    import torch

    from librascal_b200 import _native as N
    dev = torch.device("cuda")
    At = torch.as_tensor(A, dtype=torch.float32, device=dev).contiguous()
    Bt = torch.as_tensor(B, dtype=torch.float32, device=dev).contiguous()
    al = torch.as_tensor(alpha, dtype=torch.float32, device=dev)
    M, K = At.shape
    Nn = Bt.shape[0]
    e = torch.full((M,), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    if noalloc:
        N.check(N.lib().rgpu_gap_energies_noalloc(M, Nn, K, At.data_ptr(), Bt.data_ptr(), al.data_ptr(), zeta,
                                                  e.data_ptr(), None))
    else:
        C = torch.zeros((M, Nn), dtype=torch.float32, device=dev)
        N.check(N.lib().rgpu_debug_gemm_bf16x3(1, M, Nn, K, At.data_ptr(), Bt.data_ptr(), al.data_ptr(), zeta,
                                               C.data_ptr(), e.data_ptr(), None))
    torch.cuda.synchronize()
    return e.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("M,N,K,zeta", [(333, 777, 1344, 2), (1, 4, 8, 2), (1000, 600, 448, 3), (257, 260, 130, 1)])
def test_noalloc_matches_allocating_entry(M, N, K, zeta):
    A, B, alpha = _inputs(M, N, K, M + N + K)
    ref = _energies(A, B, alpha, zeta, noalloc=False)
    k = np.float32(A).astype(np.float64) @ np.float32(B).astype(np.float64).T
    e64 = (np.float32(alpha).astype(np.float64) * k ** zeta).sum(axis=1)
    scale = np.abs(ref).max()
    # two calls in a row through the same static scratch
    for _ in range(2):
        e = _energies(A, B, alpha, zeta, noalloc=True)
        assert np.isfinite(e).all()
        assert np.abs(e - ref).max() <= 1e-6 * scale
        assert np.abs(e - e64).max() <= 2e-4 * np.abs(e64).max()


def test_noalloc_reuses_scratch_across_shapes():
    """A smaller call after a larger one reads nothing the larger one left."""
    A, B, alpha = _inputs(900, 1000, 1024, 7)
    big = _energies(A, B, alpha, 2, noalloc=True)
    assert np.abs(big - _energies(A, B, alpha, 2, noalloc=False)).max() <= 1e-6 * np.abs(big).max()
    A2, B2, alpha2 = _inputs(50, 70, 96, 8)
    small = _energies(A2, B2, alpha2, 2, noalloc=True)
    ref = _energies(A2, B2, alpha2, 2, noalloc=False)
    assert np.abs(small - ref).max() <= 1e-6 * np.abs(ref).max()


def test_noalloc_fits_problems_whose_w_output_would_not():
    """The energies-only epilogue writes no W, so a problem whose BF16 W
    (4 M Np bytes, 12 MB here) would overflow the 16 MiB array still runs."""
    M, N, K = 2000, 1500, 448
    A, B, alpha = _inputs(M, N, K, 5)
    ref = _energies(A, B, alpha, 2, noalloc=False)
    for _ in range(2):
        e = _energies(A, B, alpha, 2, noalloc=True)
        assert np.abs(e - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("M,N,K", [(1 << 62, 4, 8), (4, 1 << 62, 8), (4, 4, 1 << 62), (1 << 40, 1 << 30, 64)])
def test_noalloc_rejects_sizes_whose_products_overflow(M, N, K):
    """Sizes whose scratch products would wrap around 64 bits are rejected
    with the capacity error before any pointer is touched."""
    from librascal_b200 import _native as N_
    rc = N_.lib().rgpu_gap_energies_noalloc(M, N, K, 16, 16, 16, 2, 16, None)
    assert rc == N_.ERR_CAPACITY
    assert "scratch" in N_.lib().rgpu_last_error().decode()


def test_noalloc_rejects_sizes_beyond_scratch():
    from librascal_b200 import _native as N
    # 4 * M * Kp alone is 64 MiB here, above the 16 MiB of static scratch;
    # the size check comes before any pointer is touched
    rc = N.lib().rgpu_gap_energies_noalloc(16384, 256, 1024, 16, 16, 16, 2, 16, None)
    assert rc == N.ERR_CAPACITY
    assert "scratch" in N.lib().rgpu_last_error().decode()
