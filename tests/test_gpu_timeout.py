"""Bounded device waits run out and the library stays usable.

The tcgen05 GEMMs wait on mbarriers for staged operands; each wait gives up
after a bounded number of polls, records where in a status word, and the
kernel winds down: the TMA copies and MMAs it already started are waited for
before its shared memory and TMEM are released. The test hook lowers the MMA
warp's limit to zero polls, so that wait runs out at once (nothing is
stuck: the limit is simply spent), and the call must return
RGPU_ERR_TIMEOUT. With the default restored, the next call on the same
context must succeed with correct results.
"""
import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import _native as N, synthetic
from test_gpu_parity import gap_setup, soap

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    import torch
    At = torch.as_tensor(A, dtype=torch.float32, device="cuda").contiguous()
    Bt = torch.as_tensor(B, dtype=torch.float32, device="cuda").contiguous()
    C = torch.zeros((A.shape[0], B.shape[0]), dtype=torch.float32, device="cuda")
    al = torch.zeros(B.shape[0], dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = N.lib().rgpu_debug_gemm_bf16x3(0, A.shape[0], B.shape[0], A.shape[1], At.data_ptr(), Bt.data_ptr(),
                                        al.data_ptr(), 2, C.data_ptr(), None, None)
    torch.cuda.synchronize()
    return rc, C.cpu().numpy().astype(np.float64)


def test_gemm_wait_runs_out_then_recovers():
    rng = np.random.default_rng(0)
    A = rng.random((128, 512))
    B = rng.normal(size=(256, 512))
    ref = np.float32(A).astype(np.float64) @ np.float32(B).astype(np.float64).T
    try:
        N.check(N.lib().rgpu_debug_set_gemm_wait_limit(0))
        rc, _ = _gemm(A, B)
        assert rc == N.ERR_TIMEOUT
        assert "gave up" in N.lib().rgpu_last_error().decode()
    finally:
        N.check(N.lib().rgpu_debug_set_gemm_wait_limit(-1))
    for _ in range(2):
        rc, C = _gemm(A, B)
        assert rc == 0
        assert np.abs(C - ref).max() <= 2e-4 * np.abs(ref).max()


def test_gap_predict_wait_runs_out_then_recovers():
    """The same through the persistent grouped GEMMs of the FP32 GAP path."""
    batch = synthetic.molecule_clusters(n_struct=6, seed=13)
    kw = dict(rc=5.0, n=8, l=6, sigma=0.4)
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=6)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(batch)
    E = np.zeros(len(E_ref))
    F = np.zeros(F_ref.shape)
    try:
        N.check(N.lib().rgpu_debug_set_gemm_wait_limit(0))
        rc = N.lib().rgpu_gap_predict(model.handle, st.handle, N.PRECISION_FP32, N.ptr(E, N.c_dbl_p),
                                      N.ptr(F, N.c_dbl_p))
        assert rc == N.ERR_TIMEOUT
    finally:
        N.check(N.lib().rgpu_debug_set_gemm_wait_limit(-1))
    st.invalidate()
    E, F = model.predict(st, "fp32")
    assert np.abs(E - E_ref).max() <= 1e-4 * np.abs(E_ref).max()
    assert np.abs(F - F_ref).max() <= 1e-4 * np.abs(F_ref).max()
