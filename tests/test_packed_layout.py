"""The packed column layout of the FP32 path, through the C ABI's host-only
test hook (no GPU).

The FP32 path stores each centre's power-spectrum row as the upper triangles
of the per-l Gram matrices of its coefficients in 2 x 2 tiles, grouped into
segments by the species of their rows and columns: the two equal
same-species features p(n1 n2 l) and p(n2 n1 l) of the reference's row
(calculator_spherical_invariants.hh:747-794) share one column. Packing must
keep every quantity the GAP path takes from a row: its norm and its dot
product with a sparse point packed the same way; the FP32 feature export
must give the reference's row back.
"""
import ctypes

import numpy as np
import pytest

from librascal_b200 import _native as N


def reference_row(rng, S, n, L):
    """Power-spectrum row in the reference's dense order
    ((key*n + n1)*n + n2)*(L+1) + l from random coefficients."""
    L1 = L + 1
    C = [rng.normal(size=(S * n, 2 * l + 1)) for l in range(L1)]
    P = S * (S + 1) // 2
    row = np.zeros(P * n * n * L1)
    key = 0
    for a in range(S):
        for b in range(a, S):
            s = np.sqrt(2.0) if a < b else 1.0
            for l in range(L1):
                G = C[l] @ C[l].T / np.sqrt(2 * l + 1)
                blk = G[a * n:(a + 1) * n, b * n:(b + 1) * n] * s
                for n1 in range(n):
                    for n2 in range(n):
                        row[((key * n + n1) * n + n2) * L1 + l] = blk[n1, n2]
            key += 1
    return row


def sizes(S, n, L):
    D, Dg = ctypes.c_int64(), ctypes.c_int64()
    N.check(N.lib().rgpu_debug_packed_layout(S, n, L, ctypes.byref(D), ctypes.byref(Dg), None, None, None))
    return D.value, Dg.value


def pack(S, n, L, ref):
    D, Dg = sizes(S, n, L)
    ref = np.ascontiguousarray(ref, np.float64)
    assert ref.size == D
    packed = np.zeros(Dg)
    unpacked = np.zeros(D)
    N.check(N.lib().rgpu_debug_packed_layout(S, n, L, None, None, N.ptr(ref, N.c_dbl_p), N.ptr(packed, N.c_dbl_p),
                                             N.ptr(unpacked, N.c_dbl_p)))
    return packed, unpacked


def test_benchmark_shape_sizes():
    # 5 species, n 8, l 6: 6 720 reference columns; 5 same-species segments
    # of 7 x 10 tiles (280 columns, padded to 288) and 10 cross-species
    # segments of 7 x 16 tiles (448 columns)
    assert sizes(5, 8, 6) == (6720, 5 * 288 + 10 * 448)
    # 2 species, n 12, l 9: 2 segments of 10 x 21 tiles (840, padded to 864)
    # and one of 10 x 36 (1 440)
    assert sizes(2, 12, 9) == (4320, 2 * 864 + 1440)
    # odd n: one segment holding the whole triangle (3 x 6 tiles, 72 columns,
    # padded to 96)
    assert sizes(2, 3, 2) == (3 * 9 * 3, 96)


@pytest.mark.parametrize("S,n,L", [(1, 3, 2), (2, 3, 1), (3, 3, 2), (2, 4, 3), (5, 8, 6)])
def test_norm_dot_and_export_survive_packing(S, n, L):
    rng = np.random.default_rng(S * 100 + n * 10 + L)
    p = reference_row(rng, S, n, L)
    t = rng.normal(size=p.size)  # a sparse point need not be symmetric
    xp, back = pack(S, n, L, p)
    tp, _ = pack(S, n, L, t)
    assert np.isclose(np.dot(xp, xp), np.dot(p, p), rtol=1e-12)
    assert np.isclose(np.dot(xp, tp), np.dot(p, t), rtol=1e-12, atol=1e-12 * np.abs(p).max() * np.abs(t).max())
    # the export goes through FP32
    assert np.abs(back - p).max() <= 1e-6 * np.abs(p).max()
    # fewer columns than the reference's row holds
    assert np.count_nonzero(xp) < p.size


def test_bad_shape_is_rejected():
    D = ctypes.c_int64()
    assert N.lib().rgpu_debug_packed_layout(0, 8, 6, ctypes.byref(D), None, None, None, None) != 0
