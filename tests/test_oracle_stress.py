"""The oracle's negative stress (the reference's compute_sparse_kernel_neg_stress,
models/sparse_kernel_predict.hh:291-377) against central differences of the
energy under the reference's strain displacement
(structure_managers/atomic_structure.hh:161-171: shift(a, b) += h applied to
the cell and, through the scaled coordinates, to the positions).

With r'_b = r_b + h r_a for every pair vector, V * neg_stress of the Voigt
entry (a, b) is -dE/dh; the entries are xx, yy, zz, yz (r_y g_z),
xz (r_z g_x), xy (r_x g_y).
"""
import numpy as np

from oracle import oracle as O
from librascal_b200 import synthetic

VOIGT = [(0, 0), (1, 1), (2, 2), (1, 2), (2, 0), (0, 1)]


def _strained(batch, a, b, h):
    out = {k: np.array(v, copy=True) for k, v in batch.items()}
    M = np.eye(3)
    M[b, a] += h
    out["positions"] = out["positions"] @ M.T
    out["cells"] = np.einsum("sij,kj->sik", out["cells"], M)  # rows are lattice vectors
    return out


def test_neg_stress_matches_strain_derivative():
    batch = synthetic.periodic_boxes(n_struct=1, seed=2)
    species = sorted(set(int(z) for z in batch["numbers"]))
    calc = O.Calculator(4.0, 0.5, 6, 4, 0.3)
    r = O.Run(calc, batch, species, gradients=True)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    sp_row = batch["numbers"][ca]
    idx = synthetic.select_sparse_points(X, sp_row, 5, seed=0)
    alpha = np.random.default_rng(0).normal(size=len(idx))
    T, sps = X[idx], sp_row[idx]
    E, F, NS = r.gap_stress(sps, T, alpha, 2)
    E2, F2 = r.gap(sps, T, alpha, 2)
    assert np.array_equal(E, E2) and np.array_equal(F, F2)
    V = abs(np.linalg.det(batch["cells"][0]))
    h = 1e-5
    fd = np.zeros(6)
    for k, (a, b) in enumerate(VOIGT):
        ep = O.Run(calc, _strained(batch, a, b, h), species).gap(sps, T, alpha, 2, forces=False)[0]
        em = O.Run(calc, _strained(batch, a, b, -h), species).gap(sps, T, alpha, 2, forces=False)[0]
        fd[k] = -(ep - em) / (2 * h) / V
    assert np.abs(fd - NS[0]).max() <= 1e-4 * np.abs(NS[0]).max()
