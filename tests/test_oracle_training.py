"""The oracle's sparse-kernel training matrices, checked the way the
reference checks its own (tests/test_sparse_kernels.cc:129-220) on the inputs
of reference_data/tests_only/sparse_kernel_inputs.json (tests/golden/
sparse_kernel_inputs.json):

* the K_NM gradient block against central differences of the summed K_NM
  energy rows (the reference's compute_numerical_kernel_gradients,
  models/numerical_kernel_gradients.hh:79-130), relative error below 1e-3
  with its relative_error convention;
* the gradient block times a weight vector against the GAP gradients of the
  prediction path, and its stress rows against the negative stress;
* K_NM and K_MM against their definitions, and the early return of
  compute_derivative for a structure without sparse-point species.
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, batch_from_frames, load_structures, relative_error, wrap
from oracle import oracle as O


def _cases():
    with open(os.path.join(GOLDEN, "sparse_kernel_inputs.json")) as f:
        return json.load(f)


def sparse_points_from_ids(r, batch, X, selected_ids):
    """Rows of the selected centres, grouped by species (species ascending,
    selection order inside a species) as SparsePointsBlockSparse stores
    them (models/sparse_points.hh:360-417)."""
    ca, cs, _ = r.centers()
    rows = []
    for s, ids in enumerate(selected_ids):
        first = int(np.flatnonzero(cs == s)[0])
        rows.extend(first + int(i) for i in ids)
    sps = batch["numbers"][ca[rows]]
    order = np.argsort(sps, kind="stable")
    rows = np.asarray(rows)[order]
    return X[rows], sps[order]


def case_setup(case):
    frames = load_structures()[case["structure"]][:case["n_structures"]]
    batch = batch_from_frames(frames)
    species = np.unique(batch["numbers"])
    calc = O.Calculator(case["cutoff"], case["smooth_width"], case["max_radial"], case["max_angular"],
                        case["sigma"], spline=case["spline"], normalize=case["normalize"])
    r = O.Run(calc, batch, species, gradients=True)
    X = r.power_spectrum()
    T, sps = sparse_points_from_ids(r, batch, X, case["selected_ids"])
    return calc, batch, species, r, T, sps


@pytest.mark.parametrize("i_case", range(6))
def test_kernel_gradient_block_vs_finite_differences(i_case):
    case = _cases()[i_case]
    calc, batch, species, r, T, sps = case_setup(case)
    zeta = case["zeta"]
    KD = r.kernel_nm_derivative(sps, T, zeta)
    assert KD.shape == (3 * r.n_centers, len(sps))
    h = case["h"]
    rng = np.random.default_rng(i_case)
    n_atoms = int(batch["atom_offsets"][-1])
    atoms = rng.choice(n_atoms, size=min(6, n_atoms), replace=False)
    for a in atoms:
        for c in range(3):
            k = []
            for sgn in (1, -1):
                b2 = {key: np.array(v, copy=True) for key, v in batch.items()}
                b2["positions"][a, c] += sgn * h
                b2 = wrap(b2)
                k.append(O.Run(calc, b2, species).kernel_nm(sps, T, zeta).sum(0))
            fd = (k[0] - k[1]) / (2 * h)
            # the analytic block is the reference argument, as in the reference's test
            err = relative_error(KD[3 * a + c], fd, epsilon=1e-14)
            assert err.max() < 1e-3, (a, c, err.max())


@pytest.mark.parametrize("i_case", [0, 2, 4])
def test_kernel_gradient_rows_times_weights(i_case):
    """KNM_der . w equals the gradients of the prediction path (the
    reference's second check, at a tighter bar) and the stress rows . w its
    negative stress."""
    case = _cases()[i_case]
    _, batch, _, r, T, sps = case_setup(case)
    zeta = case["zeta"]
    w = np.random.default_rng(1).normal(size=len(sps))
    KD = r.kernel_nm_derivative(sps, T, zeta, compute_neg_stress=True)
    E, F, NS = r.gap_stress(sps, T, w, zeta)
    g = KD[:3 * r.n_centers] @ w
    assert np.abs(g + F.reshape(-1)).max() <= 1e-10 * np.abs(F).max()
    ns = (KD[3 * r.n_centers:] @ w).reshape(-1, 6)
    assert np.abs(ns - NS).max() <= 1e-10 * np.abs(NS).max()
    # the energy rows . w are the energies
    K = r.kernel_nm(sps, T, zeta)
    assert np.abs(K @ w - E).max() <= 1e-12 * np.abs(E).max()


def test_kernel_nm_and_mm_definitions():
    case = _cases()[2]
    _, batch, _, r, T, sps = case_setup(case)
    X = r.power_spectrum()
    ca, cs, _ = r.centers()
    csp = batch["numbers"][ca]
    same = csp[:, None] == sps[None, :]
    ka = np.where(same, (X @ T.T) ** 2, 0.)
    assert np.abs(r.kernel_nm(sps, T, 2, "Atom") - ka).max() <= 1e-14
    ks = np.zeros((r.n_struct, len(sps)))
    np.add.at(ks, cs, ka)
    assert np.abs(r.kernel_nm(sps, T, 2) - ks).max() <= 1e-13
    kmm = O.kernel_mm(sps, T, 3)
    ref = np.where(sps[:, None] == sps[None, :], (T @ T.T) ** 3, 0.)
    assert np.abs(kmm - ref).max() <= 1e-14
    assert np.allclose(kmm, kmm.T, rtol=0, atol=1e-15)


def test_kernel_gradient_early_return():
    """A structure whose species have no sparse points ends the reference's
    loop over structures: it and every later structure keep zero rows."""
    frames = load_structures()["small_molecules-20.json:0:5"]
    batch = batch_from_frames(frames)
    species = np.unique(batch["numbers"])
    calc = O.Calculator(3.5, 0.5, 3, 3, 0.4, spline=False)
    r = O.Run(calc, batch, species, gradients=True)
    X = r.power_spectrum()
    ca, cs, _ = r.centers()
    z = batch["numbers"][ca]
    # sparse points of one species only, absent from some structure
    counts = [set(z[cs == s]) for s in range(r.n_struct)]
    target = None
    for sp in species:
        miss = [s for s in range(r.n_struct) if sp not in counts[s]]
        if miss and miss[0] > 0:
            target, first_missing = int(sp), miss[0]
            break
    assert target is not None
    rows = np.flatnonzero(z == target)[:3]
    T, sps = X[rows], z[rows]
    KD = r.kernel_nm_derivative(sps, T, 2, compute_neg_stress=True)
    off = batch["atom_offsets"]
    assert np.any(KD[:3 * off[first_missing]] != 0)
    assert np.all(KD[3 * off[first_missing]:3 * r.n_centers] == 0)
    assert np.all(KD[3 * r.n_centers + 6 * first_missing:] == 0)
