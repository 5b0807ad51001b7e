"""GPU parity of the sparse-kernel training matrices against the oracle,
through the C ABI (rgpu_sparse_kernel, rgpu_sparse_kernel_derivative,
rgpu_sparse_kernel_mm): K_NM energy rows (targets Structure and Atom), the
K_NM gradient block with its negative-stress rows, and K_MM, all FP64 with a
bar of 1e-10 of the largest value of each block. Also the reference's
sparse-kernel test inputs, compute_KNM and train_gap_model end to end.
"""
import json
import os

import numpy as np
import pytest

import librascal_b200 as rb
from helpers import GOLDEN, batch_from_frames, load_structures
from librascal_b200 import synthetic
from oracle import oracle as O
from test_gpu_parity import gap_setup, oracle_calc, soap
from test_oracle_training import sparse_points_from_ids

pytestmark = pytest.mark.gpu


def close(test, ref, tol=1e-10):
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(test - ref).max() <= tol * scale


def gpu_kernels(calc, batch, sps, T, species, zeta=2):
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    assert list(sp.species) == list(sps)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    ks = rb.Kernel(calc, name="GAP", zeta=zeta, target_type="Structure", kernel_type="Sparse")
    ka = rb.Kernel(calc, name="GAP", zeta=zeta, target_type="Atom", kernel_type="Sparse")
    return dict(K=ks(al, sp), Ka=ka(al, sp), KD=ks(al, sp, grad=(True, False), compute_neg_stress=True),
                KD0=ks(al, sp, grad=(True, False)), KMM=ks(sp))


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters"])
def test_sparse_kernel_matrices_parity(which):
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=2, seed=2), dict(rc=4.0, n=6, l=4, sigma=0.3)
    else:
        batch, kw = synthetic.molecule_clusters(n_struct=12, seed=5), dict(rc=5.0, n=8, l=6, sigma=0.4)
    r, T, sps, _, species = gap_setup(batch, kw, n_sparse=6)
    g = gpu_kernels(soap(**kw), batch, sps, T, species)
    nc = r.n_centers
    assert close(g["K"], r.kernel_nm(sps, T, 2))
    assert close(g["Ka"], r.kernel_nm(sps, T, 2, "Atom"))
    KD = r.kernel_nm_derivative(sps, T, 2, compute_neg_stress=True)
    assert g["KD"].shape == KD.shape
    assert close(g["KD"][:3 * nc], KD[:3 * nc])
    assert close(g["KD"][3 * nc:], KD[3 * nc:])
    assert np.array_equal(g["KD0"].shape, (3 * nc, len(sps)))
    assert close(g["KD0"], KD[:3 * nc])
    assert close(g["KMM"], O.kernel_mm(sps, T, 2), 1e-12)


@pytest.mark.parametrize("i_case", range(6))
def test_sparse_kernel_gradient_reference_inputs(i_case):
    """The reference's sparse-kernel gradient inputs (direct GTO, normalised
    and not): the GPU gradient block against the oracle's, which the CPU
    tests check against finite differences."""
    with open(os.path.join(GOLDEN, "sparse_kernel_inputs.json")) as f:
        case = json.load(f)[i_case]
    frames = load_structures()[case["structure"]][:case["n_structures"]]
    batch = batch_from_frames(frames)
    batch.pop("center_atoms_mask")
    species = np.unique(batch["numbers"])
    kw = dict(rc=case["cutoff"], sw=case["smooth_width"], n=case["max_radial"], l=case["max_angular"],
              sigma=case["sigma"], spline=case["spline"], normalize=case["normalize"])
    oc = oracle_calc(**kw)
    r = O.Run(oc, batch, species, gradients=True)
    X = r.power_spectrum()
    T, sps = sparse_points_from_ids(r, batch, X, case["selected_ids"])
    g = gpu_kernels(soap(grads=True, **kw), batch, sps, T, species, case["zeta"])
    KD = r.kernel_nm_derivative(sps, T, case["zeta"], compute_neg_stress=True)
    nc = r.n_centers
    assert close(g["KD"][:3 * nc], KD[:3 * nc])
    assert close(g["KD"][3 * nc:], KD[3 * nc:])
    assert close(g["K"], r.kernel_nm(sps, T, case["zeta"]))


def test_sparse_kernel_gradient_early_return():
    """A structure without sparse-point species ends the computation: it and
    every later structure keep zero rows, on the GPU as in the reference."""
    batch = synthetic.molecule_clusters(n_struct=6, seed=3)
    kw = dict(rc=5.0, n=4, l=3, sigma=0.4)
    # make structure 2 hydrogen-only and take sparse points of carbon only
    off = batch["atom_offsets"]
    batch["numbers"] = batch["numbers"].copy()
    batch["numbers"][off[2]:off[3]] = 1
    species = np.unique(batch["numbers"])
    r = O.Run(oracle_calc(**kw), batch, species, gradients=True)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    z = batch["numbers"][ca]
    rows = np.flatnonzero(z == 6)[:3]
    T, sps = X[rows], z[rows]
    g = gpu_kernels(soap(**kw), batch, sps, T, species)
    KD = r.kernel_nm_derivative(sps, T, 2, compute_neg_stress=True)
    nc = r.n_centers
    assert np.all(g["KD"][3 * off[2]:3 * nc] == 0) and np.all(g["KD"][3 * nc + 12:] == 0)
    assert np.any(g["KD"][:3 * off[2]] != 0)
    assert close(g["KD"], KD)


def test_compute_knm_and_train_gap_model():
    """compute_KNM stacks energy rows over gradient rows; train_gap_model on
    it gives the weights of the same fit done with the oracle's matrices,
    and the trained model predicts through the GPU path."""
    batch = synthetic.molecule_clusters(n_struct=10, seed=7)
    kw = dict(rc=5.0, n=6, l=4, sigma=0.4)
    r, T, sps, _, species = gap_setup(batch, kw, n_sparse=5, seed=1)
    off = batch["atom_offsets"]
    frames = [dict(positions=batch["positions"][off[i]:off[i + 1]], numbers=batch["numbers"][off[i]:off[i + 1]],
                   cell=batch["cells"][i], pbc=batch["pbc"][i]) for i in range(len(off) - 1)]
    calc = soap(grads=True, **kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    kernel = rb.Kernel(calc, name="GAP", zeta=2, target_type="Structure", kernel_type="Sparse")
    KNM = rb.compute_KNM(frames, sp, kernel, calc)
    ref = np.vstack([r.kernel_nm(sps, T, 2), r.kernel_nm_derivative(sps, T, 2)])
    assert close(KNM, ref)
    # synthetic targets from a known model
    w_true = np.random.default_rng(3).normal(size=len(sps))
    sc = {int(z): -0.5 * z for z in species}
    E, F = r.gap(sps, T, w_true, 2)
    y = E + np.array([sum(sc[int(z)] for z in batch["numbers"][off[i]:off[i + 1]]) for i in range(len(off) - 1)])
    model = rb.train_gap_model(kernel, frames, KNM, sp, y, sc, grad_train=-F, lambdas=[1e-6, 1e-6], jitter=1e-10)
    model_ref = rb.train_gap_model(kernel, frames, ref, sp, y, sc, grad_train=-F, lambdas=[1e-6, 1e-6],
                                   jitter=1e-10)
    assert np.abs(model.weights - model_ref.weights).max() <= 1e-6 * np.abs(model_ref.weights).max()
    E_fit = model.predict(rb.StructureSet(batch))
    assert np.abs(E_fit - y).max() <= 1e-4 * np.abs(y).max()
