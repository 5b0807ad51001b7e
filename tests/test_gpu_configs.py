"""GPU parity at the shapes of the benchmark configurations, through the C ABI.

  * triclinic cells (4 species, r_c 5, n 8, l 6): FP64 features and
    power-spectrum gradients at 1e-10, GAP energies and forces with 200
    sparse points per species (FP64 at 1e-10, FP32 at 1e-4);
  * a bulk box of the 100 000-atom configuration's density and composition
    (2 species, r_c 6, n 12, l 9; the 16-register radial paths of the FP32
    kernels and the FP64 tiles that need fewer warps per block): FP64
    features at 1e-10 and FP32 features at 1e-5 on 2 000 atoms, GAP
    energies and forces on a 300-atom box;
  * the molecule-cluster model at its real size (4 000 sparse points, at
    least 500 per species, D = 6 720) on 50 clusters.

Bars as in test_gpu_parity.py; the FP32 ones are max|x - x_ref| / max|x_ref|
against the FP64 oracle.
"""
import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import synthetic
from oracle import oracle as O
from test_gpu_parity import assert_features_close, oracle_calc, soap

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def _model_from(sel_batch, kw, per_species, seed):
    """Sparse points picked at random from the oracle's features of
    sel_batch, weights ~ N(0, 1)."""
    species = np.unique(sel_batch["numbers"])
    r = O.Run(oracle_calc(**kw), sel_batch, species)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    sp_row = sel_batch["numbers"][ca]
    idx = synthetic.select_sparse_points(X, sp_row, per_species, seed=seed)
    alpha = np.random.default_rng(seed).normal(size=len(idx))
    return X[idx], sp_row[idx], alpha, species


def _gap_vs_oracle(eval_batch, kw, T, sps, alpha, species, fp32_tol=1e-4):
    r = O.Run(oracle_calc(**kw), eval_batch, species, gradients=True)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(eval_batch)
    E64, F64 = model.predict(st, "fp64")
    st.invalidate()
    E32, F32 = model.predict(st, "fp32")
    assert _rel(E64, E_ref) <= 1e-10
    assert _rel(F64, F_ref) <= 1e-10
    assert _rel(E32, E_ref) <= fp32_tol
    assert _rel(F32, F_ref) <= fp32_tol
    return _rel(F32, F_ref)


TRICLINIC = dict(rc=5.0, n=8, l=6, sigma=0.4)


def test_triclinic_fp64_features_and_gradients():
    batch = synthetic.triclinic_cells(n_struct=2, n_min=32, n_max=40, seed=21)
    species = np.array([1, 6, 7, 8])
    calc = soap(grads=True, **TRICLINIC)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    keys = calc.get_keys(species)
    X = al.get_features(calc, keys=keys)
    r = O.Run(oracle_calc(**TRICLINIC), batch, species, gradients=True)
    assert X.shape == (r.n_centers, r.D)
    assert_features_close(r.power_spectrum(), X)
    dX = al.get_features_gradient(calc, keys=keys)
    ref = r.power_spectrum_gradient().reshape(dX.shape)
    assert np.abs(dX - ref).max() <= 1e-10 * np.abs(ref).max()


def test_triclinic_gap_200_points_per_species():
    sel = synthetic.triclinic_cells(n_struct=6, n_min=150, n_max=220, seed=22)
    T, sps, alpha, species = _model_from(sel, TRICLINIC, 200, seed=3)
    assert len(T) == 800 and T.shape[1] == 4480
    ev = synthetic.triclinic_cells(n_struct=3, n_min=32, n_max=48, seed=23)
    _gap_vs_oracle(ev, TRICLINIC, T, sps, alpha, species)


BULK = dict(rc=6.0, n=12, l=9, sigma=0.5)


def test_bulk_shape_features():
    batch = synthetic.bulk_box(n_atoms=2000, seed=31)
    species = np.array([8, 14])
    r = O.Run(oracle_calc(**BULK), batch, species)
    Xo = r.power_spectrum()
    calc = soap(**BULK)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    X = al.get_features(calc, keys=calc.get_keys(species))
    assert X.shape == Xo.shape == (2000, 4320)
    assert_features_close(Xo, X)
    al32 = calc.transform(rb.AtomsList(rb.StructureSet(batch)), precision="fp32")
    X32 = al32.get_features(calc, keys=calc.get_keys(species))
    assert _rel(X32, Xo) <= 1e-5


def test_bulk_shape_gap():
    sel = synthetic.bulk_box(n_atoms=2000, seed=32)
    T, sps, alpha, species = _model_from(sel, BULK, {8: 260, 14: 140}, seed=4)
    ev = synthetic.bulk_box(n_atoms=300, seed=33)
    _gap_vs_oracle(ev, BULK, T, sps, alpha, species)


CLUSTERS = dict(rc=5.0, n=8, l=6, sigma=0.4)


def test_cluster_model_at_full_size():
    """4 000 sparse points (2 000 H, 500 each of C, N, O, F) over D = 6 720:
    the benchmark's model, on the first 50 of its clusters."""
    sel = synthetic.molecule_clusters(n_struct=330, seed=41)
    per = {1: 2000, 6: 500, 7: 500, 8: 500, 9: 500}
    T, sps, alpha, species = _model_from(sel, CLUSTERS, per, seed=5)
    assert len(T) == 4000 and T.shape[1] == 6720
    ev = synthetic.molecule_clusters(n_struct=50, seed=42)
    _gap_vs_oracle(ev, CLUSTERS, T, sps, alpha, species)


@pytest.mark.parametrize("l", [3, 7, 10, 12])
def test_fp32_gap_across_max_angular(l):
    """The FP32 path at max_angular values whose kernels live in different
    translation units of the library (each holds its own copy of the
    spherical-harmonics constants)."""
    kw = dict(rc=4.0, n=4, l=l, sigma=0.4)
    batch = synthetic.molecule_clusters(n_struct=6, seed=60 + l)
    T, sps, alpha, species = _model_from(batch, kw, 6, seed=l)
    _gap_vs_oracle(batch, kw, T, sps, alpha, species)
