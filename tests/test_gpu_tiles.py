"""Every launch shape the autotuner can choose gives the same FP32 results:
each candidate of each tile field, on the molecule-cluster shape (5
species, n 8, l 6) and on the bulk shape (2 species, n 12, l 9), against
the FP64 oracle at the FP32 bar (1e-4 of the largest value). A structure
energy sum_atoms sum_m alpha_m k^2 (|k| <= 1) can be a small remainder of
large terms of both signs (the single 300-atom box here: 12 from terms of
up to 7 000 in total); its bar is then 1e-6 of that total magnitude, the
size of the rounding of FP32 kernel values k (about 1e-7 relative) summed
over every (atom, sparse point) term."""
import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import synthetic, tune
from oracle import oracle as O
from test_gpu_parity import gap_setup, oracle_calc, soap

pytestmark = pytest.mark.gpu


def _case(batch, kw, n_sparse):
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=n_sparse)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    # total magnitude of a structure's energy terms: atoms x sum_m |alpha_m|
    scale = np.diff(batch["atom_offsets"]).max() * np.abs(alpha).sum()
    E_ref = (E_ref, scale)
    return model, E_ref, F_ref, (len(species), kw["n"], kw["l"])


def _check(model, batch, E_ref, F_ref, shape, cfg):
    E_ref, scale = E_ref
    old = tune.get_config(shape)
    try:
        tune.set_config(shape, cfg)
        st = rb.StructureSet(batch)
        st.use_graphs(False)
        E, F = model.predict(st, "fp32")
    finally:
        tune.set_config(shape, old)
    assert np.abs(E - E_ref).max() <= max(1e-4 * np.abs(E_ref).max(), 1e-6 * scale)
    assert np.abs(F - F_ref).max() <= 1e-4 * np.abs(F_ref).max()


@pytest.fixture(scope="module")
def clusters():
    batch = synthetic.molecule_clusters(n_struct=40, seed=51)
    return (batch,) + _case(batch, dict(rc=5.0, n=8, l=6, sigma=0.4), 40)


@pytest.mark.parametrize("field,value", [(f, v) for f in tune.FIELDS for v in tune.CANDIDATES[f]])
def test_cluster_shape_every_candidate(clusters, field, value):
    batch, model, E_ref, F_ref, shape = clusters
    _check(model, batch, E_ref, F_ref, shape, dict(tune.DEFAULT, **{field: value}))


@pytest.mark.parametrize("cfg", [dict(exp_chunk=32, exp_warps=8, gemm_variant=2, psb_threads=160),
                                 dict(exp_chunk=8, exp_warps=2, adj_threads=64, adj_blocks_per_sm=8,
                                      psf_threads=128, gemm_variant=1)])
def test_bulk_shape_extremes(cfg):
    batch = synthetic.bulk_box(n_atoms=300, seed=52)
    model, E_ref, F_ref, shape = _case(batch, dict(rc=6.0, n=12, l=9, sigma=0.5), 30)
    _check(model, batch, E_ref, F_ref, shape, dict(tune.DEFAULT, **cfg))


@pytest.mark.parametrize("which", ["clusters", "triclinic", "bulk"])
def test_tensor_core_power_spectrum_forward(which):
    """The tcgen05 power-spectrum forward (psf_tc = 1) at tiles of 3, 4 and
    5 centres (S n = 40, 32, 24), each batch ending in a partial tile."""
    if which == "clusters":
        batch, kw = synthetic.molecule_clusters(n_struct=23, seed=61), dict(rc=5.0, n=8, l=6, sigma=0.4)
    elif which == "triclinic":
        batch, kw = synthetic.triclinic_cells(n_struct=2, n_min=33, n_max=45, seed=62), dict(rc=5.0, n=8, l=6,
                                                                                             sigma=0.4)
    else:
        batch, kw = synthetic.bulk_box(n_atoms=301, seed=63), dict(rc=6.0, n=12, l=9, sigma=0.5)
    model, E_ref, F_ref, shape = _case(batch, kw, 20)
    _check(model, batch, E_ref, F_ref, shape, dict(tune.DEFAULT, psf_tc=1))


@pytest.mark.parametrize("species,n,l", [((1, 6, 8), 5, 3), ((1, 8), 7, 4), ((1, 6, 7, 8), 3, 5)])
def test_odd_radial_single_group(species, n, l):
    """Odd max_radial: every (species, n) channel shares one group of
    ceil(S n / 2) channel pairs, whose last pair is half padding when S n is
    odd (S n = 15, 14, 12 here). Features exported into the
    reference's column order and GAP energies and forces against the FP64
    oracle."""
    batch = synthetic.triclinic_cells(n_struct=3, n_min=30, n_max=44, species=species, seed=71)
    kw = dict(rc=5.0, n=n, l=l, sigma=0.4)
    calc = soap(**kw)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)), precision="fp32")
    sp = np.unique(batch["numbers"])
    X = al.get_features(calc, keys=calc.get_keys(sp))
    Xo = O.Run(oracle_calc(**kw), batch, sp).power_spectrum()
    assert X.shape == Xo.shape
    assert np.abs(X - Xo).max() <= 1e-5 * np.abs(Xo).max()
    model, E_ref, F_ref, shape = _case(batch, kw, 20)
    _check(model, batch, E_ref, F_ref, shape, dict(tune.DEFAULT))
