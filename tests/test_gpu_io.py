"""The reference's serialised GAP model (RadialScaling cutoff, direct GTO)
run end to end on the GPU, and the MD calculator, following
tests/python/md_calculator_test.py of the reference.

This fitted model's weights reach |alpha| ~ 650 and its energies (~0.03 eV)
are what is left of terms sum_m |alpha_m| k_im of order 1e4. The FP64 path
matches the oracle to 1e-9; the FP32 fast path computes each kernel value
to ~1e-6 relative, so its error is bounded relative to that term scale
(1e-5 of sum_i sum_m |alpha_m| k_im for energies, and of the sum of the
absolute products behind each force component), not to the energies and
forces themselves."""
import os

import numpy as np
import pytest

import librascal_b200 as rb
from helpers import GOLDEN, wrap
from librascal_b200 import io
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MODEL = os.path.join(GOLDEN, "simple_gap_model.json")
XYZ = os.path.join(GOLDEN, "methane_dimer_sample.xyz")


def oracle_for(krr, batch, scales=False):
    h = krr.get_representation_calculator()._get_init_params()
    calc = O.Calculator(h["interaction_cutoff"], h["cutoff_smooth_width"], h["max_radial"], h["max_angular"],
                        h["gaussian_sigma_constant"], spline=False, normalize=h["normalize"],
                        radial_scaling=h["cutoff_function_parameters"])
    species = krr.X_train.get_species()
    r = O.Run(calc, batch, species, gradients=True)
    T = krr.X_train.dense(species)
    sps, w, z = np.asarray(krr.X_train.species), krr.weights, krr.kernel.zeta
    out = r.gap_stress(sps, T, w, z)
    if not scales:
        return out
    # term scales: sum of |alpha_m k_im| per structure; per force component
    # the sum over pairs (i, j), points m and features d of
    # |alpha_m zeta k_im^(zeta-1) dX_i/dr_j[d] T_m[d]|
    ca, cs, po = r.centers()
    K = r.kernel_nm(sps, T, z, "Atom")
    S = np.zeros(r.n_struct)
    np.add.at(S, cs, np.abs(K) @ np.abs(w))
    X = r.power_spectrum()
    same = batch["numbers"][ca][:, None] == sps[None, :]
    Wc = np.where(same, np.abs(w)[None, :] * z * np.abs(X @ T.T) ** (z - 1), 0.)  # centre x point
    dX = r.power_spectrum_gradient()  # pair x 3 x D
    centre = np.repeat(np.arange(r.n_centers), np.diff(po))
    terms = np.einsum("pcd,md->pcm", np.abs(dX), np.abs(T))
    per_pair = np.einsum("pcm,pm->pc", terms, Wc[centre])
    SF = np.zeros((len(batch["numbers"]), 3))
    np.add.at(SF, r.pairs()["j"], per_pair)
    return out + (S, SF)


def methane_batch(n):
    frames = io.read_extxyz(XYZ, ":%d" % n)
    return frames, wrap(rb.frames_to_batch(frames))


def test_reference_model_predictions():
    krr = io.load_obj(MODEL)
    frames, batch = methane_batch(20)
    E_ref, F_ref, NS_ref, S, SF = oracle_for(krr, batch, scales=True)
    st = rb.StructureSet(batch)
    krr.precision = "fp64"
    E, F, NS = krr._gap().predict_stress(st, "fp64")
    assert np.abs(E - E_ref).max() <= 1e-9 * np.abs(E_ref).max()
    assert np.abs(F - F_ref).max() <= 1e-9 * np.abs(F_ref).max()
    assert np.abs(NS - NS_ref).max() <= 1e-9 * np.abs(NS_ref).max()
    E32, F32, _ = krr._gap().predict_stress(st, "fp32")
    assert np.all(np.abs(E32 - E_ref) <= 1e-5 * S)
    assert np.all(np.abs(F32 - F_ref) <= 1e-5 * SF + 1e-12)
    # the KRR methods give the same numbers
    krr.precision = "fp64"
    assert np.allclose(krr.predict(st), E_ref, rtol=0, atol=1e-9 * np.abs(E_ref).max())
    assert np.allclose(krr.predict_forces(st), F_ref, rtol=0, atol=1e-9 * np.abs(F_ref).max())
    # the model was fitted to these energies: its error is far below their spread
    y = np.array([f["info"]["energy"] for f in frames])
    assert np.sqrt(np.mean((E_ref - y) ** 2)) < 0.5 * np.std(y)


def test_md_calculator():
    calc = rb.GenericMDCalculator(MODEL, True, XYZ)
    frame = io.read_extxyz(XYZ, 0)
    # shift the positions to match the cell convention, as the reference's test does
    pos = frame["positions"] + np.diag(frame["cell"]) / 2.0
    cell = frame["cell"]
    e1, f1, s1 = calc.calculate(pos, cell)
    assert f1.shape == pos.shape and s1.shape == (3, 3)
    assert not (np.isnan(e1).any() or np.isnan(f1).any() or np.isnan(s1).any())
    e2, f2, s2 = calc.calculate(pos, cell)
    assert np.allclose(e1, e2) and np.allclose(f1, f2) and np.allclose(s1, s2)
    # against the oracle on the same (wrapped) structure
    batch = wrap(rb.frames_to_batch([dict(frame, positions=pos)]))
    E_ref, F_ref, NS_ref = oracle_for(io.load_obj(MODEL), batch)
    assert np.abs(e1 - E_ref).max() <= 1e-9 * np.abs(E_ref).max()
    assert np.abs(f1 - F_ref).max() <= 1e-9 * np.abs(F_ref).max()
    st = np.zeros((3, 3))
    st[tuple(zip(*rb.GenericMDCalculator.matrix_indices_in_voigt_notation))] = -NS_ref[0]
    st += np.triu(st).T
    assert np.abs(s1 - st).max() <= 1e-9 * np.abs(st).max()
    # a rigid shift (with periodic wrapping) leaves everything unchanged
    e3, f3, s3 = calc.calculate(pos + np.array([5.0, 5.0, 5.0]), cell)
    assert np.allclose(e3, e1, rtol=0, atol=1e-10) and np.allclose(f3, f1, rtol=0, atol=1e-10)
    assert np.allclose(s3, s1, rtol=0, atol=1e-10)
    # the same calculator from atomic numbers
    calc2 = rb.GenericMDCalculator(MODEL, True, atomic_numbers=frame["numbers"])
    e4, f4, s4 = calc2.calculate(pos, cell)
    assert np.allclose(e4, e1) and np.allclose(f4, f1) and np.allclose(s4, s1)
    # the fast path, within its bound relative to the term scales
    _, _, _, S, SF = oracle_for(io.load_obj(MODEL), batch, scales=True)
    calc3 = rb.GenericMDCalculator(MODEL, True, XYZ, precision="fp32")
    e5, f5, s5 = calc3.calculate(pos, cell)
    assert np.all(np.abs(e5 - e1) <= 1e-5 * S)
    assert np.all(np.abs(f5 - f1) <= 1e-5 * SF + 1e-12)
