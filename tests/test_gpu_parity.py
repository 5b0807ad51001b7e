"""GPU parity against the CPU oracle, through the C ABI.

Bars:
  * neighbour list: identical pairs, order, shifts, distances and directions
    (bit-exact; the oracle fixes the FP association, no FMA);
  * plain FP64 features and gradients: <= 1e-10 in the reference's
    relative_error convention (math/utils.hh:152-225);
  * plain FP64 GAP energies/forces: <= 1e-10 relative;
  * fast FP32/TF32 adjoint forces: max|F - F_ref| / max|F_ref| <= 1e-4.
"""
import json
import os

import numpy as np
import pytest

import librascal_b200 as rb
from helpers import GOLDEN, batch_from_frames, load_structures, relative_error, wrap
from librascal_b200 import synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def soap(rc=3.5, sw=0.5, n=4, l=3, sigma=0.4, spline=True, grads=False, normalize=True, rs=None):
    """rs: None for the shifted cosine, or dict(rate, scale, exponent) for
    the RadialScaling cutoff."""
    opt = dict(Spline=dict(accuracy=1e-8)) if spline else {}
    cut = dict(cutoff_function_type="RadialScaling", cutoff_function_parameters=dict(rs)) if rs else {}
    return rb.SphericalInvariants(interaction_cutoff=rc, cutoff_smooth_width=sw, max_radial=n,
                                  max_angular=l, gaussian_sigma_type="Constant",
                                  gaussian_sigma_constant=sigma, optimization=opt,
                                  compute_gradients=grads, normalize=normalize, **cut)


def oracle_calc(rc=3.5, sw=0.5, n=4, l=3, sigma=0.4, spline=True, normalize=True, rs=None):
    return O.Calculator(rc, sw, n, l, sigma, spline=spline, normalize=normalize,
                        accuracy=1e-8 if spline else 1e-8, radial_scaling=rs)


def subset(batch, idx):
    off = batch["atom_offsets"]
    parts = dict(positions=[], numbers=[], cells=[], pbc=[])
    new_off = [0]
    for i in idx:
        a0, a1 = off[i], off[i + 1]
        parts["positions"].append(batch["positions"][a0:a1])
        parts["numbers"].append(batch["numbers"][a0:a1])
        parts["cells"].append(batch["cells"][i])
        parts["pbc"].append(batch["pbc"][i])
        new_off.append(new_off[-1] + a1 - a0)
    return dict(atom_offsets=np.asarray(new_off, np.int64), positions=np.concatenate(parts["positions"]),
                numbers=np.concatenate(parts["numbers"]), cells=np.asarray(parts["cells"]),
                pbc=np.asarray(parts["pbc"]))


def nl_cases():
    structs = load_structures()
    cases = []
    for name, rcs in [("CaCrP2O7_mvc-11955_symmetrized.json", [2.0, 3.0, 5.5]),
                      ("small_molecule.json", [2.0, 3.5]),
                      ("simple_cubic_8.json", [1.0, 2.5]),
                      ("linked_cell_break_0.json", [3.0]),
                      ("diamond_cubic_distorted.json", [5.0]),
                      ("SiC_moissanite.json", [4.0]),
                      ("methane.json", [3.0])]:
        if name in structs:
            for rc in rcs:
                cases.append((name, batch_from_frames(structs[name]), rc))
    cases.append(("periodic_boxes", synthetic.periodic_boxes(n_struct=4), 4.0))
    cases.append(("triclinic_cells", subset(synthetic.triclinic_cells(n_struct=8), range(8)), 5.0))
    cases.append(("molecule_clusters", synthetic.molecule_clusters(n_struct=64), 5.0))
    return cases


@pytest.mark.parametrize("case", nl_cases(), ids=lambda c: "%s-rc%s" % (c[0], c[2]))
def test_neighbour_list_bit_exact(case):
    name, batch, rc = case
    st = rb.StructureSet(batch)
    st.build_neighbour_list(rc)
    g = st.neighbour_list()
    species = np.unique(batch["numbers"])
    r = O.Run(oracle_calc(rc=rc), batch, species)
    ca, cs, po = r.centers()
    p = r.pairs()
    assert np.array_equal(g["center_atom"], ca)
    assert np.array_equal(g["pair_offsets"], po)
    assert np.array_equal(g["j"], p["j"])
    assert np.array_equal(g["shift"], p["shift"])
    assert np.array_equal(g["distance"], p["distance"])  # bitwise
    assert np.array_equal(g["direction"], p["direction"])


def test_neighbour_list_center_mask():
    structs = load_structures()
    frames = [dict(f) for f in structs["CaCrP2O7_mvc-11955_symmetrized.json"]]
    n = len(frames[0]["numbers"])
    frames[0]["center_atoms_mask"] = [i % 3 != 1 for i in range(n)]
    batch = batch_from_frames(frames)
    st = rb.StructureSet(batch)
    st.build_neighbour_list(3.0)
    g = st.neighbour_list()
    r = O.Run(oracle_calc(rc=3.0), batch, np.unique(batch["numbers"]))
    ca, cs, po = r.centers()
    p = r.pairs()
    assert np.array_equal(g["center_atom"], ca)
    assert np.array_equal(g["j"], p["j"]) and np.array_equal(g["distance"], p["distance"])


def test_rc_epsilon_edge_case():
    # Twelve atoms, six at distance rc and six at rc - 2 eps from the
    # centre; pairs exactly at rc are kept (d^2 <= rc^2).
    rc, eps = 3.0, 1e-6
    pos = [[0, 0, 0]]
    for k, d in enumerate([rc] * 3 + [rc - 2 * eps] * 3):
        v = np.zeros(3)
        v[k % 3] = d if k < 3 else -d
        pos.append(v)
    pos = np.asarray(pos, float) + 10.0
    batch = batch_from_frames([dict(positions=pos, numbers=[1] * len(pos), cell=np.eye(3) * 20.,
                                    pbc=[False] * 3)])
    st = rb.StructureSet(batch)
    st.build_neighbour_list(rc)
    g = st.neighbour_list()
    r = O.Run(oracle_calc(rc=rc), batch, [1])
    assert np.array_equal(g["j"], r.pairs()["j"])
    assert g["pair_offsets"][1] - g["pair_offsets"][0] == 1 + 6


def test_invalid_structures_raise():
    good = dict(positions=[[1., 1., 1.], [2., 1., 1.]], numbers=[1, 1], cell=np.eye(3) * 5., pbc=[True] * 3)
    bad = dict(good, positions=[[1., 1., 1.], [6., 1., 1.]])
    with pytest.raises(RuntimeError, match="inside the unit cell"):
        st = rb.StructureSet(batch_from_frames([good, bad]))
        st.build_neighbour_list(3.0)
    zero = dict(good, cell=np.zeros((3, 3)))
    with pytest.raises(RuntimeError, match="filled with zeros"):
        st = rb.StructureSet(batch_from_frames([zero]))
        st.build_neighbour_list(3.0)
    badz = dict(good, numbers=[1, 200])
    with pytest.raises(RuntimeError, match="range"):
        rb.StructureSet(batch_from_frames([badz]))


def features_vs_oracle(batch, calc_kwargs, species=None):
    calc = soap(**calc_kwargs)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    species = np.unique(batch["numbers"]) if species is None else species
    keys = calc.get_keys(species)
    X = al.get_features(calc, keys=keys)
    oc = oracle_calc(**{k: v for k, v in calc_kwargs.items() if k != "grads"})
    r = O.Run(oc, batch, species)
    return X, r.power_spectrum(), al, calc, r


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters", "CaCrP2O7"])
def test_powerspectrum_fp64_parity(which):
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=4), dict(rc=4.0, n=6, l=4, sigma=0.3)
    elif which == "molecule_clusters":
        batch, kw = synthetic.molecule_clusters(n_struct=40), dict(rc=5.0, n=8, l=6, sigma=0.4)
    else:
        batch = batch_from_frames(load_structures()["CaCrP2O7_mvc-11955_symmetrized.json"])
        kw = dict(rc=5.0, n=6, l=5, sigma=0.3)
    X, Xo, *_ = features_vs_oracle(batch, kw)
    assert X.shape == Xo.shape
    assert_features_close(Xo, X)


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters"])
def test_powerspectrum_fp32_features(which):
    """FP32 fast-path features, exported back into the reference's key and
    column order, within FP32 rounding of the FP64 oracle."""
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=3, seed=4), dict(rc=4.0, n=6, l=4, sigma=0.3)
    else:
        batch, kw = synthetic.molecule_clusters(n_struct=30, seed=3), dict(rc=5.0, n=8, l=6, sigma=0.4)
    calc = soap(**kw)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)), precision="fp32")
    species = np.unique(batch["numbers"])
    X = al.get_features(calc, keys=calc.get_keys(species))
    Xo = O.Run(oracle_calc(**kw), batch, species).power_spectrum()
    assert X.shape == Xo.shape
    assert np.abs(X - Xo).max() <= 1e-5 * np.abs(Xo).max()


def assert_features_close(ref, test, rel=1e-10):
    """<= 1e-10 relative on every entry above 1e-6 of its row maximum; below
    that, entries are sums over m that cancel to ~1e-9 of the row scale, so an
    ulp of any input (cos, hypot, the spline) moves them by ~1e-10 relative:
    there the bar is 1e-14 of the row maximum, absolute."""
    scale = np.abs(ref).max(axis=1, keepdims=True)
    scale = np.where(scale > 0, scale, 1.0)
    d = np.abs(test - ref)
    big = np.abs(ref) > 1e-6 * scale
    assert (d[big] / np.abs(ref[big])).max(initial=0.0) <= rel
    assert (d / scale).max() <= 1e-14


def test_expansion_golden_on_gpu():
    z = np.load(os.path.join(GOLDEN, "expansion_reference.npz"))
    meta = json.loads(str(z["meta"]))
    structs = load_structures()
    for i, m in enumerate(meta):
        batch = batch_from_frames(structs[m["structure"]])
        opt = dict(Spline=dict(accuracy=m["accuracy"])) if m["spline"] else {}
        rs = m["radial_scaling"]
        cut = dict(cutoff_function_type="RadialScaling", cutoff_function_parameters=dict(rs)) if rs else {}
        calc = rb.SphericalExpansion(interaction_cutoff=m["cutoff"], cutoff_smooth_width=m["smooth_width"],
                                     max_radial=m["max_radial"], max_angular=m["max_angular"],
                                     gaussian_sigma_type="Constant", gaussian_sigma_constant=m["sigma"],
                                     optimization=opt, **cut)
        al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
        C = al.get_features(calc, keys=calc.get_keys(np.unique(batch["numbers"])))
        ref = z["features_%d" % i]
        assert relative_error(ref, C, 1e-14).max() < 3e-6  # tests/test_calculator.cc:460-496


def test_kernel_golden_on_gpu():
    z = np.load(os.path.join(GOLDEN, "kernel_reference.npz"))
    meta = json.loads(str(z["meta"]))
    batch = batch_from_frames(load_structures()[str(z["structures"])])
    S = len(batch["atom_offsets"]) - 1
    for i, m in enumerate(meta):
        calc = soap(rc=m["cutoff"], sw=m["smooth_width"], n=m["max_radial"], l=m["max_angular"],
                    sigma=m["sigma"], spline=m["spline"], normalize=m["normalize"])
        al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
        X = al.get_features(calc, keys=calc.get_keys(np.unique(batch["numbers"])))
        info = al.get_representation_info()
        kk = (X @ X.T) ** m["zeta"]
        if m["target_type"] == "Structure":
            K = np.array([[kk[np.ix_(info[:, 0] == a, info[:, 0] == c)].mean() for c in range(S)]
                          for a in range(S)])
        else:
            K = kk
        assert relative_error(z["kernel_%d" % i], K).max() < 1e-10  # tests/test_kernels.cc:68-136


def test_powerspectrum_gradient_fp64_parity():
    batch = synthetic.molecule_clusters(n_struct=6, seed=3)
    kw = dict(rc=5.0, n=4, l=3, sigma=0.4)
    calc = soap(grads=True, **kw)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    species = np.unique(batch["numbers"])
    keys = calc.get_keys(species)
    dX = al.get_features_gradient(calc, keys=keys)
    r = O.Run(oracle_calc(**kw), batch, species, gradients=True)
    ref = r.power_spectrum_gradient().reshape(dX.shape)
    scale = np.abs(ref).max()
    assert np.abs(dX - ref).max() <= 1e-10 * scale
    info = al.get_gradients_info()
    assert info.shape == (r.n_pairs, 5)


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters"])
def test_expansion_gradient_fp64_parity(which):
    """Dense spherical-expansion gradients (3 rows per pair, self pairs
    included; a pair carries only its neighbour's species key, the self pair
    every key) against the oracle's restatement of
    calculator_spherical_expansion.hh:2327-2366."""
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=2, seed=4), dict(rc=4.0, n=6, l=4, sigma=0.3)
    else:
        batch, kw = synthetic.molecule_clusters(n_struct=6, seed=3), dict(rc=5.0, n=4, l=3, sigma=0.4)
    calc = rb.SphericalExpansion(interaction_cutoff=kw["rc"], cutoff_smooth_width=0.5, max_radial=kw["n"],
                                 max_angular=kw["l"], gaussian_sigma_type="Constant",
                                 gaussian_sigma_constant=kw["sigma"],
                                 optimization=dict(Spline=dict(accuracy=1e-8)), compute_gradients=True)
    al = calc.transform(rb.AtomsList(rb.StructureSet(batch)))
    species = np.unique(batch["numbers"])
    dC = al.get_features_gradient(calc, keys=calc.get_keys(species))
    r = O.Run(oracle_calc(**kw), batch, species, gradients=True)
    ref = r.expansion_gradient()                       # (pairs, S, 3, n, K)
    ref = np.transpose(ref, (0, 2, 1, 3, 4)).reshape(dC.shape)
    assert np.abs(dC - ref).max() <= 1e-10 * np.abs(ref).max()
    C = al.get_features(calc, keys=calc.get_keys(species))
    C_ref = r.expansion().reshape(C.shape)
    assert_features_close(C_ref, C)
    # FP32 expansion rows (padded l-blocks on the device) exported in the same layout
    al32 = calc.transform(rb.AtomsList(rb.StructureSet(batch)), precision="fp32")
    C32 = al32.get_features(calc, keys=calc.get_keys(species))
    assert np.abs(C32 - C_ref).max() <= 1e-5 * np.abs(C_ref).max()


def gap_setup(batch, kw, n_sparse=6, seed=0, zeta=2):
    species = np.unique(batch["numbers"])
    oc = oracle_calc(**kw)
    r = O.Run(oc, batch, species, gradients=True)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    sp_row = batch["numbers"][ca]
    idx = synthetic.select_sparse_points(X, sp_row, n_sparse, seed=seed)
    rng = np.random.default_rng(seed)
    alpha = rng.normal(size=len(idx))
    return r, X[idx], sp_row[idx], alpha, species


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gap_energy_forces_parity(precision):
    batch = synthetic.molecule_clusters(n_struct=12, seed=5)
    kw = dict(rc=5.0, n=8, l=6, sigma=0.4)
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=8)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(batch)
    E, F = model.predict(st, precision)
    if precision == "fp64":
        assert np.abs(E - E_ref).max() <= 1e-10 * np.abs(E_ref).max()
        assert np.abs(F - F_ref).max() <= 1e-10 * np.abs(F_ref).max()
    else:
        # energies are sums of alpha_m k^2 with alpha ~ N(0, 1): the FP32 /
        # BF16x3 error is reported relative to the largest energy
        assert np.abs(E - E_ref).max() <= 1e-4 * np.abs(E_ref).max()
        assert np.abs(F - F_ref).max() <= 1e-4 * np.abs(F_ref).max()


def test_gap_forces_periodic_and_fd():
    batch = synthetic.periodic_boxes(n_struct=2, seed=2)
    kw = dict(rc=4.0, n=6, l=4, sigma=0.3)
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=5)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(batch)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-4)]:
        E, F = model.predict(st, prec)
        assert np.abs(F - F_ref).max() <= tol * np.abs(F_ref).max(), prec
    # central finite differences of the GPU FP64 energy (h = 1e-4 A)
    h = 1e-4
    rng = np.random.default_rng(0)
    for a in rng.choice(batch["atom_offsets"][-1], 4, replace=False):
        for c in range(3):
            ep = []
            for sgn in (1, -1):
                b2 = dict(batch)
                b2["positions"] = batch["positions"].copy()
                b2["positions"][a, c] += sgn * h
                b2 = wrap(b2)
                st2 = rb.StructureSet(b2)
                ep.append(model.predict(st2, "fp64", forces=False)[0].sum())
            fd = -(ep[0] - ep[1]) / (2 * h)
            assert abs(fd - F_ref[a, c]) <= 1e-6 * max(1.0, np.abs(F_ref).max())


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters"])
def test_gap_neg_stress_parity(which):
    """Negative stress per structure (Voigt xx, yy, zz, yz, xz, xy) of both
    GPU paths against the oracle's compute_sparse_kernel_neg_stress
    restatement; KRR.predict_stress returns its negative."""
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=2, seed=2), dict(rc=4.0, n=6, l=4, sigma=0.3)
    else:
        batch, kw = synthetic.molecule_clusters(n_struct=12, seed=5), dict(rc=5.0, n=8, l=6, sigma=0.4)
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=6)
    E_ref, F_ref, NS_ref = r.gap_stress(sps, T, alpha, 2)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(batch)
    scale = np.abs(NS_ref).max()
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-4)]:
        E, F, NS = model.predict_stress(st, prec)
        assert NS.shape == NS_ref.shape
        assert np.abs(NS - NS_ref).max() <= tol * scale, prec
        assert np.abs(F - F_ref).max() <= tol * np.abs(F_ref).max(), prec
        E2, F2 = model.predict(st, prec)
        assert np.array_equal(E, E2) or np.abs(E - E2).max() <= 1e-12 * np.abs(E).max()
    kernel = rb.Kernel(calc, name="GAP", zeta=2, target_type="Structure", kernel_type="Sparse")
    krr = rb.KRR(alpha, kernel, sp, {}, precision="fp64")
    assert np.abs(krr.predict_stress(st) + NS_ref).max() <= 1e-10 * scale


def test_empty_and_isolated_atoms():
    frames = [dict(positions=[[5., 5., 5.]], numbers=[1], cell=np.eye(3) * 10., pbc=[False] * 3),
              dict(positions=[[1., 1., 1.], [9., 9., 9.]], numbers=[8, 1], cell=np.eye(3) * 10.,
                   pbc=[False] * 3)]
    batch = batch_from_frames(frames)
    X, Xo, *_ = features_vs_oracle(batch, dict(rc=3.0, n=4, l=3, sigma=0.4))
    assert_features_close(Xo, X)


RS = dict(rate=1.0, scale=4.5, exponent=4.0)


@pytest.mark.parametrize("which", ["periodic_boxes", "molecule_clusters"])
def test_radial_scaling_parity(which):
    """The RadialScaling cutoff (the one of the reference's serialised GAP
    model) on every GPU path: FP64 and FP32 features, FP64 power-spectrum
    gradients, and GAP energies, forces and negative stress at both
    precisions, against the oracle."""
    if which == "periodic_boxes":
        batch, kw = synthetic.periodic_boxes(n_struct=2, seed=6), dict(rc=4.5, n=6, l=4, sigma=0.4, rs=RS)
    else:
        batch, kw = synthetic.molecule_clusters(n_struct=12, seed=8), dict(rc=5.0, n=6, l=4, sigma=0.5, rs=RS)
    X, Xo, al, calc, r0 = features_vs_oracle(batch, kw)
    assert_features_close(Xo, X)
    species = np.unique(batch["numbers"])
    al32 = calc.transform(rb.AtomsList(rb.StructureSet(batch)), precision="fp32")
    X32 = al32.get_features(calc, keys=calc.get_keys(species))
    assert np.abs(X32 - Xo).max() <= 1e-5 * np.abs(Xo).max()
    cg = soap(grads=True, **kw)
    alg = cg.transform(rb.AtomsList(rb.StructureSet(batch)))
    dX = alg.get_features_gradient(cg, keys=cg.get_keys(species))
    r = O.Run(oracle_calc(**kw), batch, species, gradients=True)
    ref = r.power_spectrum_gradient().reshape(dX.shape)
    assert np.abs(dX - ref).max() <= 1e-10 * np.abs(ref).max()
    rr, T, sps, alpha, _ = gap_setup(batch, kw, n_sparse=5)
    E_ref, F_ref, NS_ref = rr.gap_stress(sps, T, alpha, 2)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    st = rb.StructureSet(batch)
    for prec, tol in [("fp64", 1e-10), ("fp32", 1e-4)]:
        E, F, NS = model.predict_stress(st, prec)
        assert np.abs(E - E_ref).max() <= tol * np.abs(E_ref).max(), prec
        assert np.abs(F - F_ref).max() <= tol * np.abs(F_ref).max(), prec
        assert np.abs(NS - NS_ref).max() <= tol * np.abs(NS_ref).max(), prec
