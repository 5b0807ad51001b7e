"""Regenerate the golden fixtures in this folder from the reference's own data.

Run from the repository root, in a checkout that has the reference tree:

    python tests/golden/make_golden.py /path/to/librascal

It reads only data files of the reference (``reference_data/``): the
mpmath/scipy-generated known-answer files for 1F1 and Y_lm, the expansion and
kernel golden matrices written by the reference's own scripts, and the test
input structures. Everything it writes is small (a few MB) and is committed,
so the tests never need the reference tree at run time.

Written files:
  hyp1f1.npz            a, b, z, val, der              (tests/test_math_hyp1f1.cc)
  spherical_harmonics.npz  lmax, unit vectors, Y, ALPs   (tests/test_math_spherical_harmonics.cc)
  expansion_reference.npz  GTO + ShiftedCosine subset of spherical_expansion_reference.ubjson
  kernel_reference.npz     PowerSpectrum subset of kernel_reference.ubjson
  structures.json          test input structures (ASE-db json subset)
  sparse_kernel_inputs.json  parameters of the reference's sparse-kernel
                           gradient tests (tests/test_sparse_kernels.cc:129-220)

  simple_gap_model.json, methane_dimer_sample.xyz
                           the reference's serialised GAP model and its
                           structures, copied unchanged
                           (tests/python/md_calculator_test.py)

`python tests/golden/make_golden.py <ref> sparse_kernel_inputs` rewrites only
the sparse-kernel inputs, `... <ref> model_files` only the model files.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ubjson_reader  # noqa: E402


def read_ase_db(path, start=0, length=None):
    """Frames of an ASE-db json file, sorted by integer id."""
    d = json.load(open(path))
    ids = sorted(int(k) for k in d if k.isdigit())
    ids = ids[start:] if length is None else ids[start:start + length]
    frames = []
    for i in ids:
        e = d[str(i)]
        cell = np.array(e.get("cell", np.zeros((3, 3))), dtype=float).reshape(3, 3)
        pbc = np.array(e.get("pbc", [False] * 3), dtype=bool)
        frames.append(dict(positions=np.array(e["positions"], dtype=float).tolist(),
                           numbers=[int(x) for x in e["numbers"]],
                           cell=cell.tolist(), pbc=[bool(x) for x in pbc]))
    return frames


def sparse_kernel_inputs(ref_root):
    """The cases of reference_data/tests_only/sparse_kernel_inputs.json, with
    each structure file named by its key in structures.json."""
    td = os.path.join(ref_root, "reference_data", "tests_only")
    cases = []
    for e in json.load(open(os.path.join(td, "sparse_kernel_inputs.json"))):
        hy = e["calculator"]
        f = os.path.basename(e["filename"])
        n = int(e["n_structures"])
        key = f if f != "small_molecules-20.json" else "%s:0:%d" % (f, n)
        cases.append(dict(
            structure=key, n_structures=n,
            cutoff=float(hy["cutoff_function"]["cutoff"]["value"]),
            smooth_width=float(hy["cutoff_function"]["smooth_width"]["value"]),
            sigma=float(hy["gaussian_density"]["gaussian_sigma"]["value"]),
            max_radial=int(hy["max_radial"]), max_angular=int(hy["max_angular"]),
            normalize=bool(hy["normalize"]),
            spline="Spline" in hy["radial_contribution"].get("optimization", {}),
            zeta=int(e["kernel"]["zeta"]), target_type=e["kernel"]["target_type"],
            h=float(e["h"]), selected_ids=e["selected_ids"]))
    json.dump(cases, open(os.path.join(HERE, "sparse_kernel_inputs.json"), "w"), indent=1)


def model_files(ref_root):
    import shutil
    shutil.copyfile(os.path.join(ref_root, "reference_data", "tests_only", "simple_gap_model.json"),
                    os.path.join(HERE, "simple_gap_model.json"))
    shutil.copyfile(os.path.join(ref_root, "reference_data", "inputs", "methane_dimer_sample.xyz"),
                    os.path.join(HERE, "methane_dimer_sample.xyz"))


def main(ref_root):
    td = os.path.join(ref_root, "reference_data", "tests_only")
    inp = os.path.join(ref_root, "reference_data", "inputs")

    # --- 1F1 known answers (mpmath, 200 digits)
    h = ubjson_reader.load(os.path.join(td, "hyp1f1_reference.ubjson"))
    np.savez_compressed(os.path.join(HERE, "hyp1f1.npz"),
                        a=np.array([e["a"] for e in h]), b=np.array([e["b"] for e in h]),
                        z=np.array([e["z"] for e in h]), val=np.array([e["val"] for e in h]),
                        der=np.array([e["der"] for e in h]))

    # --- spherical harmonics known answers
    s = ubjson_reader.load(os.path.join(td, "spherical_harmonics_reference.ubjson"))
    np.savez_compressed(os.path.join(HERE, "spherical_harmonics.npz"),
                        lmax=np.array([e["max_angular_l"] for e in s]),
                        unit_vector=np.array([e["unit_vector"] for e in s]),
                        harmonics=np.array([np.asarray(e["harmonics"]) for e in s]),
                        alps=np.array([np.asarray(e["alps"]) for e in s]))

    structures = {}
    # --- spherical expansion goldens: GTO with the ShiftedCosine or RadialScaling cutoff, no RDR
    se = ubjson_reader.load(os.path.join(td, "spherical_expansion_reference.ubjson"))
    files = [os.path.basename(f) for f in se["filenames"]]
    for f in files:
        structures[f] = read_ase_db(os.path.join(inp, f))
    cases = []
    i_case = 0
    for i_f, f in enumerate(files):
        for rc in se["cutoffs"]:
            block = se["rep_info"][i_case]
            i_case += 1
            for e in block:
                hy = e["hypers"]
                rcontrib = hy["radial_contribution"]
                opt = list(rcontrib.get("optimization", {}).keys())
                cf = hy["cutoff_function"]
                if rcontrib["type"] != "GTO" or cf["type"] not in ("ShiftedCosine", "RadialScaling"):
                    continue
                rs = None
                if cf["type"] == "RadialScaling":
                    rs = dict(rate=float(cf["rate"]["value"]), scale=float(cf["scale"]["value"]),
                              exponent=float(cf["exponent"]["value"]))
                if "RadialDimReduction" in opt:
                    continue
                spline = "Spline" in opt
                acc = rcontrib["optimization"]["Spline"]["accuracy"] if spline else 0.0
                cases.append(dict(
                    structure=f, cutoff=float(hy["cutoff_function"]["cutoff"]["value"]),
                    smooth_width=float(hy["cutoff_function"]["smooth_width"]["value"]),
                    sigma=float(hy["gaussian_density"]["gaussian_sigma"]["value"]),
                    max_radial=int(hy["max_radial"]), max_angular=int(hy["max_angular"]),
                    spline=spline, accuracy=float(acc), radial_scaling=rs,
                    features=np.asarray(e["feature_matrix"], dtype=float)))
    np.savez_compressed(
        os.path.join(HERE, "expansion_reference.npz"),
        meta=json.dumps([{k: v for k, v in c.items() if k != "features"} for c in cases]),
        **{"features_%d" % i: c["features"] for i, c in enumerate(cases)})

    # --- kernel goldens: PowerSpectrum entries only
    kr = ubjson_reader.load(os.path.join(td, "kernel_reference.ubjson"))
    kfile = os.path.basename(kr["filename"])
    structures[kfile + ":%d:%d" % (kr["start"], kr["length"])] = read_ase_db(
        os.path.join(inp, kfile), kr["start"], kr["length"])
    kcases = []
    for e in kr["rep_info"]["spherical_invariants"][0]:
        hy = e["hypers_rep"]
        if hy["soap_type"] != "PowerSpectrum":
            continue
        opt = hy["radial_contribution"].get("optimization", {})
        kcases.append(dict(
            cutoff=float(hy["cutoff_function"]["cutoff"]["value"]),
            smooth_width=float(hy["cutoff_function"]["smooth_width"]["value"]),
            sigma=float(hy["gaussian_density"]["gaussian_sigma"]["value"]),
            max_radial=int(hy["max_radial"]), max_angular=int(hy["max_angular"]),
            normalize=bool(hy["normalize"]), spline="Spline" in opt,
            target_type=e["hypers_kernel"]["target_type"], zeta=int(e["hypers_kernel"]["zeta"]),
            kernel=np.asarray(e["kernel_matrix"], dtype=float)))
    np.savez_compressed(
        os.path.join(HERE, "kernel_reference.npz"),
        structures=kfile + ":%d:%d" % (kr["start"], kr["length"]),
        meta=json.dumps([{k: v for k, v in c.items() if k != "kernel"} for c in kcases]),
        **{"kernel_%d" % i: c["kernel"] for i, c in enumerate(kcases)})

    # --- neighbour-list test inputs used by the reference's adaptor tests
    for f in ["simple_cubic_8.json", "linked_cell_break_0.json", "diamond_cubic_distorted.json",
              "diamond_2atom_distorted.json", "SiC_moissanite.json", "SiCGe_wurtzite_like.json",
              "methane.json", "molecular_crystal.json"]:
        p = os.path.join(inp, f)
        if os.path.exists(p):
            try:
                structures[f] = read_ase_db(p)
            except Exception as exc:  # not an ASE-db file
                print("skip", f, exc)
    json.dump(structures, open(os.path.join(HERE, "structures.json"), "w"))
    print("expansion cases", len(cases), "kernel cases", len(kcases),
          "structure files", len(structures))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    only = sys.argv[2:]
    if not only:
        main(root)
    if not only or only == ["sparse_kernel_inputs"]:
        sparse_kernel_inputs(root)
    if not only or only == ["model_files"]:
        model_files(root)
