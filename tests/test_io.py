"""Model and structure files (no GPU needed): the reference's serialised GAP
model loads, serialises back to the same JSON, and survives a dump/load
round trip; extended XYZ and ASE-db JSON readers; the MD calculator's
argument checks."""
import json
import os

import numpy as np
import pytest

import librascal_b200 as rb
from helpers import GOLDEN, load_structures
from librascal_b200 import io

MODEL = os.path.join(GOLDEN, "simple_gap_model.json")
XYZ = os.path.join(GOLDEN, "methane_dimer_sample.xyz")


def _int_keys(o):
    return {(int(k) if isinstance(k, str) and k.lstrip("-").isdigit() else k): v for k, v in o.items()}


def _canonical(d):
    """JSON text of a BaseIO dict with numpy arrays as the ["npy", list] form."""
    def conv(o):
        if isinstance(o, dict):
            return {str(k): conv(v) for k, v in o.items()}
        if isinstance(o, (list, tuple)):
            return [conv(x) for x in o]
        if isinstance(o, np.ndarray):
            return ["npy", conv(o.tolist())]
        if isinstance(o, (np.integer,)):
            return int(o)
        if isinstance(o, (np.floating,)):
            return float(o)
        return o
    return json.loads(json.dumps(conv(d), sort_keys=True))


def test_load_reference_model():
    krr = io.load_obj(MODEL)
    assert isinstance(krr, rb.KRR)
    assert krr.kernel.zeta == 2 and krr.kernel.kernel_type == "Sparse"
    assert krr.self_contributions == {1: 0, 6: 0}
    calc = krr.get_representation_calculator()
    assert calc.hypers["cutoff_function"]["type"] == "RadialScaling"
    sp = krr.X_train
    assert sp.size() == 30 and sp.species == [1] * 20 + [6] * 10
    assert krr.weights.shape == (30,)
    T = sp.get_features()
    assert T.shape == (30, 3 * calc.inner_size())
    # normalised power spectra
    assert np.allclose(np.linalg.norm(T, axis=1), 1.0, atol=1e-12)


def test_reference_model_serialises_back_unchanged():
    with open(MODEL) as f:
        original = json.load(f, object_hook=_int_keys)
    again = io.to_dict(io.load_obj(MODEL))
    assert _canonical(again) == _canonical(original)


def test_dump_load_round_trip(tmp_path):
    krr = io.load_obj(MODEL)
    fn = str(tmp_path / "model.json")
    io.dump_obj(fn, krr)
    krr2 = io.load_obj(fn)
    assert np.array_equal(krr2.weights, krr.weights)
    assert np.array_equal(krr2.X_train.get_features(), krr.X_train.get_features())
    assert krr2.X_train.species == krr.X_train.species
    assert krr2.kernel.zeta == krr.kernel.zeta
    assert krr2.get_representation_calculator().hypers == krr.get_representation_calculator().hypers
    assert _canonical(io.to_dict(krr2)) == _canonical(io.to_dict(krr))


def test_large_arrays_go_to_npy_files(tmp_path, monkeypatch):
    monkeypatch.setattr(io, "_LARGE", 100)
    krr = io.load_obj(MODEL)
    fn = str(tmp_path / "m.json")
    io.dump_obj(fn, krr)
    side = [p for p in os.listdir(tmp_path) if p.endswith(".npy")]
    assert side == ["m-krr-weights.npy"]
    assert np.array_equal(io.load_obj(fn).weights, krr.weights)


def test_read_extxyz():
    frames = io.read_extxyz(XYZ)
    assert len(frames) == 100
    f = frames[0]
    assert f["numbers"].tolist() == [6, 1, 1, 1, 1, 6, 1, 1, 1, 1]
    assert f["positions"].shape == (10, 3) and f["arrays"]["force"].shape == (10, 3)
    assert np.array_equal(f["cell"], np.eye(3) * 30.0) and f["pbc"].tolist() == [True] * 3
    assert abs(f["info"]["energy"] - (-0.00961079)) < 1e-15
    assert f["info"]["comment"].startswith("Sample of 100 methane dimers")
    assert len(io.read_extxyz(XYZ, ":10")) == 10
    assert io.read_extxyz(XYZ, 3)["info"]["energy"] == frames[3]["info"]["energy"]


def test_read_ase_json_matches_fixture(tmp_path):
    frames = load_structures()["small_molecules-20.json:0:5"]
    db = {"ids": list(range(1, 6)), "nextid": 6}
    for i, f in enumerate(frames, start=1):
        db[str(i)] = dict(positions=f["positions"], numbers=f["numbers"], cell=f["cell"], pbc=f["pbc"])
    fn = str(tmp_path / "s.json")
    json.dump(db, open(fn, "w"))
    got = io.read_ase_json(fn, start=1, length=3)
    assert len(got) == 3
    for g, f in zip(got, frames[1:4]):
        assert np.array_equal(g["positions"], np.asarray(f["positions"]))
        assert g["numbers"].tolist() == list(f["numbers"])
    with pytest.raises(RuntimeError, match="not recognized"):
        json.dump({"1": {}}, open(fn, "w"))
        io.read_ase_json(fn)


def test_md_calculator_arguments():
    with pytest.raises(ValueError, match="Must specify one of 'structure_template' or 'atomic_numbers'"):
        rb.GenericMDCalculator(MODEL, True)
    with pytest.raises(ValueError, match="incompatible with 'is_periodic' setting"):
        rb.GenericMDCalculator(MODEL, False, XYZ)
