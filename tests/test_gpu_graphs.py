"""FP32 predictions recorded as CUDA graphs per size bucket.

The first call of a bucket runs the ordinary path and records the bucket;
later calls replay the graph. A replay must give the ordinary path's
results (to the FP64 force atomics' summation order, 1e-12 relative), new
positions of the same sizes must replay correctly, a neighbour list that
outgrows the recorded capacities must fall back to the ordinary path and be
recorded again, and invalid input must still raise the reference's error.
"""
import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import synthetic
from test_gpu_parity import gap_setup, soap

pytestmark = pytest.mark.gpu

KW = dict(rc=5.0, n=8, l=6, sigma=0.4)


def _model(batch, n_sparse=8, seed=0):
    r, T, sps, alpha, species = gap_setup(batch, KW, n_sparse=n_sparse, seed=seed)
    calc = soap(**KW)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    return rb.GAPModel(calc, sp, alpha, 2), r, T, sps, alpha


def _close(a, b, rel=1e-12):
    return np.abs(a - b).max() <= rel * np.abs(b).max()


def _ordinary(model, batch, stress=False):
    st = rb.StructureSet(batch)
    st.use_graphs(False)
    return model.predict_stress(st, "fp32") if stress else model.predict(st, "fp32")


def test_replay_matches_ordinary_and_oracle():
    batch = synthetic.molecule_clusters(n_struct=30, seed=21)
    model, r, T, sps, alpha = _model(batch)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    E0, F0 = _ordinary(model, batch)
    st = rb.StructureSet(batch)
    E1, F1 = model.predict(st, "fp32")   # ordinary path, then the bucket is recorded
    assert st.graph_info()[:3] == (1, 0, 1)
    for k in range(3):
        st.invalidate()
        E2, F2 = model.predict(st, "fp32")  # replays
        assert st.graph_info()[1] == k + 1
        assert _close(E2, E0) and _close(F2, F0)
    assert st.graph_info()[3] > 10  # kernels per replay
    assert np.abs(E2 - E_ref).max() <= 1e-4 * np.abs(E_ref).max()
    assert np.abs(F2 - F_ref).max() <= 1e-4 * np.abs(F_ref).max()


def test_replay_with_new_positions_and_stress():
    batch = synthetic.molecule_clusters(n_struct=20, seed=22)
    model, *_ = _model(batch)
    st = rb.StructureSet(batch)
    model.predict_stress(st, "fp32")
    rng = np.random.default_rng(0)
    for k in range(2):
        # small moves keep every atom inside its (bounding-box) cell
        new = dict(batch)
        new["positions"] = batch["positions"] + 0.01 * rng.normal(size=batch["positions"].shape)
        off = batch["atom_offsets"]
        for i in range(len(off) - 1):
            c = np.diag(batch["cells"][i])
            new["positions"][off[i]:off[i + 1]] = np.clip(new["positions"][off[i]:off[i + 1]], 1e-6, c - 1e-6)
        st.set(new)
        E, F, S = model.predict_stress(st, "fp32")
        E0, F0, S0 = _ordinary(model, new, stress=True)
        assert _close(E, E0) and _close(F, F0) and _close(S, S0, 1e-10)
    assert st.graph_info()[1] == 2


def test_outputs_left_on_device_is_its_own_bucket():
    batch = synthetic.molecule_clusters(n_struct=10, seed=23)
    model, *_ = _model(batch)
    st = rb.StructureSet(batch)
    model.predict(st, "fp32", energies=False, forces=False)
    model.predict(st, "fp32", energies=False, forces=False)
    model.predict(st, "fp32")
    E, F = model.predict(st, "fp32")
    info = st.graph_info()
    assert info[0] == 2 and info[2] == 2 and info[1] == 2
    E0, F0 = _ordinary(model, batch)
    assert _close(E, E0) and _close(F, F0)


def test_outgrown_capacities_fall_back_and_record_again():
    batch = synthetic.molecule_clusters(n_struct=20, seed=24)
    model, *_ = _model(batch)
    st = rb.StructureSet(batch)
    model.predict(st, "fp32")
    assert st.graph_info()[2] == 1
    # the same clusters squeezed towards their cell centres: many more pairs
    dense = dict(batch)
    pos = batch["positions"].copy()
    off = batch["atom_offsets"]
    for i in range(len(off) - 1):
        c = 0.5 * np.diag(batch["cells"][i])
        pos[off[i]:off[i + 1]] = c + 0.6 * (pos[off[i]:off[i + 1]] - c)
    dense["positions"] = pos
    st.set(dense)
    E, F = model.predict(st, "fp32")
    E0, F0 = _ordinary(model, dense)
    assert _close(E, E0) and _close(F, F0)
    assert st.graph_info()[2] == 2  # recorded again with larger capacities
    st.invalidate()
    E, F = model.predict(st, "fp32")
    assert _close(E, E0) and _close(F, F0)


def test_invalid_input_after_recording_raises_reference_error():
    batch = synthetic.molecule_clusters(n_struct=6, seed=25)
    model, *_ = _model(batch)
    st = rb.StructureSet(batch)
    model.predict(st, "fp32")
    bad = dict(batch)
    pos = batch["positions"].copy()
    pos[0] = np.diag(batch["cells"][0]) * 1.5  # outside its cell
    bad["positions"] = pos
    st.set(bad)
    with pytest.raises(RuntimeError, match="not inside the unit cell"):
        model.predict(st, "fp32")
