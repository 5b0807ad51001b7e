"""rgpu_md_step: the FP32 MD step replayed as a recorded CUDA graph gives the
same energies, forces and negative stress as the ordinary FP32 path
(rgpu_gap_predict_stress) step after step, including a step whose
neighbour list outgrows the recorded capacities, and reports invalid
positions with the reference's message."""
import numpy as np
import pytest

import librascal_b200 as rb
from helpers import wrap
from librascal_b200 import synthetic
from test_gpu_parity import gap_setup, soap

pytestmark = pytest.mark.gpu


def close(a, b, tol=1e-12):
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


def setup_box(seed=0):
    batch = synthetic.periodic_boxes(n_struct=1, seed=seed, side=12.0, n_atoms=150)
    kw = dict(rc=4.0, n=6, l=4, sigma=0.3)
    r, T, sps, alpha, species = gap_setup(batch, kw, n_sparse=6)
    calc = soap(**kw)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    return batch, rb.GAPModel(calc, sp, alpha, 2)


class Ordinary:
    """The ordinary FP32 path on a handle of its own, kept across steps: a
    new handle would allocate device memory, and any allocation makes the
    MD step record its graph anew instead of replaying it."""

    def __init__(self, model, batch):
        self.model = model
        self.st = rb.StructureSet(batch)

    def __call__(self, pos):
        self.st.update_positions(pos)
        return self.model.predict_stress(self.st, "fp32")


def test_md_step_matches_ordinary_path():
    batch, model = setup_box()
    st = rb.StructureSet(batch)
    ordinary = Ordinary(model, batch)
    ordinary(batch["positions"])
    rng = np.random.default_rng(1)
    pos = batch["positions"].copy()
    for step in range(8):
        pos = wrap(dict(batch, positions=pos + 0.02 * rng.normal(size=pos.shape)))["positions"]
        E, F, NS = model.md_step(st, pos, stress=True)
        E0, F0, NS0 = ordinary(pos)
        # same kernels and inputs; only the order of FP64 atomic additions differs
        assert close(E, E0) and close(F, F0) and close(NS, NS0), step
        recorded, caps, replays, _ = st.md_step_info()
        assert recorded and min(caps) > 0, step
    # the later steps replayed the recorded graph (the first ones may record
    # again while the comparison handle's buffers still grow)
    assert replays >= 3, st.md_step_info()
    # without the stress, on the same handle (records a new graph)
    E, F, NS = model.md_step(st, pos, stress=False)
    assert NS is None and close(F, F0)


def test_md_step_outgrows_capacities():
    batch, model = setup_box(seed=3)
    st = rb.StructureSet(batch)
    ordinary = Ordinary(model, batch)
    pos = batch["positions"].copy()
    ordinary(pos)
    for _ in range(3):
        model.md_step(st, pos, stress=True)
    assert st.md_step_info()[2] >= 1
    # pull every atom towards the box centre: the pair count grows far past
    # the 25 % headroom, so the step goes through the ordinary path
    centre = 0.5 * np.diag(batch["cells"][0])
    squeezed = centre + 0.6 * (pos - centre)
    _, caps0, _, _ = st.md_step_info()
    E, F, NS = model.md_step(st, squeezed, stress=True)
    E0, F0, NS0 = ordinary(squeezed)
    assert close(E, E0) and close(F, F0) and close(NS, NS0)
    recorded, caps1, _, reason = st.md_step_info()
    assert recorded and caps1[2] > caps0[2] and reason == 204  # outgrown, recorded again
    # and later steps replay a graph recorded for the new counts
    for k in range(3):
        p = squeezed + 0.001 * k
        E, F, NS = model.md_step(st, p, stress=True)
        E0, F0, NS0 = ordinary(p)
        assert close(E, E0) and close(F, F0) and close(NS, NS0)
    assert st.md_step_info()[2] >= 1


def test_md_step_invalid_positions():
    batch, model = setup_box(seed=5)
    st = rb.StructureSet(batch)
    ordinary = Ordinary(model, batch)
    pos = batch["positions"].copy()
    ordinary(pos)
    model.md_step(st, pos)
    model.md_step(st, pos)
    assert st.md_step_info()[2] == 1
    bad = pos.copy()
    bad[7] += np.array([50.0, 0.0, 0.0])  # outside the cell
    with pytest.raises(RuntimeError, match="not inside the unit cell"):
        model.md_step(st, bad)
    # the handle recovers with valid positions
    E, F, _ = model.md_step(st, pos)
    E0, F0, _ = ordinary(pos)
    assert close(E, E0) and close(F, F0)
