"""The adjoint path behind torch.autograd (gap_energy): the forward gives the
FP32 energies, the backward the position gradients from the power-spectrum
backward and the pair adjoint, with CUDA positions and gradients staying on
the device. Checked against the oracle's forces (the reference's
KRR.predict_forces, bindings/rascal/models/krr.py:123-166) at the FP32 bar
(1e-4 of the largest force), against central differences of the FP64 GPU
energy, and for an upstream gradient that differs per structure.
"""
import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import _native as N, synthetic
from oracle import oracle as O
from test_gpu_parity import gap_setup, soap

pytestmark = pytest.mark.gpu

KW = dict(rc=5.0, n=8, l=6, sigma=0.4)


def _setup(seed=7, n_struct=10, n_sparse=12):
    batch = synthetic.molecule_clusters(n_struct=n_struct, seed=seed)
    r, T, sps, alpha, species = gap_setup(batch, KW, n_sparse=n_sparse, seed=seed)
    E_ref, F_ref = r.gap(sps, T, alpha, 2)
    calc = soap(**KW)
    sp = rb.SparsePoints(calc)
    sp.add_dense(sps, T, calc.get_keys(species))
    model = rb.GAPModel(calc, sp, alpha, 2)
    return batch, model, E_ref, F_ref


def test_autograd_forces_match_oracle():
    import torch
    batch, model, E_ref, F_ref = _setup()
    st = rb.StructureSet(batch)
    pos = torch.tensor(batch["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    E = rb.gap_energy(pos, model, st)
    assert E.is_cuda and E.shape == (len(batch["atom_offsets"]) - 1,)
    (g,) = torch.autograd.grad(E.sum(), pos)
    assert g.is_cuda
    E = E.detach().cpu().numpy()
    g = g.cpu().numpy()
    assert np.abs(E - E_ref).max() <= 1e-4 * np.abs(E_ref).max()
    assert np.abs(-g - F_ref).max() <= 1e-4 * np.abs(F_ref).max()


def test_autograd_upstream_gradient_per_structure():
    import torch
    batch, model, E_ref, F_ref = _setup(seed=8)
    st = rb.StructureSet(batch)
    w = np.random.default_rng(0).normal(size=len(E_ref))
    pos = torch.tensor(batch["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    E = rb.gap_energy(pos, model, st)
    (g,) = torch.autograd.grad((E * torch.tensor(w, device="cuda")).sum(), pos)
    sidx = np.repeat(np.arange(len(E_ref)), np.diff(batch["atom_offsets"]))
    ref = -F_ref * w[sidx][:, None]
    assert np.abs(g.cpu().numpy() - ref).max() <= 1e-4 * np.abs(ref).max()


def test_autograd_against_finite_differences_of_fp64_energy():
    """Central differences (h = 1e-4 A) of the FP64 GPU energy of one
    structure against the autograd gradient of the FP32 path."""
    import torch
    batch, model, _, _ = _setup(seed=9, n_struct=3)
    st = rb.StructureSet(batch)
    pos0 = np.asarray(batch["positions"], dtype=np.float64)
    pos = torch.tensor(pos0, device="cuda", requires_grad=True)
    (g,) = torch.autograd.grad(rb.gap_energy(pos, model, st).sum(), pos)
    g = g.cpu().numpy()
    ref = rb.StructureSet(batch)
    h = 1e-4
    rng = np.random.default_rng(1)
    picks = [(int(a), int(c)) for a, c in zip(rng.integers(0, len(pos0), 8), rng.integers(0, 3, 8))]
    fd = []
    for a, c in picks:
        e = []
        for sgn in (1, -1):
            p = pos0.copy()
            p[a, c] += sgn * h
            ref.update_positions(p)
            E, _ = model.predict(ref, "fp64", forces=False)
            e.append(E.sum())
        fd.append((e[0] - e[1]) / (2 * h))
    fd = np.array(fd)
    got = np.array([g[a, c] for a, c in picks])
    assert np.abs(got - fd).max() <= 1e-4 * np.abs(g).max()


def test_autograd_host_positions():
    """Host positions are accepted too: the gradient comes back on the host."""
    import torch
    batch, model, _, F_ref = _setup(seed=10, n_struct=4)
    st = rb.StructureSet(batch)
    pos = torch.tensor(batch["positions"], dtype=torch.float64, requires_grad=True)
    E = rb.gap_energy(pos, model, st)
    assert not E.is_cuda
    E.sum().backward()
    assert not pos.grad.is_cuda
    assert np.abs(-pos.grad.numpy() - F_ref).max() <= 1e-4 * np.abs(F_ref).max()


def test_backward_needs_its_forward():
    import torch
    batch, model, _, _ = _setup(seed=11, n_struct=3)
    st = rb.StructureSet(batch)
    pos = torch.tensor(batch["positions"], dtype=torch.float64, device="cuda")
    E = torch.empty(3, dtype=torch.float64, device="cuda")
    N.check(N.lib().rgpu_gap_forward_dev(model.handle, st.handle, pos.data_ptr(), E.data_ptr()))
    st.invalidate()  # another call on the structures in between
    g = torch.ones(3, dtype=torch.float64, device="cuda")
    out = torch.empty((st.n_atoms, 3), dtype=torch.float64, device="cuda")
    rc = N.lib().rgpu_gap_backward_dev(model.handle, st.handle, g.data_ptr(), out.data_ptr())
    assert rc == N.ERR_NOT_COMPUTED
