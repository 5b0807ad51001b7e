"""librascal_b200: B200-native SOAP power spectrum and sparse-GAP energies and
forces, a drop-in for librascal's descriptor hot path.

Public API (same names and arguments as the reference's Python package):
  SphericalInvariants, SphericalExpansion   representations/
  AtomsList                                 neighbourlist/
  SparsePoints, Kernel, KRR,
  compute_sparse_kernel_gradients           models/
plus StructureSet / GAPModel (direct handles on the C ABI) and gap_energy
(torch.autograd.Function over the adjoint force path).
"""
from ._native import LIB_PATH, lib  # noqa: F401
from .models import (KRR, GAPModel, Kernel, SparsePoints, compute_KNM, compute_sparse_kernel_gradients,  # noqa: F401
                     gap_energy, train_gap_model)
from .neighbourlist import AtomsList, StructureSet, frames_to_batch  # noqa: F401
from .representations import SphericalExpansion, SphericalInvariants  # noqa: F401
from .io import dump_obj, load_obj, read_ase_json, read_extxyz  # noqa: F401
from .genericmd import GenericMDCalculator  # noqa: F401

__all__ = ["SphericalInvariants", "SphericalExpansion", "AtomsList", "StructureSet", "SparsePoints",
           "Kernel", "KRR", "GAPModel", "compute_sparse_kernel_gradients", "compute_KNM", "train_gap_model",
           "gap_energy", "dump_obj", "load_obj", "read_ase_json", "read_extxyz", "GenericMDCalculator",
           "frames_to_batch"]
