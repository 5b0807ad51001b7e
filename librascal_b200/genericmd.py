"""Calculator-style interface for MD drivers (i-PI and the like).

Mirrors GenericMDCalculator of bindings/rascal/models/genericmd.py:9-130: it
loads a model JSON (the reference's own format, `io.load_obj`), takes the
atom types from a structure template (extended XYZ or ASE-db JSON) or from
a list of atomic numbers, and returns energy, forces and the 3 x 3 stress
for each position and cell update, assuming the order and identity of the
atoms do not change.

Each step keeps one structures handle. With the FP32 path on a periodic
system whose cell does not change, a step is one `rgpu_md_step` call: the
whole step, neighbour list included, is recorded once as a CUDA graph and
replayed with the new positions. Otherwise the positions are updated in
place and one `rgpu_gap_predict_stress` call returns energy, forces and
stress together; no device buffer is reallocated after the first step.
"""
import numpy as np

from . import io
from .neighbourlist import StructureSet, frames_to_batch


class GenericMDCalculator:
    """Generic MD driver for a GAP model.

    precision: "fp64" runs the reference's arithmetic, "fp32" the adjoint
    fast path (forces within 1e-4 of the largest force).
    """

    matrix_indices_in_voigt_notation = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))

    def __init__(self, model_json, is_periodic, structure_template=None, atomic_numbers=None,
                 precision="fp64"):
        self.model_filename = model_json
        self.model = io.load_obj(model_json)
        self.model.precision = precision
        self.representation = self.model.get_representation_calculator()
        self.is_periodic = is_periodic
        if structure_template is not None:
            self.template_filename = structure_template
            if str(structure_template).endswith(".json"):
                frame = io.read_ase_json(structure_template, 0, 1)[0]
            else:
                frame = io.read_extxyz(structure_template, 0)
            self.numbers = np.asarray(frame["numbers"], np.int32)
            pbc = np.asarray(frame["pbc"], bool)
            if is_periodic is not None and is_periodic != bool(np.any(pbc)):
                raise ValueError("Structure template PBC flags: " + str(pbc) +
                                 " incompatible with 'is_periodic' setting")
            self.pbc = pbc
        elif atomic_numbers is not None:
            self.numbers = np.asarray(atomic_numbers, np.int32)
            self.pbc = np.array([bool(is_periodic)] * 3)
        else:
            raise ValueError("Must specify one of 'structure_template' or 'atomic_numbers'")
        self.structures = None
        self._cell = None

    def _wrap(self, positions, cell):
        """Fold positions into the cell along periodic directions, with the
        1e-11 tolerance the reference applies before its first step."""
        if not np.any(self.pbc):
            return positions
        eps = 1e-11
        f = positions @ np.linalg.inv(cell)
        for k in range(3):
            if self.pbc[k]:
                f[:, k] = (f[:, k] + eps) % 1.0 - eps
        return f @ cell

    def calculate(self, positions, cell_matrix):
        """Energy (array of one), forces (N x 3) and stress (3 x 3, eV/A^3)
        for positions N x 3 and the cell (rows are lattice vectors; zeros
        for a non-periodic system)."""
        positions = np.asarray(positions, float)
        cell_matrix = np.asarray(cell_matrix, float)
        if positions.shape != (len(self.numbers), 3):
            raise ValueError("Improper shape of positions (is the number of atoms consistent?)")
        if cell_matrix.shape != (3, 3):
            raise ValueError("Improper shape of cell info (expected 3x3 matrix)")
        pos = self._wrap(positions, cell_matrix)
        frame = dict(positions=pos, numbers=self.numbers, cell=cell_matrix, pbc=self.pbc)
        batch = frames_to_batch([frame])
        new_cell = self.structures is None or self._cell is None or not np.array_equal(self._cell, cell_matrix) \
            or not np.any(self.pbc)
        if new_cell:
            # first step, a new cell, or a cluster whose bounding-box cell follows the atoms
            if self.structures is None:
                self.structures = StructureSet(batch)
            else:
                self.structures.set(batch)
            self._cell = cell_matrix.copy()
        if self.model.precision == "fp32" and np.any(self.pbc):
            E, F, NS = self.model._gap().md_step(self.structures, batch["positions"], stress=True)
        else:
            if not new_cell:
                self.structures.update_positions(batch["positions"])
            E, F, NS = self.model._gap().predict_stress(self.structures, self.model.precision)
        energy = E
        stress_voigt = -NS[0]
        stress_matrix = np.zeros((3, 3))
        stress_matrix[tuple(zip(*self.matrix_indices_in_voigt_notation))] = stress_voigt
        # the reference adds the transposed upper triangle, its diagonal
        # included, so the diagonal entries come out doubled
        # (models/genericmd.py:126-127); kept for identical results
        stress_matrix += np.triu(stress_matrix).T
        return energy, F, stress_matrix
