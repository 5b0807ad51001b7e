"""Shared test helpers: structure batches, error metrics, wrapping."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DBL_FTOL = 100.0 * np.finfo(np.float64).eps


def load_structures():
    with open(os.path.join(GOLDEN, "structures.json")) as f:
        return json.load(f)


def sanitize(pos, cell, pbc):
    """A zero cell of a non-periodic frame becomes the bounding box x1.05
    with the atoms centred (bindings/rascal/neighbourlist/structure_manager.py:280-299)."""
    if not np.any(pbc) and np.allclose(cell, 0):
        L = (pos.max(0) - pos.min(0)) * 1.05
        cell = np.diag(L)
        pos = pos + (0.5 * L - pos.mean(0))
    return pos, cell


def batch_from_frames(frames):
    pos, num, cells, pbc, mask, off = [], [], [], [], [], [0]
    for f in frames:
        p = np.asarray(f["positions"], dtype=float)
        c = np.asarray(f["cell"], dtype=float).reshape(3, 3)
        pb = np.asarray(f["pbc"], dtype=int).reshape(3)
        p, c = sanitize(p, c, pb)
        pos.append(p)
        num.append(np.asarray(f["numbers"], dtype=np.int32))
        cells.append(c)
        pbc.append(pb)
        mask.append(np.asarray(f.get("center_atoms_mask", np.ones(len(p), bool)), dtype=bool))
        off.append(off[-1] + len(p))
    return dict(atom_offsets=np.asarray(off, dtype=np.int64), positions=np.concatenate(pos),
                numbers=np.concatenate(num), cells=np.asarray(cells), pbc=np.asarray(pbc),
                center_atoms_mask=np.concatenate(mask))


def wrap(batch):
    """Fold periodic atoms back into their cell (atomic_structure.hh:180-195)."""
    b = dict(batch)
    pos = batch["positions"].copy()
    for s in range(len(b["atom_offsets"]) - 1):
        a0, a1 = b["atom_offsets"][s], b["atom_offsets"][s + 1]
        if np.any(b["pbc"][s]):
            c = b["cells"][s]
            f = pos[a0:a1] @ np.linalg.inv(c)
            f = np.where(b["pbc"][s].astype(bool), np.mod(f, 1.0), f)
            pos[a0:a1] = f @ c
    b["positions"] = pos
    return b


def relative_error(ref, test, epsilon=DBL_FTOL):
    """math/utils.hh:152-225: relative error where |ref| > epsilon, else absolute."""
    ref = np.asarray(ref)
    test = np.asarray(test)
    d = np.abs(ref - test)
    r = np.abs(ref)
    big = r > epsilon
    return np.where(big, d / np.where(big, r, 1.0), d)
