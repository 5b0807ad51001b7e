"""Structure batches: the B200 counterpart of rascal's AtomsList.

Mirrors bindings/rascal/neighbourlist/structure_manager.py:19-300 (AtomsList,
convert_to_structure_list, sanitize_non_periodic_structure) and the
ManagerCollection bindings (bindings/bind_py_structure_manager.cc:472-905).
A whole list of frames becomes one structure set on the device; the
neighbour list is built there for all of them at once.
"""
import ctypes

import numpy as np

from . import _native as N


def _frame_arrays(frame):
    """(positions N x 3, numbers, cell 3 x 3 with rows = lattice vectors,
    pbc, center mask) of an ase.Atoms-like object or a dict."""
    if hasattr(frame, "get_positions"):
        pos = np.asarray(frame.get_positions(), dtype=float)
        num = np.asarray(frame.get_atomic_numbers(), dtype=np.int32)
        cell = np.asarray(frame.get_cell(), dtype=float).reshape(3, 3)
        pbc = np.asarray(frame.get_pbc(), dtype=np.int32).reshape(3)
        arrays = getattr(frame, "arrays", {})
        mask = arrays.get("center_atoms_mask", None) if hasattr(arrays, "get") else None
    elif isinstance(frame, dict):
        pos = np.asarray(frame["positions"], dtype=float)
        num = np.asarray(frame["numbers"] if "numbers" in frame else frame["atom_types"],
                         dtype=np.int32).reshape(-1)
        if pos.ndim == 2 and pos.shape[0] == 3 and pos.shape[1] == len(num) and len(num) != 3:
            pos = pos.T  # rascal's internal 3 x N layout
        cell = np.asarray(frame.get("cell", np.zeros((3, 3))), dtype=float).reshape(3, 3)
        pbc = np.asarray(frame.get("pbc", [0, 0, 0]), dtype=np.int32).reshape(3)
        mask = frame.get("center_atoms_mask", None)
    else:
        raise RuntimeError("Cannot convert structure of type {}".format(type(frame)))
    if mask is None:
        mask = np.ones(len(num), dtype=bool)
    return pos.reshape(-1, 3), num, cell, pbc, np.asarray(mask, dtype=bool).reshape(-1)


def sanitize_non_periodic_structure(pos, cell, pbc):
    """A non-periodic frame with a zero cell gets the bounding box x1.05 as
    its cell and is centred in it (structure_manager.py:265-300)."""
    if np.all(pbc == 0) and np.allclose(cell, np.zeros((3, 3))):
        bounds = np.array([pos.min(axis=0), pos.max(axis=0)])
        L = (bounds[1] - bounds[0]) * 1.05
        cell = np.diag(L)
        pos = pos + (0.5 * L - pos.mean(axis=0))
    return pos, cell


def frames_to_batch(frames):
    """Flat batch arrays of a list of frames."""
    if hasattr(frames, "get_positions") or isinstance(frames, dict):
        frames = [frames]
    pos, num, cells, pbc, mask, off = [], [], [], [], [], [0]
    for f in frames:
        p, n, c, pb, m = _frame_arrays(f)
        p, c = sanitize_non_periodic_structure(p, c, pb)
        pos.append(p)
        num.append(n)
        cells.append(c)
        pbc.append(pb)
        mask.append(m)
        off.append(off[-1] + len(n))
    return dict(atom_offsets=np.asarray(off, dtype=np.int64),
                positions=np.concatenate(pos) if pos else np.zeros((0, 3)),
                numbers=np.concatenate(num) if num else np.zeros(0, np.int32),
                cells=np.asarray(cells, dtype=float).reshape(-1, 3, 3),
                pbc=np.asarray(pbc, dtype=np.int32).reshape(-1, 3),
                center_atoms_mask=np.concatenate(mask) if mask else np.zeros(0, bool))


class StructureSet:
    """Device-resident batch of structures (one rgpu_structures handle)."""

    def __init__(self, batch=None):
        h = ctypes.c_void_p()
        N.check(N.lib().rgpu_structures_create(ctypes.byref(h)))
        self._h = h
        if batch is not None:
            self.set(batch)

    @property
    def handle(self):
        return self._h

    def set(self, batch):
        self.batch = batch
        off = N.i64(batch["atom_offsets"])
        pos = N.f64(batch["positions"])
        num = N.i32(batch["numbers"])
        cel = N.f64(batch["cells"])
        pbc = N.i32(batch["pbc"])
        mask = batch.get("center_atoms_mask")
        m = None
        if mask is not None and not np.all(mask):
            m = np.ascontiguousarray(mask, dtype=np.uint8)
        N.check(N.lib().rgpu_structures_set(self._h, len(off) - 1, N.ptr(off, N.c_i64_p),
                                            N.ptr(pos, N.c_dbl_p), N.ptr(num, N.c_int_p),
                                            N.ptr(cel, N.c_dbl_p), N.ptr(pbc, N.c_int_p),
                                            N.ptr(m, N.c_u8_p)))
        self.n_structures = len(off) - 1
        self.n_atoms = int(off[-1])

    def update_positions(self, positions):
        pos = N.f64(positions)
        N.check(N.lib().rgpu_structures_update_positions(self._h, N.ptr(pos, N.c_dbl_p)))
        self.batch = dict(self.batch, positions=pos)

    def invalidate(self):
        """Recompute the neighbour list and features on the next call."""
        N.check(N.lib().rgpu_structures_invalidate(self._h))

    def stream(self):
        """The cudaStream_t (as an int) this set's kernels run on."""
        p = ctypes.c_void_p()
        N.check(N.lib().rgpu_structures_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def use_graphs(self, enable=True):
        """Record FP32 predictions as CUDA graphs per size bucket (the
        default) or always run the ordinary path (rgpu_structures_use_graphs)."""
        N.check(N.lib().rgpu_structures_use_graphs(self._h, int(bool(enable))))

    def graph_info(self):
        """(buckets held, replays, recordings, kernels of the last replayed
        graph) of the recorded FP32 predictions."""
        info = np.zeros(4, np.int64)
        N.check(N.lib().rgpu_structures_graph_info(self._h, N.ptr(info, N.c_i64_p)))
        return tuple(int(x) for x in info)

    def stage_times(self):
        """Device ms of the stages of the last GAP prediction (see the header)."""
        out = np.zeros(8)
        N.check(N.lib().rgpu_stage_times(self._h, N.ptr(out, N.c_dbl_p), 8))
        return out

    def build_neighbour_list(self, cutoff):
        N.check(N.lib().rgpu_neighbour_list_build(self._h, float(cutoff)))

    def neighbour_list(self):
        nc, np_ = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib().rgpu_neighbour_list_size(self._h, ctypes.byref(nc), ctypes.byref(np_)))
        nc, npairs = nc.value, np_.value
        ca = np.zeros(nc, np.int32)
        po = np.zeros(nc + 1, np.int64)
        j = np.zeros(npairs, np.int32)
        sh = np.zeros((npairs, 3), np.int32)
        d = np.zeros(npairs)
        dr = np.zeros((npairs, 3))
        N.check(N.lib().rgpu_neighbour_list_get(self._h, N.ptr(ca, N.c_int_p), N.ptr(po, N.c_i64_p),
                                                N.ptr(j, N.c_int_p), N.ptr(sh, N.c_int_p),
                                                N.ptr(d, N.c_dbl_p), N.ptr(dr, N.c_dbl_p)))
        return dict(center_atom=ca, pair_offsets=po, j=j, shift=sh, distance=d, direction=dr)

    def synchronize(self):
        N.check(N.lib().rgpu_synchronize(self._h))

    def md_step_info(self):
        """(recorded, (site, box, pair capacities), replays since the
        recording, reason code of the last step that did not replay) of the
        MD step graph (rgpu_md_step_info)."""
        rec = ctypes.c_int32()
        info = np.zeros(6, np.int64)
        N.check(N.lib().rgpu_md_step_info(self._h, ctypes.byref(rec), N.ptr(info, N.c_i64_p)))
        self.md_graph_kernels = int(info[5])
        return bool(rec.value), tuple(int(c) for c in info[:3]), int(info[3]), int(info[4])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and N._lib is not None:
            N._lib.rgpu_structures_destroy(h)
            self._h = None


class AtomsList:
    """A list of structures with a representation computed on the device.

    Mirrors rascal.neighbourlist.AtomsList (structure_manager.py:19-229).
    """

    def __init__(self, frames, nl_options=None, start=None, length=None):
        self.nl_options = nl_options
        if isinstance(frames, StructureSet):
            self.structures = frames
        else:
            batch = frames_to_batch(frames)
            self.structures = StructureSet(batch)
        self._calc = None
        self._precision = N.PRECISION_FP64

    def __len__(self):
        return self.structures.n_structures

    @property
    def batch(self):
        return self.structures.batch

    def _computed(self, calculator):
        if self._calc is not calculator:
            raise RuntimeError("the representation of this calculator has not been computed")

    def get_species(self):
        n = ctypes.c_int32()
        sp = np.zeros(130, np.int32)
        N.check(N.lib().rgpu_get_species(self.structures.handle, ctypes.byref(n), N.ptr(sp, N.c_int_p)))
        return sp[:n.value].copy()

    def get_keys(self, calculator):
        n = ctypes.c_int32()
        N.check(N.lib().rgpu_get_feature_keys(calculator.handle, self.structures.handle,
                                              ctypes.byref(n), None))
        keys = np.zeros(2 * n.value, np.int32)
        N.check(N.lib().rgpu_get_feature_keys(calculator.handle, self.structures.handle,
                                              ctypes.byref(n), N.ptr(keys, N.c_int_p)))
        return keys.reshape(-1, 2)

    def get_features(self, calculator, species=None, keys=None):
        """Dense features, rows = centres, columns = sorted keys x block
        (bind_py_structure_manager.cc:573-614)."""
        self._computed(calculator)
        if keys is None:
            keys = calculator.get_keys(species) if species is not None else self.get_keys(calculator)
        keys = N.i32(np.asarray(keys).reshape(-1, 2))
        nc = self.n_centers()
        inner = calculator.inner_size()
        out = np.zeros((nc, len(keys) * inner))
        N.check(N.lib().rgpu_get_features(calculator.handle, self.structures.handle, len(keys),
                                          N.ptr(keys, N.c_int_p), N.ptr(out, N.c_dbl_p)))
        return out

    def get_features_gradient(self, calculator, species=None, keys=None):
        """Dense gradients, 3 rows per pair incl. self pairs
        (bind_py_structure_manager.cc:621-668)."""
        self._computed(calculator)
        if keys is None:
            keys = calculator.get_keys(species) if species is not None else self.get_keys(calculator)
        keys = N.i32(np.asarray(keys).reshape(-1, 2))
        nl = self.structures.neighbour_list()
        npairs = len(nl["j"])
        inner = calculator.inner_size()
        out = np.zeros((3 * npairs, len(keys) * inner))
        N.check(N.lib().rgpu_get_features_gradient(calculator.handle, self.structures.handle,
                                                   len(keys), N.ptr(keys, N.c_int_p),
                                                   N.ptr(out, N.c_dbl_p)))
        return out

    def n_centers(self):
        nc, np_ = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib().rgpu_neighbour_list_size(self.structures.handle, ctypes.byref(nc),
                                                 ctypes.byref(np_)))
        return nc.value

    def get_representation_info(self):
        """(structure, centre, species) per centre row."""
        nl = self.structures.neighbour_list()
        b = self.batch
        off = b["atom_offsets"]
        struct = np.searchsorted(off, nl["center_atom"], side="right") - 1
        return np.stack([struct, np.arange(len(struct)), b["numbers"][nl["center_atom"]]],
                        axis=1).astype(np.int32)

    def get_gradients_info(self):
        """(structure, centre atom, neighbour atom, species_i, species_j) per
        pair incl. self pairs, atom indices global
        (bind_py_structure_manager.cc:708-745)."""
        nl = self.structures.neighbour_list()
        b = self.batch
        off = b["atom_offsets"]
        counts = np.diff(nl["pair_offsets"])
        ci = np.repeat(nl["center_atom"], counts)
        struct = np.searchsorted(off, ci, side="right") - 1
        return np.stack([struct, ci, nl["j"], b["numbers"][ci], b["numbers"][nl["j"]]],
                        axis=1).astype(np.int32)

    def get_distances(self):
        return self.structures.neighbour_list()["distance"]

    def get_direction_vectors(self):
        return self.structures.neighbour_list()["direction"]
