"""Sparse GAP prediction on the B200 path.

Mirrors bindings/rascal/models/{sparse_points.py, kernels.py, krr.py} for
prediction: SparsePoints (the reference's SparsePointsBlockSparse,
src/rascal/models/sparse_points.hh:50-448), Kernel (GAP, Sparse),
KRR.predict / predict_forces (models/krr.py:92-166) and
compute_sparse_kernel_gradients (bind_py_models.cc:148-200). Energies and
forces of a whole AtomsList come from one rgpu_gap_predict call:

  precision="fp64"  the reference's own algorithm on the GPU (materialised
                    dX/dr contracted with the scaled sparse points), FP64;
  precision="fp32"  the adjoint path: FP32 expansion, TF32 tensor-core GEMMs
                    with FP32 accumulation, dE/dC contracted with dC/dr
                    recomputed per pair; FP64 energy reduction.

PyTorch is used only by GAPEnergy (a torch.autograd.Function around the
adjoint path) and is imported lazily.
"""
import ctypes

import numpy as np

from . import _native as N
from .neighbourlist import AtomsList, StructureSet, _frame_arrays, frames_to_batch

_PREC = {"fp64": N.PRECISION_FP64, "fp32": N.PRECISION_FP32}


class SparsePoints:
    """Selected environments (sparse points) with their dense features.

    Rows are stored per key, as the reference stores `values[sp][key]`; the
    dense matrix over a species layout is assembled on demand.
    """

    def __init__(self, representation):
        self._representation = representation
        self.species = []       # central species of each point
        self.values = []        # dict key -> vector, per point
        self._models = {}       # zeta -> GAPModel with zero weights (kernel matrices)

    def _group_by_species(self):
        """Points of one species together, species ascending, insertion
        order inside a species: the column order of the reference's
        SparsePointsBlockSparse (offset(sp) + index, sparse_points.hh:341-417)."""
        order = sorted(range(len(self.species)), key=lambda i: self.species[i])
        self.species = [self.species[i] for i in order]
        self.values = [self.values[i] for i in order]
        self._models = {}  # device copies made by Kernel, now stale

    def size(self):
        return len(self.species)

    def __len__(self):
        return self.size()

    def extend(self, managers, selected_ids):
        """Add the centres `selected_ids[i_structure]` of `managers`
        (models/sparse_points.py extend, sparse_points.hh:360-417)."""
        calc = self._representation
        keys = managers.get_keys(calc)
        X = managers.get_features(calc, keys=keys)
        info = managers.get_representation_info()
        inner = calc.inner_size()
        row0 = 0
        off = managers.batch["atom_offsets"]
        mask = managers.batch.get("center_atoms_mask")
        for i_struct, ids in enumerate(selected_ids):
            if mask is not None:
                n_c = int(np.sum(mask[off[i_struct]:off[i_struct + 1]]))
            else:
                n_c = int(off[i_struct + 1] - off[i_struct])
            for i in ids:
                if i >= n_c:
                    raise RuntimeError("selected id %d out of range" % i)
                r = row0 + int(i)
                v = {}
                for k, key in enumerate(keys):
                    blk = X[r, k * inner:(k + 1) * inner]
                    if np.any(blk != 0):
                        v[(int(key[0]), int(key[1]))] = blk.copy()
                self.values.append(v)
                self.species.append(int(info[r, 2]))
            row0 += n_c
        self._group_by_species()

    def add_dense(self, species, T, keys):
        """Add points from a dense matrix with the given key layout."""
        inner = self._representation.inner_size()
        for s, row in zip(species, np.asarray(T)):
            v = {}
            for k, key in enumerate(keys):
                blk = row[k * inner:(k + 1) * inner]
                if np.any(blk != 0):
                    v[(int(key[0]), int(key[1]))] = np.array(blk, dtype=float)
            self.values.append(v)
            self.species.append(int(s))
        self._group_by_species()

    def get_species(self):
        sp = set(self.species)
        for v in self.values:
            for k in v:
                sp.update(k)
        return sorted(sp)

    def dense(self, species):
        """T [n_points x D] in the power-spectrum layout of `species`."""
        species = sorted(species)
        keys = self._representation.get_keys(species)
        inner = self._representation.inner_size()
        T = np.zeros((self.size(), len(keys) * inner))
        kid = {(int(a), int(b)): i for i, (a, b) in enumerate(keys)}
        for r, v in enumerate(self.values):
            for key, blk in v.items():
                T[r, kid[key] * inner:(kid[key] + 1) * inner] = blk
        return T

    def get_features(self):
        return self.dense(self.get_species())

    # --- serialisation in the reference's format (models/sparse_points.py,
    # models/sparse_points.hh:456-498): per central species, per key, the
    # rows of the points that have the key, with their index in the species
    def _get_init_params(self):
        return dict(representation=self._representation)

    def _get_data(self):
        inner = self._representation.inner_size()
        species = sorted(set(self.species))
        counters = [[z, 0] for z in range(130)]
        values, indices, keys_sp, all_keys = [], [], [], set()
        for sp in species:
            points = [i for i, s in enumerate(self.species) if s == sp]
            counters[sp][1] = len(points)
            per_key = {}
            for local, i in enumerate(points):
                for key, blk in self.values[i].items():
                    idx, val = per_key.setdefault(tuple(int(k) for k in key), ([], []))
                    idx.append(local)
                    val.extend(float(x) for x in blk)
            ks = sorted(per_key)
            all_keys.update(ks)
            values.append([sp, [[list(k), per_key[k][1]] for k in ks]])
            indices.append([sp, [[list(k), per_key[k][0]] for k in ks]])
            keys_sp.append([sp, [list(k) for k in ks]])
        return dict(sparse_points=dict(
            name="rascal::SparsePointsBlockSparse<rascal::CalculatorSphericalInvariants>",
            values=values, indices=indices, counters=counters, inner_size=inner, center_species=species,
            keys=[list(k) for k in sorted(all_keys)], keys_sp=keys_sp))

    def _set_data(self, data):
        d = data["sparse_points"]
        inner = int(d["inner_size"])
        if inner != self._representation.inner_size():
            raise RuntimeError("sparse points of inner size %d do not match the representation (%d)"
                               % (inner, self._representation.inner_size()))
        counts = {int(z): int(c) for z, c in d["counters"]}
        indices = {int(sp): v for sp, v in d["indices"]}
        self.species, self.values = [], []
        for sp, per_key in sorted((int(sp), v) for sp, v in d["values"]):
            points = [dict() for _ in range(counts.get(sp, 0))]
            idx_of = {tuple(int(x) for x in k): idx for k, idx in indices[sp]}
            for key, flat in per_key:
                key = tuple(int(x) for x in key)
                flat = np.asarray(flat, dtype=float).reshape(-1, inner)
                for r, local in enumerate(idx_of[key]):
                    points[int(local)][key] = flat[r].copy()
            self.species.extend([sp] * len(points))
            self.values.extend(points)
        self._models = {}


class Kernel:
    """GAP kernel (models/kernels.py:16-164), Sparse only. Every matrix is
    computed on the GPU in FP64 through a GAP model handle with zero
    weights:

      kernel(sparse_points)                     K_MM
      kernel(managers, sparse_points)           K_NM energy rows
      kernel(managers, sparse_points, grad=(True, False), compute_neg_stress)
                                                K_NM gradient (+ stress) rows
    """

    def __init__(self, representation, name="GAP", kernel_type="Sparse", target_type="Structure", zeta=2,
                 **kwargs):
        if name not in ("GAP", "Cosine"):
            raise RuntimeError("Kernel name must be one of: Cosine, GAP.")
        if not (isinstance(zeta, (int, np.integer)) and zeta > 0):
            raise ValueError("The given zeta has to be a positive integer.")
        if name != "GAP" or kernel_type != "Sparse":
            raise NotImplementedError("only the sparse GAP kernel is on the B200 path")
        if target_type not in ("Structure", "Atom"):
            raise RuntimeError("Given target_type " + str(target_type) + " is not known."
                               " It is either 'Structure' or 'Atom')")
        self._representation = representation
        self.name = name
        self.kernel_type = kernel_type
        self.target_type = target_type
        self.zeta = int(zeta)

    def _get_init_params(self):
        return dict(representation=self._representation, name=self.name, kernel_type=self.kernel_type,
                    target_type=self.target_type, zeta=self.zeta)

    def _get_data(self):
        return dict()

    def _set_data(self, data):
        pass

    def _model(self, sparse_points):
        """A zero-weight model holding the sparse points on the device, kept
        with the sparse points until they change."""
        key = (id(self._representation), self.zeta)
        model = sparse_points._models.get(key)
        if model is None:
            model = GAPModel(self._representation, sparse_points, None, self.zeta)
            sparse_points._models[key] = model
        return model

    def __call__(self, X, Y=None, grad=(False, False), compute_neg_stress=False):
        if Y is None and grad == (False, False):
            if not isinstance(X, SparsePoints):
                raise NotImplementedError("the sparse kernel of a single argument needs SparsePoints")
            model = self._model(X)
            out = np.zeros((X.size(), X.size()))
            if X.size():
                N.check(N.lib().rgpu_sparse_kernel_mm(model.handle, N.ptr(out, N.c_dbl_p)))
            return out
        if not isinstance(Y, SparsePoints):
            raise NotImplementedError("the sparse kernel needs SparsePoints as its second argument")
        st = X.structures if isinstance(X, AtomsList) else X
        model = self._model(Y)
        if grad == (True, False):
            n_c = X.n_centers() if isinstance(X, AtomsList) else st.n_atoms
            rows = 3 * n_c + (6 * st.n_structures if compute_neg_stress else 0)
            out = np.zeros((rows, Y.size()))
            N.check(N.lib().rgpu_sparse_kernel_derivative(model.handle, st.handle, int(bool(compute_neg_stress)),
                                                          N.ptr(out, N.c_dbl_p)))
            return out
        if grad == (False, False):
            atom = self.target_type == "Atom"
            rows = (X.n_centers() if isinstance(X, AtomsList) else st.n_atoms) if atom else st.n_structures
            out = np.zeros((rows, Y.size()))
            N.check(N.lib().rgpu_sparse_kernel(model.handle, st.handle, int(atom), N.ptr(out, N.c_dbl_p)))
            return out
        raise NotImplementedError("The configuration: {} is not implemented for kernel {} in {} mode.".format(
            grad, self.name, self.kernel_type))


class GAPModel:
    """Device copy of a sparse GAP model (one rgpu_gap_model handle)."""

    def __init__(self, representation, sparse_points, weights, zeta, self_contributions=None):
        self.representation = representation
        self.species = sparse_points.get_species()
        T = N.f64(sparse_points.dense(self.species))
        w = None
        if weights is not None:
            w = N.f64(np.asarray(weights).reshape(-1))
            if len(w) != sparse_points.size():
                raise ValueError("weights size mismatch {}!={}".format(len(w), sparse_points.size()))
        sp = N.i32(self.species)
        sps = N.i32(sparse_points.species)
        sc = N.f64([(self_contributions or {}).get(s, 0.) for s in self.species])
        h = ctypes.c_void_p()
        N.check(N.lib().rgpu_gap_model_create(representation.handle, len(sp), N.ptr(sp, N.c_int_p), len(sps),
                                              N.ptr(sps, N.c_int_p), N.ptr(T, N.c_dbl_p), N.ptr(w, N.c_dbl_p),
                                              int(zeta), N.ptr(sc, N.c_dbl_p), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def predict(self, structures, precision="fp32", energies=True, forces=True):
        """(energies per structure, forces N x 3) for a StructureSet."""
        E = np.zeros(structures.n_structures) if energies else None
        F = np.zeros((structures.n_atoms, 3)) if forces else None
        N.check(N.lib().rgpu_gap_predict(self._h, structures.handle, _PREC[precision], N.ptr(E, N.c_dbl_p),
                                         N.ptr(F, N.c_dbl_p)))
        return E, F

    def predict_stress(self, structures, precision="fp32"):
        """(energies, forces, negative stress n_structures x 6 in the Voigt
        order xx, yy, zz, yz, xz, xy) for a StructureSet."""
        E = np.zeros(structures.n_structures)
        F = np.zeros((structures.n_atoms, 3))
        NS = np.zeros((structures.n_structures, 6))
        N.check(N.lib().rgpu_gap_predict_stress(self._h, structures.handle, _PREC[precision], N.ptr(E, N.c_dbl_p),
                                                N.ptr(F, N.c_dbl_p), N.ptr(NS, N.c_dbl_p)))
        return E, F, NS

    def md_step(self, structures, positions, stress=False):
        """One MD step on `structures` with new `positions` (n_atoms x 3,
        inside the cells), FP32 path: (energies, forces, negative stress or
        None). After the first call the step replays a recorded CUDA graph
        (rgpu_md_step)."""
        pos = N.f64(positions)
        E = np.zeros(structures.n_structures)
        F = np.zeros((structures.n_atoms, 3))
        NS = np.zeros((structures.n_structures, 6)) if stress else None
        N.check(N.lib().rgpu_md_step(self._h, structures.handle, N.ptr(pos, N.c_dbl_p), N.ptr(E, N.c_dbl_p),
                                     N.ptr(F, N.c_dbl_p), N.ptr(NS, N.c_dbl_p)))
        structures.batch = dict(structures.batch, positions=pos)
        return E, F, NS

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and N._lib is not None:
            N._lib.rgpu_gap_model_destroy(h)
            self._h = None


class KRR:
    """Sparse GAP model: predictions of energies and forces
    (bindings/rascal/models/krr.py:12-166)."""

    def __init__(self, weights, kernel, X_train, self_contributions, description="KRR potential model",
                 units=None, precision="fp64"):
        self.weights = np.asarray(weights, dtype=float)
        self.kernel = kernel
        self.X_train = X_train
        self.self_contributions = self_contributions
        self.target_type = kernel.target_type
        self.description = description
        self.units = dict(units or {})
        self.units.setdefault("energy", "eV")
        self.units.setdefault("length", "AA")
        self.precision = precision
        self._model = None

    def _get_init_params(self):
        return dict(weights=self.weights, kernel=self.kernel, X_train=self.X_train,
                    self_contributions=self.self_contributions, description=self.description,
                    units=self.units.copy())

    def _get_data(self):
        return dict()

    def _set_data(self, data):
        pass

    def get_representation_calculator(self):
        return self.kernel._representation

    def _gap(self):
        if self._model is None:
            self._model = GAPModel(self.kernel._representation, self.X_train, self.weights.reshape(-1),
                                   self.kernel.zeta, self.self_contributions)
        return self._model

    def _structures(self, managers):
        if isinstance(managers, AtomsList):
            return managers.structures
        if isinstance(managers, StructureSet):
            return managers
        return StructureSet(frames_to_batch(managers))

    def predict(self, managers, KNM=None):
        if KNM is not None:
            Y0 = self._baseline(managers)
            return Y0 + np.dot(KNM, self.weights).reshape(-1)
        if self.target_type != "Structure":
            raise NotImplementedError("per-atom targets are not on the B200 path")
        E, _ = self._gap().predict(self._structures(managers), self.precision, forces=False)
        return E

    def predict_forces(self, managers, KNM=None):
        if self.kernel.kernel_type != "Sparse":
            raise NotImplementedError("force prediction only implemented for kernels with kernel_type=='Sparse'")
        if KNM is not None:
            return -np.dot(KNM, self.weights).reshape((-1, 3))
        _, F = self._gap().predict(self._structures(managers), self.precision, energies=False)
        return F

    def predict_energy_forces(self, managers):
        return self._gap().predict(self._structures(managers), self.precision)

    def predict_stress(self, managers, KNM=None):
        """Stress per structure in the Voigt order xx, yy, zz, yz, xz, xy
        (bindings/rascal/models/krr.py:168-210): minus the negative stress of
        compute_sparse_kernel_neg_stress."""
        if self.kernel.kernel_type != "Sparse":
            raise NotImplementedError("stress prediction only implemented for kernels with kernel_type=='Sparse'")
        st = self._structures(managers)
        if KNM is not None:
            if 6 * st.n_structures != KNM.shape[0]:
                raise ValueError("KNM size mismatch {}!={}".format(6 * st.n_structures, KNM.shape[0]))
            return -np.dot(KNM, self.weights).reshape((st.n_structures, 6))
        _, _, NS = self._gap().predict_stress(st, self.precision)
        return -NS

    def _baseline(self, managers):
        st = self._structures(managers)
        b = st.batch
        Y0 = np.zeros(st.n_structures)
        for i in range(st.n_structures):
            for z in b["numbers"][b["atom_offsets"][i]:b["atom_offsets"][i + 1]]:
                Y0[i] += self.self_contributions.get(int(z), 0.)
        return Y0


def compute_sparse_kernel_gradients(representation, kernel, managers, sparse_points, weights,
                                    precision="fp64"):
    """Gradients of the GAP energy w.r.t. positions, N_atoms x 3
    (models/sparse_kernel_predict.hh:206-266)."""
    model = GAPModel(representation, sparse_points, np.asarray(weights).reshape(-1), kernel.zeta)
    st = managers.structures if isinstance(managers, AtomsList) else managers
    _, F = model.predict(st, precision, energies=False)
    return -F


def _frame_numbers(frame):
    return _frame_arrays(frame)[1]


def compute_KNM(frames, X_sparse, kernel, soap):
    """Energy rows of the kernel (one per structure) stacked over its
    gradient rows (three per atom, structure after structure)
    (bindings/rascal/models/krr.py:246-343). All frames go through one
    batched call of each kernel on the GPU. A frame none of whose species
    has sparse points keeps zero rows: the reference computes each frame
    separately, so its early return for such a frame
    (models/sparse_kernels.hh:347-349) touches no other frame."""
    frames = list(getattr(frames, "iterable", frames))
    n_at = np.array([len(_frame_numbers(f)) for f in frames], dtype=np.int64)
    n_struct = len(frames)
    stride = np.concatenate([[0], np.cumsum(3 * n_at)]) + n_struct
    KNM = np.zeros((n_struct + int(3 * n_at.sum()), X_sparse.size()))
    sparse_species = set(X_sparse.species)
    good = [i for i, f in enumerate(frames) if sparse_species & set(int(z) for z in _frame_numbers(f))]
    if not good:
        return KNM
    feat = soap.transform([frames[i] for i in good])
    en = kernel(feat, X_sparse)
    grad = kernel(feat, X_sparse, grad=(True, False))
    g0 = 0
    for k, i in enumerate(good):
        KNM[i] = en[k]
        KNM[stride[i]:stride[i + 1]] = grad[g0:g0 + 3 * n_at[i]]
        g0 += 3 * n_at[i]
    return KNM


def train_gap_model(kernel, frames, KNM_, X_sparse, y_train, self_contributions, grad_train=None,
                    lambdas=None, jitter=1e-8):
    """Sparse GAP (subset of regressors) fit (bindings/rascal/models/krr.py:
    346-477): weights = lstsq(K_MM + K_NM^T K_NM, K_NM^T y) with K_NM and y
    scaled by the regularisation lambdas[0] / std(y) * sqrt(n_atoms) for
    the energy rows and lambdas[1] / std(y) for the gradient rows, after the
    self contributions are taken from y. K_MM comes from the GPU; the
    normal equations are solved on the host in FP64, as in the reference."""
    KMM = kernel(X_sparse)
    Y = np.array(y_train, dtype=float).reshape((-1, 1))
    KNM = np.array(KNM_, dtype=float)
    n_struct = Y.shape[0]
    n_atoms = np.zeros(n_struct)
    Y0 = np.zeros((n_struct, 1))
    for i, frame in enumerate(frames):
        z = _frame_numbers(frame)
        n_atoms[i] = len(z)
        for sp in z:
            Y0[i] += self_contributions[int(sp)]
    Y = Y - Y0
    delta = np.std(Y)
    scale = lambdas[0] / delta * np.sqrt(n_atoms)[:, None]
    KNM[:n_struct] /= scale
    Y /= scale
    if grad_train is not None:
        KNM[n_struct:] /= lambdas[1] / delta
        F = np.array(grad_train, dtype=float).reshape((-1, 1)) / (lambdas[1] / delta)
        Y = np.vstack([Y, F])
    KMM[np.diag_indices_from(KMM)] += jitter
    K = KMM + KNM.T @ KNM
    Y = KNM.T @ Y
    weights = np.linalg.lstsq(K, Y, rcond=None)[0]
    return KRR(weights, kernel, X_sparse, self_contributions)


def gap_energy(positions, model, structures):
    """Energies of `structures` at `positions` (torch tensor, n_atoms x 3,
    FP64, on a CUDA device or the host) through the FP32 adjoint path,
    differentiable with respect to the positions.

    The forward computes the energies only and leaves the neighbour list,
    the features and W = alpha zeta k^(zeta-1) on the device; the backward
    runs the second GEMM, the power-spectrum backward and the pair adjoint
    (rgpu_gap_forward_dev / rgpu_gap_backward_dev), so
    torch.autograd.grad(E.sum(), positions) gives -forces, the reference's
    KRR.predict_forces (bindings/rascal/models/krr.py:123-166). CUDA
    positions and gradients stay on the device."""
    return _gap_function().apply(positions, model, structures)


_GAPFn = None


def _gap_function():
    global _GAPFn
    if _GAPFn is None:
        import torch

        def _order(structures):
            """The library's stream for these structures, and a helper that
            makes one stream wait for work enqueued on another."""
            ext = torch.cuda.ExternalStream(structures.stream())

            def after(waiter, producer):
                ev = torch.cuda.Event()
                ev.record(producer)
                waiter.wait_event(ev)
            return ext, after

        class GAPEnergy(torch.autograd.Function):
            """E(r) forward; dE/dr from the adjoint kernels (no stored dX/dr)."""

            @staticmethod
            def forward(ctx, positions, model, structures):
                dev = positions.device if positions.is_cuda else torch.device("cuda", torch.cuda.current_device())
                pos = positions.detach().to(dev, torch.float64).contiguous()
                if pos.shape != (structures.n_atoms, 3):
                    raise ValueError("positions must be n_atoms x 3")
                E = torch.empty(structures.n_structures, dtype=torch.float64, device=dev)
                ext, after = _order(structures)
                after(ext, torch.cuda.current_stream(dev))  # positions are ready
                N.check(N.lib().rgpu_gap_forward_dev(model.handle, structures.handle, pos.data_ptr(),
                                                     E.data_ptr()))
                after(torch.cuda.current_stream(dev), ext)
                ctx.model = model
                ctx.structures = structures
                ctx.in_device = positions.device
                ctx.in_dtype = positions.dtype
                return E.to(positions.device, positions.dtype)

            @staticmethod
            def backward(ctx, gE):
                structures = ctx.structures
                dev = torch.device("cuda", torch.cuda.current_device()) if not gE.is_cuda else gE.device
                g = gE.detach().to(dev, torch.float64).contiguous()
                out = torch.empty((structures.n_atoms, 3), dtype=torch.float64, device=dev)
                ext, after = _order(structures)
                after(ext, torch.cuda.current_stream(dev))
                N.check(N.lib().rgpu_gap_backward_dev(ctx.model.handle, structures.handle, g.data_ptr(),
                                                      out.data_ptr()))
                after(torch.cuda.current_stream(dev), ext)
                return out.to(ctx.in_device, ctx.in_dtype), None, None

        _GAPFn = GAPEnergy
    return _GAPFn
