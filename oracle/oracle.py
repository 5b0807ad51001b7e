"""ctypes wrapper around the CPU FP64 oracle (``rascal_oracle.cpp``).

TEST INFRASTRUCTURE ONLY. The oracle is a plain CPU restatement of the
reference's descriptor hot path; tests, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg use it as the checker. The product package
never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "librascal_oracle.so")
_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_long_p = ctypes.POINTER(ctypes.c_long)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)


def build():
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_hyp1f1.restype = ctypes.c_double
        L.orc_hyp1f1.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_calc_new.restype = ctypes.c_void_p
        L.orc_calc_new.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] * 3 + [
            ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_calc_free.argtypes = [ctypes.c_void_p]
        L.orc_calc_set_radial_scaling.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 3
        L.orc_calc_spline_size.argtypes = [ctypes.c_void_p]
        L.orc_calc_spline_table.argtypes = [ctypes.c_void_p, c_dbl_p, c_dbl_p, c_dbl_p]
        L.orc_calc_gto.argtypes = [ctypes.c_void_p, c_dbl_p, c_dbl_p, c_dbl_p]
        L.orc_calc_radial.argtypes = [ctypes.c_void_p, ctypes.c_double, c_dbl_p, c_dbl_p]
        L.orc_spherical_harmonics.argtypes = [ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p]
        L.orc_hyp1f1_table.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, c_dbl_p, ctypes.c_int, ctypes.c_double,
                                       c_dbl_p, c_dbl_p]
        L.orc_run.restype = ctypes.c_void_p
        L.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_int, c_long_p, c_dbl_p, c_int_p,
                              c_dbl_p, c_int_p, c_u8_p, ctypes.c_int, c_int_p,
                              ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_run_free.argtypes = [ctypes.c_void_p]
        L.orc_run_n_centers.restype = ctypes.c_long
        L.orc_run_n_centers.argtypes = [ctypes.c_void_p]
        L.orc_run_n_pairs.restype = ctypes.c_long
        L.orc_run_n_pairs.argtypes = [ctypes.c_void_p]
        L.orc_run_dim.argtypes = [ctypes.c_void_p]
        L.orc_run_centers.argtypes = [ctypes.c_void_p, c_int_p, c_int_p, c_long_p]
        L.orc_run_pairs.argtypes = [ctypes.c_void_p, c_int_p, c_int_p, c_int_p, c_dbl_p, c_dbl_p, c_int_p]
        for f in ("orc_run_expansion", "orc_run_expansion_grad",
                  "orc_run_powerspectrum", "orc_run_powerspectrum_grad"):
            getattr(L, f).argtypes = [ctypes.c_void_p, c_dbl_p]
        L.orc_run_gap.argtypes = [ctypes.c_void_p, ctypes.c_int, c_int_p, c_dbl_p, c_dbl_p,
                                  ctypes.c_int, c_dbl_p, c_dbl_p]
        L.orc_run_gap_stress.argtypes = [ctypes.c_void_p, ctypes.c_int, c_int_p, c_dbl_p, c_dbl_p,
                                         ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p]
        L.orc_run_kernel_nm.argtypes = [ctypes.c_void_p, ctypes.c_int, c_int_p, c_dbl_p, ctypes.c_int,
                                         ctypes.c_int, c_dbl_p]
        L.orc_run_kernel_nm_derivative.argtypes = [ctypes.c_void_p, ctypes.c_int, c_int_p, c_dbl_p,
                                                    ctypes.c_int, ctypes.c_int, c_dbl_p]
        L.orc_kernel_mm.argtypes = [ctypes.c_int, ctypes.c_int, c_int_p, c_dbl_p, ctypes.c_int, c_dbl_p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def hyp1f1(a, b, z, derivative=False, mmax=200, tol=1e-15):
    return lib().orc_hyp1f1(a, b, z, int(derivative), mmax, tol)


def spherical_harmonics(lmax, direction, gradients=False):
    K = (lmax + 1) ** 2
    d = np.ascontiguousarray(direction, dtype=np.float64)
    Y = np.zeros(K)
    dY = np.zeros((3, K)) if gradients else None
    lib().orc_spherical_harmonics(lmax, _p(d, c_dbl_p), _p(Y, c_dbl_p),
                                  _p(dY, c_dbl_p) if gradients else None)
    return (Y, dY) if gradients else Y


class Calculator:
    """GTO / ShiftedCosine / constant-sigma expansion parameters."""

    def __init__(self, interaction_cutoff, cutoff_smooth_width, max_radial,
                 max_angular, gaussian_sigma_constant, spline=True,
                 accuracy=1e-8, normalize=True, radial_scaling=None):
        """radial_scaling: None for the shifted cosine, or a dict with rate,
        scale and exponent for the RadialScaling cutoff."""
        self.rc = float(interaction_cutoff)
        self.n = int(max_radial)
        self.l = int(max_angular)
        err = ctypes.create_string_buffer(512)
        self.h = lib().orc_calc_new(self.rc, float(cutoff_smooth_width),
                                    float(gaussian_sigma_constant), self.n, self.l,
                                    int(spline), float(accuracy), int(normalize), err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        if radial_scaling is not None:
            lib().orc_calc_set_radial_scaling(self.h, float(radial_scaling["rate"]),
                                              float(radial_scaling["scale"]), float(radial_scaling["exponent"]))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_calc_free(self.h)
            self.h = None

    def spline_table(self):
        G = lib().orc_calc_spline_size(self.h)
        W = self.n * (self.l + 1)
        grid = np.zeros(G)
        y = np.zeros((G, W))
        y2h = np.zeros((G, W))
        lib().orc_calc_spline_table(self.h, _p(grid, c_dbl_p), _p(y, c_dbl_p), _p(y2h, c_dbl_p))
        return grid, y, y2h

    def gto(self):
        on = np.zeros((self.n, self.n))
        cf = np.zeros(self.n)
        fb = np.zeros(self.n)
        lib().orc_calc_gto(self.h, _p(on, c_dbl_p), _p(cf, c_dbl_p), _p(fb, c_dbl_p))
        return on, cf, fb

    def radial(self, r):
        W = self.n * (self.l + 1)
        RI = np.zeros(W)
        dRI = np.zeros(W)
        lib().orc_calc_radial(self.h, float(r), _p(RI, c_dbl_p), _p(dRI, c_dbl_p))
        return RI.reshape(self.n, self.l + 1), dRI.reshape(self.n, self.l + 1)


class Run:
    """Neighbour list, expansion, power spectrum (and gradients) of a batch.

    ``batch`` is a dict with the flat arrays ``atom_offsets`` (S+1),
    ``positions`` (N,3), ``numbers`` (N), ``cells`` (S,3,3; rows are lattice
    vectors), ``pbc`` (S,3) and optionally ``center_atoms_mask`` (N).
    """

    def __init__(self, calc, batch, species, gradients=False):
        self.calc = calc
        off = np.ascontiguousarray(batch["atom_offsets"], dtype=np.int64)
        pos = np.ascontiguousarray(batch["positions"], dtype=np.float64)
        typ = np.ascontiguousarray(batch["numbers"], dtype=np.int32)
        cel = np.ascontiguousarray(batch["cells"], dtype=np.float64)
        pbc = np.ascontiguousarray(batch["pbc"], dtype=np.int32)
        mask = batch.get("center_atoms_mask")
        if mask is not None:
            mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self.species = np.ascontiguousarray(sorted(set(int(s) for s in species)), dtype=np.int32)
        err = ctypes.create_string_buffer(512)
        self.h = lib().orc_run(calc.h, len(off) - 1, _p(off, c_long_p), _p(pos, c_dbl_p),
                               _p(typ, c_int_p), _p(cel, c_dbl_p), _p(pbc, c_int_p),
                               _p(mask, c_u8_p) if mask is not None else None,
                               len(self.species), _p(self.species, c_int_p), int(gradients),
                               err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.gradients = gradients
        self.n_struct = len(off) - 1
        self.n_atoms = int(off[-1])
        self.n_centers = lib().orc_run_n_centers(self.h)
        self.n_pairs = lib().orc_run_n_pairs(self.h)
        self.D = lib().orc_run_dim(self.h)
        self.S = len(self.species)
        self.K = (calc.l + 1) ** 2

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_run_free(self.h)
            self.h = None

    def centers(self):
        ca = np.zeros(self.n_centers, dtype=np.int32)
        cs = np.zeros(self.n_centers, dtype=np.int32)
        po = np.zeros(self.n_centers + 1, dtype=np.int64)
        lib().orc_run_centers(self.h, _p(ca, c_int_p), _p(cs, c_int_p), _p(po, c_long_p))
        return ca, cs, po

    def pairs(self):
        P = self.n_pairs
        ce = np.zeros(P, dtype=np.int32)
        jg = np.zeros(P, dtype=np.int32)
        sh = np.zeros((P, 3), dtype=np.int32)
        di = np.zeros(P)
        dr = np.zeros((P, 3))
        jt = np.zeros(P, dtype=np.int32)
        lib().orc_run_pairs(self.h, _p(ce, c_int_p), _p(jg, c_int_p), _p(sh, c_int_p),
                            _p(di, c_dbl_p), _p(dr, c_dbl_p), _p(jt, c_int_p))
        return dict(center=ce, j=jg, shift=sh, distance=di, direction=dr, j_type=jt)

    def expansion(self):
        out = np.zeros((self.n_centers, self.S, self.calc.n, self.K))
        lib().orc_run_expansion(self.h, _p(out, c_dbl_p))
        return out

    def expansion_gradient(self):
        out = np.zeros((self.n_pairs, self.S, 3, self.calc.n, self.K))
        if lib().orc_run_expansion_grad(self.h, _p(out, c_dbl_p)) != 0:
            raise RuntimeError("gradients were not computed")
        return out

    def power_spectrum(self):
        out = np.zeros((self.n_centers, self.D))
        lib().orc_run_powerspectrum(self.h, _p(out, c_dbl_p))
        return out

    def power_spectrum_gradient(self):
        out = np.zeros((self.n_pairs, 3, self.D))
        if lib().orc_run_powerspectrum_grad(self.h, _p(out, c_dbl_p)) != 0:
            raise RuntimeError("gradients were not computed")
        return out

    def gap_stress(self, sparse_species, T, alpha, zeta):
        """Energies, forces and the negative stress per structure (Voigt xx,
        yy, zz, yz, xz, xy; the reference's compute_sparse_kernel_neg_stress)."""
        sps = np.ascontiguousarray(sparse_species, dtype=np.int32)
        T = np.ascontiguousarray(T, dtype=np.float64)
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        E = np.zeros(self.n_struct)
        F = np.zeros((self.n_atoms, 3))
        NS = np.zeros((self.n_struct, 6))
        rc = lib().orc_run_gap_stress(self.h, len(sps), _p(sps, c_int_p), _p(T, c_dbl_p), _p(al, c_dbl_p),
                                      int(zeta), _p(E, c_dbl_p), _p(F, c_dbl_p), _p(NS, c_dbl_p))
        if rc != 0:
            raise RuntimeError("the stress needs a run with gradients")
        return E, F, NS

    def gap(self, sparse_species, T, alpha, zeta, forces=True):
        """Energies (per structure, no baseline) and forces (-dE/dr)."""
        sps = np.ascontiguousarray(sparse_species, dtype=np.int32)
        T = np.ascontiguousarray(T, dtype=np.float64)
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        E = np.zeros(self.n_struct)
        F = np.zeros((self.n_atoms, 3)) if forces else None
        rc = lib().orc_run_gap(self.h, len(sps), _p(sps, c_int_p), _p(T, c_dbl_p), _p(al, c_dbl_p),
                               int(zeta), _p(E, c_dbl_p), _p(F, c_dbl_p) if forces else None)
        if rc != 0:
            raise RuntimeError("forces need a run with gradients")
        return (E, F) if forces else E

    def kernel_nm(self, sparse_species, T, zeta, target_type="Structure"):
        """K_NM energy rows: per structure, or per centre for target "Atom"."""
        sps = np.ascontiguousarray(sparse_species, dtype=np.int32)
        T = np.ascontiguousarray(T, dtype=np.float64)
        atom = target_type == "Atom"
        out = np.zeros((self.n_centers if atom else self.n_struct, len(sps)))
        lib().orc_run_kernel_nm(self.h, len(sps), _p(sps, c_int_p), _p(T, c_dbl_p), int(zeta), int(atom),
                                _p(out, c_dbl_p))
        return out

    def kernel_nm_derivative(self, sparse_species, T, zeta, compute_neg_stress=False):
        """K_NM gradient rows: 3 per centre (x, y, z), then 6 negative-stress
        rows per structure (Voigt xx, yy, zz, yz, xz, xy) when asked."""
        sps = np.ascontiguousarray(sparse_species, dtype=np.int32)
        T = np.ascontiguousarray(T, dtype=np.float64)
        rows = 3 * self.n_centers + (6 * self.n_struct if compute_neg_stress else 0)
        out = np.zeros((rows, len(sps)))
        rc = lib().orc_run_kernel_nm_derivative(self.h, len(sps), _p(sps, c_int_p), _p(T, c_dbl_p), int(zeta),
                                                int(compute_neg_stress), _p(out, c_dbl_p))
        if rc != 0:
            raise RuntimeError("kernel gradients need a run with gradients")
        return out


def kernel_mm(sparse_species, T, zeta):
    """K_MM: (T_a . T_b)^zeta within a species, 0 across species."""
    sps = np.ascontiguousarray(sparse_species, dtype=np.int32)
    T = np.ascontiguousarray(T, dtype=np.float64)
    out = np.zeros((len(sps), len(sps)))
    lib().orc_kernel_mm(len(sps), T.shape[1], _p(sps, c_int_p), _p(T, c_dbl_p), int(zeta), _p(out, c_dbl_p))
    return out
