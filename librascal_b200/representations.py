"""SphericalInvariants / SphericalExpansion on the B200 path.

Same constructor arguments and hypers dict as the reference wrappers
(bindings/rascal/representations/spherical_invariants.py:209-337,
spherical_expansion.py, base.py:83 for the default spline optimisation).
The hypers are passed to the C ABI as JSON, exactly as the reference passes
them to its C++ calculator.
"""
import ctypes
import json
from copy import deepcopy
from itertools import product

import numpy as np

from . import _native as N
from .neighbourlist import AtomsList


def cutoff_function_dict_switch(cutoff_function_type, **kwargs):
    if cutoff_function_type == "ShiftedCosine":
        return dict(type=cutoff_function_type,
                    cutoff=dict(value=kwargs["interaction_cutoff"], unit="AA"),
                    smooth_width=dict(value=kwargs["cutoff_smooth_width"], unit="AA"))
    if cutoff_function_type == "RadialScaling":
        return dict(type=cutoff_function_type,
                    cutoff=dict(value=kwargs["interaction_cutoff"], unit="AA"),
                    smooth_width=dict(value=kwargs["cutoff_smooth_width"], unit="AA"),
                    rate=dict(value=kwargs["rate"], unit="AA"),
                    scale=dict(value=kwargs["scale"], unit="AA"),
                    exponent=dict(value=kwargs["exponent"], unit="AA"))
    raise NotImplementedError("cutoff_function: " + cutoff_function_type + " has not been implemented.")


def check_optimization_for_spherical_representations(optimization, optimization_args):
    if optimization_args is not None:
        optimization = dict(Spline=dict(accuracy=optimization_args["accuracy"]))
    if optimization is None:
        optimization = dict(Spline=dict(accuracy=1e-8))
    optimization = deepcopy(optimization)
    if "RadialDimReduction" in optimization and "Spline" not in optimization:
        raise ValueError("Optimization key `RadialDimReduction` can only be used with `Spline`, "
                         "please set the spline arguments in `optimization`")
    return optimization


def get_power_spectrum_index_mapping(sp_pairs, n_max, l_max):
    feat_idx2coeff_idx = {}
    i_feat = 0
    for sp_pair, n1, n2, l in product(sp_pairs, range(n_max), range(n_max), range(l_max)):
        feat_idx2coeff_idx[i_feat] = dict(a=sp_pair[0], b=sp_pair[1], n1=n1, n2=n2, l=l)
        i_feat += 1
    return feat_idx2coeff_idx


class _Calculator:
    """Holds an rgpu_calculator handle."""
    name = None

    def _create(self):
        h = ctypes.c_void_p()
        N.check(N.lib().rgpu_calculator_create(self.name.encode(), json.dumps(self.hypers).encode(),
                                               ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and N._lib is not None:
            N._lib.rgpu_calculator_destroy(h)
            self._h = None

    def spline_table(self):
        """(grid, y, y''h^2/6) of the FP64 radial spline built on the host."""
        G, W = ctypes.c_int32(), ctypes.c_int32()
        N.check(N.lib().rgpu_calculator_spline_shape(self._h, ctypes.byref(G), ctypes.byref(W)))
        grid = np.zeros(G.value)
        y = np.zeros((G.value, W.value))
        y2 = np.zeros((G.value, W.value))
        N.check(N.lib().rgpu_calculator_spline_table(self._h, N.ptr(grid, N.c_dbl_p), N.ptr(y, N.c_dbl_p),
                                                     N.ptr(y2, N.c_dbl_p)))
        return grid, y, y2

    def get_name(self):
        buf = ctypes.create_string_buffer(1 << 16)
        N.check(N.lib().rgpu_calculator_name(self._h, buf, len(buf)))
        return buf.value.decode()

    def transform(self, frames, precision="fp64"):
        """Compute the representation of `frames` (list of ase.Atoms-like
        objects or dicts, or an AtomsList) and return the AtomsList."""
        if not isinstance(frames, AtomsList):
            frames = AtomsList(frames, self.nl_options)
        prec = N.PRECISION_FP64 if precision == "fp64" else N.PRECISION_FP32
        N.check(N.lib().rgpu_compute(self._h, frames.structures.handle, prec,
                                     int(bool(self.hypers.get("compute_gradients", False)))))
        frames._calc = self
        frames._precision = prec
        return frames


class SphericalInvariants(_Calculator):
    """SOAP power spectrum (soap_type="PowerSpectrum") on the B200 path."""

    def __init__(self, interaction_cutoff, cutoff_smooth_width, max_radial, max_angular,
                 gaussian_sigma_type, gaussian_sigma_constant=0.3, cutoff_function_type="ShiftedCosine",
                 soap_type="PowerSpectrum", inversion_symmetry=True, radial_basis="GTO", normalize=True,
                 optimization=None, optimization_args=None, expansion_by_species_method="environment wise",
                 global_species=None, compute_gradients=False, cutoff_function_parameters=dict(),
                 coefficient_subselection=None):
        self.name = "sphericalinvariants"
        self.hypers = dict()
        if global_species is None:
            global_species = []
        elif not isinstance(global_species, list):
            global_species = list(global_species)
        self.update_hyperparameters(
            max_radial=max_radial, max_angular=max_angular, soap_type=soap_type, normalize=normalize,
            inversion_symmetry=inversion_symmetry, expansion_by_species_method=expansion_by_species_method,
            global_species=global_species, compute_gradients=compute_gradients,
            coefficient_subselection=coefficient_subselection)
        if self.hypers["coefficient_subselection"] is None:
            del self.hypers["coefficient_subselection"]
        self.cutoff_function_parameters = deepcopy(cutoff_function_parameters)
        cutoff_function_parameters = dict(cutoff_function_parameters)
        cutoff_function_parameters.update(interaction_cutoff=interaction_cutoff,
                                          cutoff_smooth_width=cutoff_smooth_width)
        cutoff_function = cutoff_function_dict_switch(cutoff_function_type, **cutoff_function_parameters)
        gaussian_density = dict(type=gaussian_sigma_type,
                                gaussian_sigma=dict(value=gaussian_sigma_constant, unit="AA"))
        optimization = check_optimization_for_spherical_representations(optimization, optimization_args)
        radial_contribution = dict(type=radial_basis, optimization=optimization)
        self.update_hyperparameters(cutoff_function=cutoff_function, gaussian_density=gaussian_density,
                                    radial_contribution=radial_contribution)
        if soap_type == "RadialSpectrum":
            self.update_hyperparameters(max_angular=0)
        self.nl_options = [
            dict(name="centers", args=[]),
            dict(name="neighbourlist", args=dict(cutoff=interaction_cutoff)),
            dict(name="centercontribution", args=dict()),
            dict(name="strict", args=dict(cutoff=interaction_cutoff)),
        ]
        self._create()

    def update_hyperparameters(self, **hypers):
        allowed_keys = {
            "interaction_cutoff", "cutoff_smooth_width", "max_radial", "max_angular",
            "gaussian_sigma_type", "gaussian_sigma_constant", "soap_type", "inversion_symmetry",
            "cutoff_function", "normalize", "gaussian_density", "radial_contribution",
            "cutoff_function_parameters", "expansion_by_species_method", "compute_gradients",
            "global_species", "coefficient_subselection"}
        self.hypers.update({k: hypers[k] for k in hypers if k in allowed_keys})

    def inner_size(self):
        n, l = self.hypers["max_radial"], self.hypers["max_angular"]
        return n * n * (l + 1)

    def get_num_coefficients(self, n_species=1):
        return n_species * (n_species + 1) // 2 * self.inner_size()

    def get_keys(self, species):
        species = sorted(set(int(s) for s in species))
        return np.array([[a, b] for i, a in enumerate(species) for b in species[i:]], dtype=np.int32)

    def _get_init_params(self):
        """Constructor arguments, as the reference serialises them
        (spherical_invariants.py:451-480)."""
        gd, cf, rc = self.hypers["gaussian_density"], self.hypers["cutoff_function"], \
            self.hypers["radial_contribution"]
        p = dict(interaction_cutoff=cf["cutoff"]["value"], cutoff_smooth_width=cf["smooth_width"]["value"],
                 max_radial=self.hypers["max_radial"], max_angular=self.hypers["max_angular"],
                 soap_type=self.hypers["soap_type"], inversion_symmetry=self.hypers["inversion_symmetry"],
                 normalize=self.hypers["normalize"],
                 expansion_by_species_method=self.hypers["expansion_by_species_method"],
                 global_species=self.hypers["global_species"], compute_gradients=self.hypers["compute_gradients"],
                 gaussian_sigma_type=gd["type"], gaussian_sigma_constant=gd["gaussian_sigma"]["value"],
                 cutoff_function_type=cf["type"], radial_basis=rc["type"], optimization=rc["optimization"],
                 cutoff_function_parameters=self.cutoff_function_parameters)
        if "coefficient_subselection" in self.hypers:
            p["coefficient_subselection"] = self.hypers["coefficient_subselection"]
        return p

    def _get_data(self):
        return dict()

    def _set_data(self, data):
        pass


class SphericalExpansion(_Calculator):
    """Density expansion coefficients c^i_{a n lm} on the B200 path."""

    def __init__(self, interaction_cutoff, cutoff_smooth_width, max_radial, max_angular,
                 gaussian_sigma_type, gaussian_sigma_constant=0.3, cutoff_function_type="ShiftedCosine",
                 radial_basis="GTO", optimization=None, optimization_args=None,
                 expansion_by_species_method="environment wise", global_species=None,
                 compute_gradients=False, cutoff_function_parameters=dict()):
        self.name = "sphericalexpansion"
        if global_species is None:
            global_species = []
        self.cutoff_function_parameters = deepcopy(cutoff_function_parameters)
        cutoff_function_parameters = dict(cutoff_function_parameters)
        cutoff_function_parameters.update(interaction_cutoff=interaction_cutoff,
                                          cutoff_smooth_width=cutoff_smooth_width)
        optimization = check_optimization_for_spherical_representations(optimization, optimization_args)
        self.hypers = dict(
            interaction_cutoff=interaction_cutoff, cutoff_smooth_width=cutoff_smooth_width,
            max_radial=max_radial, max_angular=max_angular, gaussian_sigma_type=gaussian_sigma_type,
            gaussian_sigma_constant=gaussian_sigma_constant,
            expansion_by_species_method=expansion_by_species_method, global_species=list(global_species),
            compute_gradients=compute_gradients,
            cutoff_function=cutoff_function_dict_switch(cutoff_function_type, **cutoff_function_parameters),
            gaussian_density=dict(type=gaussian_sigma_type,
                                  gaussian_sigma=dict(value=gaussian_sigma_constant, unit="AA")),
            radial_contribution=dict(type=radial_basis, optimization=optimization))
        self.nl_options = [
            dict(name="centers", args=[]),
            dict(name="neighbourlist", args=dict(cutoff=interaction_cutoff)),
            dict(name="centercontribution", args=dict()),
            dict(name="strict", args=dict(cutoff=interaction_cutoff)),
        ]
        self._create()

    def inner_size(self):
        n, l = self.hypers["max_radial"], self.hypers["max_angular"]
        return n * (l + 1) ** 2

    def get_num_coefficients(self, n_species=1):
        return n_species * self.inner_size()

    def get_keys(self, species):
        species = sorted(set(int(s) for s in species))
        return np.array([[a, a] for a in species], dtype=np.int32)

    def _get_init_params(self):
        h = self.hypers
        return dict(interaction_cutoff=h["interaction_cutoff"], cutoff_smooth_width=h["cutoff_smooth_width"],
                    max_radial=h["max_radial"], max_angular=h["max_angular"],
                    gaussian_sigma_type=h["gaussian_sigma_type"],
                    gaussian_sigma_constant=h["gaussian_sigma_constant"],
                    cutoff_function_type=h["cutoff_function"]["type"],
                    radial_basis=h["radial_contribution"]["type"],
                    optimization=h["radial_contribution"]["optimization"],
                    expansion_by_species_method=h["expansion_by_species_method"],
                    global_species=h["global_species"], compute_gradients=h["compute_gradients"],
                    cutoff_function_parameters=self.cutoff_function_parameters)

    def _get_data(self):
        return dict()

    def _set_data(self, data):
        pass
