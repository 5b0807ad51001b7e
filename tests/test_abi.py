"""The C-ABI library: it loads, exports every entry point of
include/rascal_b200.h, and its host-side FP64 spline builder reproduces the
oracle's table bit for bit (no GPU needed for these)."""
import os
import re

import numpy as np
import pytest

import librascal_b200 as rb
from librascal_b200 import _native
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "rascal_b200.h")).read()
    decl = r"^\s*(?:rgpu_status|const char \*|int|int64_t)\s+(rgpu_\w+)\s*\("
    return sorted(set(re.findall(decl, text, flags=re.M)))


def test_library_exports_every_header_symbol():
    lib = _native.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_native.SIGNATURES), set(names) ^ set(_native.SIGNATURES)
    assert lib.rgpu_version() >= 1


@pytest.mark.parametrize("rc,sw,n,l,sigma,acc", [
    (4.0, 0.5, 6, 4, 0.3, 1e-8),
    (5.0, 0.5, 8, 6, 0.4, 1e-8),
    (6.0, 0.5, 12, 9, 0.5, 1e-8),
    (3.0, 1.0, 4, 3, 0.2, 1e-8),
    (3.5, 0.5, 6, 2, 0.5, 1e-6),
])
def test_spline_table_matches_oracle_bitwise(rc, sw, n, l, sigma, acc):
    calc = rb.SphericalInvariants(interaction_cutoff=rc, cutoff_smooth_width=sw, max_radial=n,
                                  max_angular=l, gaussian_sigma_type="Constant",
                                  gaussian_sigma_constant=sigma,
                                  optimization=dict(Spline=dict(accuracy=acc)))
    g, y, y2 = calc.spline_table()
    oc = O.Calculator(rc, sw, n, l, sigma, spline=True, accuracy=acc)
    og, oy, oy2 = oc.spline_table()
    assert g.shape == og.shape and y.shape == oy.shape
    assert np.array_equal(g, og)
    assert np.array_equal(y, oy)
    assert np.array_equal(y2, oy2)


def test_invalid_hypers_raise_like_the_reference():
    with pytest.raises(RuntimeError, match="Smearing type"):
        rb.SphericalInvariants(4.0, 0.5, 4, 3, gaussian_sigma_type="PerSpecies")
    with pytest.raises(RuntimeError, match="PowerSpectrum"):
        rb.SphericalInvariants(4.0, 0.5, 4, 3, gaussian_sigma_type="Constant", soap_type="BiSpectrum")
    with pytest.raises(RuntimeError, match="max_angular"):
        rb.SphericalInvariants(4.0, 0.5, 4, 13, gaussian_sigma_type="Constant")
    with pytest.raises(ValueError):
        rb.SphericalInvariants(4.0, 0.5, 4, 3, gaussian_sigma_type="Constant",
                               optimization=dict(RadialDimReduction={}))


def test_calculator_name_is_prefix_plus_hypers():
    calc = rb.SphericalInvariants(4.0, 0.5, 4, 3, gaussian_sigma_type="Constant")
    name = calc.get_name()
    assert name.startswith("sphericalinvariants_{")
    assert '"max_radial":4' in name
