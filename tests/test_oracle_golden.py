"""Pin the CPU oracle against the reference's own golden data.

Each test mirrors a reference test and uses its tolerance:
  * tests/test_math_hyp1f1.cc:42-113           (15 * DBL_FTOL)
  * tests/test_math_spherical_harmonics.cc:50-100 (|dY| <= 2 * DBL_FTOL)
  * tests/test_calculator.cc:460-496           (expansion, delta 3e-6)
  * tests/test_kernels.cc:68-136               (PowerSpectrum kernels, 1e-10)
"""
import json
import os

import numpy as np
import pytest

from helpers import DBL_FTOL, GOLDEN, batch_from_frames, load_structures, relative_error
from oracle import oracle as O


def test_hyp1f1_known_answers():
    z = np.load(os.path.join(GOLDEN, "hyp1f1.npz"))
    err_v = err_d = 0.0
    for a, b, x, v, d in zip(z["a"], z["b"], z["z"], z["val"], z["der"]):
        val = O.hyp1f1(a, b, x, False, 200, 1e-15)
        der = O.hyp1f1(a, b, x, True, 200, 1e-15)
        err_v = max(err_v, abs((v - val) / v))
        err_d = max(err_d, abs((d - der) / d))
    assert err_v <= 15 * DBL_FTOL
    assert err_d <= 15 * DBL_FTOL


def test_hyp1f1_recursion_matches_direct():
    # tests/test_math_hyp1f1.cc:91-113 with the fixture of tests/test_math.hh:476-515:
    # mean relative difference between recursion and direct evaluation <= 3 DBL_FTOL
    lib = O.lib()
    for rc in [2.0, 3.0, 5.0, 7.0, 8.0]:
        for l_max in [4, 5, 9, 15, 16, 20]:
            for n_max in [4, 5, 9, 15, 16, 20]:
                fac_b = np.array([0.5 * ((rc - 0.5) * max(np.sqrt(n), 1.0) / n_max) ** 2
                                  for n in range(n_max)])
                for r in [1.0, 2.0, 3.0, 4.0, 5.5, 6.5, 7.5, 7.9]:
                    if r >= rc:
                        continue
                    out = []
                    for rec in (0, 1):
                        v = np.zeros(n_max * (l_max + 1))
                        dd = np.zeros(n_max * (l_max + 1))
                        lib.orc_hyp1f1_table(n_max, l_max, r, 0.4, fac_b.ctypes.data_as(O.c_dbl_p),
                                             rec, 1e-14, v.ctypes.data_as(O.c_dbl_p),
                                             dd.ctypes.data_as(O.c_dbl_p))
                        out.append((v, dd))
                    (v0, d0), (v1, d1) = out
                    assert np.mean(np.abs(v0 - v1) / v0) <= 3 * DBL_FTOL
                    assert np.mean(np.abs(d0 - d1) / d0) <= 3 * DBL_FTOL


def test_spherical_harmonics_known_answers():
    z = np.load(os.path.join(GOLDEN, "spherical_harmonics.npz"))
    for lmax, u, Y in zip(z["lmax"], z["unit_vector"], z["harmonics"]):
        mine = O.spherical_harmonics(int(lmax), u)
        assert np.linalg.norm(mine - Y) <= 2 * DBL_FTOL


@pytest.mark.parametrize("lmax", [3, 6])
def test_spherical_harmonics_gradient_fd(lmax):
    # tests/test_math.hh:216-456 with spherical_harmonics_gradient_test.json:
    # the Cartesian gradient of Y_lm(r/|r|) times |r| on the unit sphere.
    rng = np.random.default_rng(1)
    h = 1e-6
    for _ in range(10):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        Y, dY = O.spherical_harmonics(lmax, d, gradients=True)
        for c in range(3):
            e = np.zeros(3)
            e[c] = h
            yp = O.spherical_harmonics(lmax, (d + e) / np.linalg.norm(d + e))
            ym = O.spherical_harmonics(lmax, (d - e) / np.linalg.norm(d - e))
            assert np.allclose((yp - ym) / (2 * h), dY[c], atol=1e-7)


def test_expansion_golden():
    z = np.load(os.path.join(GOLDEN, "expansion_reference.npz"))
    meta = json.loads(str(z["meta"]))
    structs = load_structures()
    # 16 ShiftedCosine and 16 RadialScaling cases, direct and spline
    assert len(meta) == 32
    assert sum(m["radial_scaling"] is not None for m in meta) == 16
    for i, m in enumerate(meta):
        b = batch_from_frames(structs[m["structure"]])
        calc = O.Calculator(m["cutoff"], m["smooth_width"], m["max_radial"], m["max_angular"],
                            m["sigma"], spline=m["spline"], accuracy=m["accuracy"] or 1e-8,
                            radial_scaling=m["radial_scaling"])
        r = O.Run(calc, b, np.unique(b["numbers"]))
        C = r.expansion().reshape(r.n_centers, -1)
        ref = z["features_%d" % i]
        assert C.shape == ref.shape
        err = relative_error(ref, C, 1e-14).max()
        # reference delta is 3e-6; the restatement reproduces it far tighter
        assert err < 1e-9, (m, err)


def test_powerspectrum_kernel_golden():
    z = np.load(os.path.join(GOLDEN, "kernel_reference.npz"))
    meta = json.loads(str(z["meta"]))
    frames = load_structures()[str(z["structures"])]
    b = batch_from_frames(frames)
    S = len(b["atom_offsets"]) - 1
    for i, m in enumerate(meta):
        calc = O.Calculator(m["cutoff"], m["smooth_width"], m["max_radial"], m["max_angular"],
                            m["sigma"], spline=m["spline"], normalize=m["normalize"])
        r = O.Run(calc, b, np.unique(b["numbers"]))
        X = r.power_spectrum()
        _, cs, _ = r.centers()
        kk = (X @ X.T) ** m["zeta"]
        if m["target_type"] == "Structure":
            K = np.array([[kk[np.ix_(cs == a, cs == c)].mean() for c in range(S)] for a in range(S)])
        else:
            K = kk
        err = relative_error(z["kernel_%d" % i], K).max()
        assert err < 1e-10, (m, err)
