"""The oracle's RadialScaling cutoff (representations/cutoff_functions.hh:
178-280) in the position gradients: power-spectrum gradients against
central differences of the features. Its values are pinned by the
reference's expansion goldens (tests/test_oracle_golden.py)."""
import numpy as np

from librascal_b200 import synthetic
from oracle import oracle as O


def test_radial_scaling_gradient_fd():
    batch = synthetic.molecule_clusters(n_struct=2, seed=1)
    calc = O.Calculator(5.0, 0.5, 4, 3, 0.5, radial_scaling=dict(rate=1.0, scale=2.0, exponent=4.0))
    species = np.unique(batch["numbers"])
    r = O.Run(calc, batch, species, gradients=True)
    dX = r.power_spectrum_gradient()
    pr = r.pairs()
    _, _, po = r.centers()
    centre_of_pair = np.repeat(np.arange(r.n_centers), np.diff(po))
    h = 1e-5
    for a in (0, int(batch["atom_offsets"][1]) + 2):
        for c in range(3):
            X = []
            for sgn in (1, -1):
                b2 = {k: np.array(v, copy=True) for k, v in batch.items()}
                b2["positions"][a, c] += sgn * h
                X.append(O.Run(calc, b2, species).power_spectrum())
            fd = (X[0] - X[1]) / (2 * h)
            an = np.zeros_like(fd)
            sel = pr["j"] == a
            np.add.at(an, centre_of_pair[sel], dX[sel, c])
            assert np.abs(an - fd).max() <= 1e-6 * max(np.abs(fd).max(), 1e-3), (a, c)
