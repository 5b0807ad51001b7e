"""Seeded synthetic structure batches with the shapes of the benchmark
configurations (no public dataset is named for this path, so these stand in
for one). Each function returns a batch dict (see neighbourlist.frames_to_batch):
atom_offsets, positions, numbers, cells (rows are lattice vectors), pbc.

  periodic_boxes     16 cubic boxes, 10 A, 64 atoms, Z in {1, 8}
  triclinic_cells    256 sheared cells, 0.1 atoms/A^3, 32..512 atoms, Z in {1,6,7,8}
  bulk_box           one cubic box of 100 000 atoms at 0.05 atoms/A^3, Z in {14, 8} 1:2
  molecule_clusters  10 000 non-periodic random-walk clusters of 3..29 atoms,
                     Z in {1,6,7,8,9} with half hydrogen
"""
import numpy as np


def _pack(frames):
    pos, num, cells, pbc, off = [], [], [], [], [0]
    for p, z, c, pb in frames:
        pos.append(p)
        num.append(z)
        cells.append(c)
        pbc.append(pb)
        off.append(off[-1] + len(z))
    return dict(atom_offsets=np.asarray(off, np.int64), positions=np.concatenate(pos).astype(float),
                numbers=np.concatenate(num).astype(np.int32), cells=np.asarray(cells, float),
                pbc=np.asarray(pbc, np.int32))


def _fill_cell(rng, cell, n, dmin, max_tries=200000):
    """n points uniform in the periodic cell with minimum-image distance >= dmin."""
    inv = np.linalg.inv(cell)
    frac = np.zeros((n, 3))
    k = 0
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms at this density")
        f = rng.random(3)
        if k:
            d = frac[:k] - f
            d -= np.round(d)
            r = d @ cell
            if np.min(np.einsum("ij,ij->i", r, r)) < dmin * dmin:
                continue
        frac[k] = f
        k += 1
    del inv
    return frac @ cell


def periodic_boxes(seed=0, n_struct=16, side=10.0, n_atoms=64, species=(1, 8), dmin=0.9):
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n_struct):
        cell = np.eye(3) * side
        pos = _fill_cell(rng, cell, n_atoms, dmin)
        z = rng.choice(species, size=n_atoms)
        frames.append((pos, z, cell, [1, 1, 1]))
    return _pack(frames)


def triclinic_cells(seed=0, n_struct=256, density=0.1, n_min=32, n_max=512, species=(1, 6, 7, 8),
                    shear=0.1, dmin=0.9):
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n_struct):
        n = int(rng.integers(n_min, n_max + 1))
        m = np.eye(3) + np.where(np.eye(3) == 1, 0., rng.uniform(-shear, shear, (3, 3)))
        vol = n / density
        a = (vol / abs(np.linalg.det(m))) ** (1. / 3.)
        cell = a * m
        pos = _fill_cell(rng, cell, n, dmin)
        z = rng.choice(species, size=n)
        frames.append((pos, z, cell, [1, 1, 1]))
    return _pack(frames)


def bulk_box(seed=0, n_atoms=100000, density=0.05, species=(14, 8), ratio=(1, 2), dmin=1.2):
    rng = np.random.default_rng(seed)
    side = (n_atoms / density) ** (1. / 3.)
    ng = max(1, int(side // dmin))
    h = side / ng
    grid = {}
    pos = np.zeros((n_atoms, 3))
    k = 0
    while k < n_atoms:
        cand = rng.random((4096, 3)) * side
        for p in cand:
            g = tuple((p // h).astype(int) % ng)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for q in grid.get(((g[0] + dx) % ng, (g[1] + dy) % ng, (g[2] + dz) % ng), ()):
                            d = pos[q] - p
                            d -= side * np.round(d / side)
                            if d @ d < dmin * dmin:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[k] = p
                grid.setdefault(g, []).append(k)
                k += 1
                if k == n_atoms:
                    break
    w = np.asarray(ratio, float)
    z = rng.choice(species, size=n_atoms, p=w / w.sum())
    return _pack([(pos, z, np.eye(3) * side, [1, 1, 1])])


def molecule_clusters(seed=0, n_struct=10000, n_min=3, n_max=29, species=(1, 6, 7, 8, 9), h_fraction=0.5,
                      bond=(1.0, 1.6), dmin=0.9):
    """Random-walk chains: each atom sits at a random bond length from the
    previous one (or from a random earlier atom when the chain is boxed in),
    rejecting placements closer than dmin to any atom. The cell is zero and
    non-periodic; AtomsList turns it into the bounding box x1.05."""
    rng = np.random.default_rng(seed)
    heavy = [s for s in species if s != 1]
    frames = []
    for _ in range(n_struct):
        n = int(rng.integers(n_min, n_max + 1))
        pos = np.zeros((n, 3))
        k = 1
        anchor = 0
        fails = 0
        while k < n:
            v = rng.normal(size=3)
            v *= rng.uniform(*bond) / np.linalg.norm(v)
            p = pos[anchor] + v
            d = pos[:k] - p
            if np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin:
                fails += 1
                if fails > 20:
                    anchor = int(rng.integers(0, k))
                    fails = 0
                continue
            pos[k] = p
            anchor = k
            k += 1
            fails = 0
        z = np.where(rng.random(n) < h_fraction, 1, rng.choice(heavy, size=n))
        # non-periodic cell: the bounding box x1.05 with the box centred in it
        # (centring on the box midpoint keeps every atom inside the cell;
        # centring on the mean, as a zero cell gets in AtomsList, may not)
        L = (pos.max(0) - pos.min(0)) * 1.05
        L = np.maximum(L, 1e-3)
        pos = pos + (0.5 * L - 0.5 * (pos.max(0) + pos.min(0)))
        frames.append((pos, z, np.diag(L), [0, 0, 0]))
    return _pack(frames)


def select_sparse_points(features, species_of_row, per_species, seed=0):
    """Seeded random choice of `per_species` rows per central species
    (dict species -> count, or an int for all species)."""
    rng = np.random.default_rng(seed)
    idx = []
    for s in sorted(set(int(x) for x in species_of_row)):
        rows = np.flatnonzero(species_of_row == s)
        k = per_species if isinstance(per_species, int) else per_species.get(s, 0)
        k = min(k, len(rows))
        idx.extend(sorted(rng.choice(rows, size=k, replace=False).tolist()))
    return np.asarray(idx, dtype=np.int64)
