"""Structure-parallel sharding (the N > 1 path) on CPU: partition properties
and a world-size-2 gloo run in which each rank predicts its shard and the
gathered energies and forces equal the unsharded prediction.

The per-rank compute here is the CPU oracle (the GPU path is exercised by the
-m gpu tests); what is under test is the partition, the sub-batches, the
gather order and the max-over-ranks reduction.
"""
import os
import socket

import numpy as np
import pytest

from librascal_b200 import sharding, synthetic

HYPERS = (5.0, 0.5, 4, 3, 0.4)


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 8):
        for n in (0, 1, 5, 100):
            costs = rng.integers(1, 900, size=n).astype(float)
            parts = sharding.partition(costs, world)
            assert len(parts) == world
            assert parts[0][0] == 0 and parts[-1][1] == n
            for (a, b), (c, _) in zip(parts, parts[1:]):
                assert a <= b == c
            if n >= world:
                loads = [costs[a:b].sum() for a, b in parts]
                # a contiguous cut is off the ideal by at most one structure
                assert max(loads) <= costs.sum() / world + costs.max()


def test_partition_rejects_bad_input():
    with pytest.raises(ValueError):
        sharding.partition([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        sharding.partition([1.0], 0)


def test_shard_batch_rebases_offsets():
    batch = synthetic.molecule_clusters(n_struct=5, seed=1)
    off = batch["atom_offsets"]
    sub = sharding.shard_batch(batch, 2, 4)
    assert sub["atom_offsets"][0] == 0
    assert np.array_equal(sub["atom_offsets"], off[2:5] - off[2])
    assert np.array_equal(sub["positions"], batch["positions"][off[2]:off[4]])
    assert np.array_equal(sub["numbers"], batch["numbers"][off[2]:off[4]])
    assert np.array_equal(sub["cells"], batch["cells"][2:4])


def _model(batch):
    from oracle import oracle as O
    species = sorted(set(int(z) for z in batch["numbers"]))
    calc = O.Calculator(*HYPERS)
    r = O.Run(calc, batch, species)
    X = r.power_spectrum()
    ca, _, _ = r.centers()
    sp_row = batch["numbers"][ca]
    idx = synthetic.select_sparse_points(X, sp_row, 3, seed=0)
    alpha = np.random.default_rng(0).normal(size=len(idx))
    return calc, species, X[idx], sp_row[idx], alpha


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batch = synthetic.molecule_clusters(n_struct=7, seed=3)
        calc, species, T, sps, alpha = _model(batch)
        a, b = sharding.partition(sharding.structure_costs(batch), world)[rank]
        sub = sharding.shard_batch(batch, a, b)
        E, F = O.Run(calc, sub, species, gradients=True).gap(sps, T, alpha, 2)
        E_all, F_all = sharding.gather_results(E, F)
        slowest = sharding.max_over_ranks(float(rank + 1))
        if rank == 0:
            E_ref, F_ref = O.Run(calc, batch, species, gradients=True).gap(sps, T, alpha, 2)
            np.savez(os.path.join(out_dir, "result.npz"), E=E_all, F=F_all, E_ref=E_ref, F_ref=F_ref,
                     slowest=slowest)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gloo_two_ranks_gather_matches_unsharded(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    z = np.load(tmp_path / "result.npz")
    assert z["slowest"] == 2.0
    assert z["E"].shape == z["E_ref"].shape and z["F"].shape == z["F_ref"].shape
    # per-structure work is identical whichever rank runs it
    assert np.array_equal(z["E"], z["E_ref"])
    assert np.array_equal(z["F"], z["F_ref"])
