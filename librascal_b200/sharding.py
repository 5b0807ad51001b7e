"""Structure-parallel sharding of the path across ranks, one process per GPU.

Structures are independent all the way from the neighbour list to the GAP
energies and forces (the reference computes them one manager at a time,
bindings/rascal/models/krr.py:92-166), so a rank needs nothing from another
rank during a prediction. A batch is cut into contiguous shards of nearly
equal cost, each rank predicts its own shard with its own copy of the model,
and the per-structure energies and per-atom forces are gathered once at the
end, in the batch's order. The only collectives are that gather and the
max-over-ranks of a timing.
"""
import numpy as np

BATCH_KEYS_PER_STRUCTURE = ("cells", "pbc")
BATCH_KEYS_PER_ATOM = ("positions", "numbers", "center_atoms_mask")


def partition(costs, world):
    """Contiguous [start, stop) ranges of structures, one per rank, with the
    cumulative cost cut as close as possible to k * total / world. Every
    structure lands in exactly one range; ranges may be empty when there are
    fewer structures than ranks."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world size must be >= 1")
    if np.any(costs < 0):
        raise ValueError("structure costs must be non-negative")
    n = len(costs)
    csum = np.concatenate([[0.0], np.cumsum(costs)])
    total = csum[-1]
    cuts = [0]
    for k in range(1, world):
        target = total * k / world
        c = int(np.searchsorted(csum, target, side="left"))
        # the nearer of the two boundaries around the target
        if 0 < c <= n and abs(csum[c - 1] - target) <= abs(csum[c] - target):
            c -= 1
        cuts.append(min(max(c, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def structure_costs(batch):
    """Default cost: atoms squared per structure (pairs grow with the atom
    count for clusters smaller than the cutoff sphere)."""
    n = np.diff(np.asarray(batch["atom_offsets"]))
    return n.astype(np.float64) ** 2


def shard_batch(batch, start, stop):
    """Sub-batch of structures [start, stop) with rebased atom offsets."""
    off = np.asarray(batch["atom_offsets"])
    a0, a1 = int(off[start]), int(off[stop])
    out = dict(atom_offsets=off[start:stop + 1] - a0)
    for k in BATCH_KEYS_PER_STRUCTURE:
        if k in batch:
            out[k] = np.asarray(batch[k])[start:stop]
    for k in BATCH_KEYS_PER_ATOM:
        if k in batch:
            out[k] = np.asarray(batch[k])[a0:a1]
    return out


def gather_results(energies, forces, group=None):
    """All ranks' per-structure energies and per-atom forces, concatenated in
    rank order (the batch order for shards from `partition`). Returns the
    full arrays on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, (np.asarray(energies), np.asarray(forces)), group=group)
    E = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0)
    F = np.concatenate([p[1].reshape(-1, 3) for p in parts]) if parts else np.zeros((0, 3))
    return E, F


def max_over_ranks(x, group=None, device=None):
    """Largest value of a float over all ranks (timings are reported as the
    slowest rank). `device` is where the reduction tensor lives: a CUDA
    device for NCCL, None (CPU) for gloo."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
