"""Placement of independent chains and serving requests on the GPUs of a node.

The reference runs one isotherm point per MPI rank (gcmc.f:334-417, basic_comms.f); here a rank
drives one GPU, and a GPU runs many chains in one persistent batch or many requests in one
server.  Chains never exchange data while they run, so a placement is only a partition: each
chain goes, whole, to one GPU, chosen so that the GPUs carry similar work and none exceeds its
device memory.  Every rank computes the same partition from the same list (the assignment is a
deterministic function of its inputs), so placing needs no communication; the one collective is
the gather of per-chain results at the end of a run.
"""
import ctypes

from ._lib import check, lib


def footprint(directory, voxel_edge=2.0):
    """(device bytes, algorithmic bytes of one move) of a deck's chain or serving slot, from the
    host tables alone (no GPU)."""
    b, c = ctypes.c_longlong(0), ctypes.c_double(0.0)
    check(lib().fmc_deck_footprint(str(directory).encode(), float(voxel_edge), ctypes.byref(b), ctypes.byref(c)))
    return int(b.value), float(c.value)


def assign(work, n_gpus, sizes=None, capacity=None):
    """GPU index of each item: items in decreasing work, each to the GPU with the least work so
    far among those whose memory still holds it (ties to the lower index).  `work` is the work of
    each item (moves x cost per move, or any proportional measure), `sizes` its device bytes and
    `capacity` the bytes a GPU offers.  Raises ValueError if an item fits on no GPU."""
    n = len(work)
    if n_gpus < 1:
        raise ValueError("n_gpus must be at least 1")
    if sizes is not None and len(sizes) != n:
        raise ValueError("one size per item")
    load = [0.0] * n_gpus
    used = [0] * n_gpus
    out = [-1] * n
    for i in sorted(range(n), key=lambda k: (-float(work[k]), k)):
        best = -1
        for g in range(n_gpus):
            if capacity is not None and sizes is not None and used[g] + sizes[i] > capacity:
                continue
            if best < 0 or load[g] < load[best]:
                best = g
        if best < 0:
            raise ValueError(f"item {i} ({sizes[i]} bytes) fits on no GPU")
        out[i] = best
        load[best] += float(work[i])
        if sizes is not None:
            used[best] += int(sizes[i])
    return out


def share(items, placement, rank):
    """The items placed on `rank`'s GPU, in their original order, with their indices."""
    return [(i, it) for i, (it, g) in enumerate(zip(items, placement)) if g == rank]


def gather(results, dist_module=None):
    """Every rank's list of (index, result) pairs, merged and in index order, on every rank
    (torch.distributed.all_gather_object; a single process returns its own list)."""
    if dist_module is None:
        import torch.distributed as dist_module
    if not dist_module.is_available() or not dist_module.is_initialized():
        return sorted(results, key=lambda x: x[0])
    parts = [None] * dist_module.get_world_size()
    dist_module.all_gather_object(parts, list(results))
    merged = [r for p in parts for r in p]
    return sorted(merged, key=lambda x: x[0])
