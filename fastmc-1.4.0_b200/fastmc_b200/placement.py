"""Placement of independent chains and serving requests on the GPUs of a node.

The reference runs one isotherm point per MPI rank (gcmc.f:334-417, basic_comms.f); here a rank
drives one GPU, and a GPU runs many chains in one persistent batch or many requests in one
server.  Chains never exchange data while they run, so a placement is only a partition: each
chain goes, whole, to one GPU, chosen so that the GPUs carry similar work and none exceeds its
device memory.  Every rank computes the same partition from the same list (the assignment is a
deterministic function of its inputs), so placing needs no communication; the one collective is
the gather of per-chain results at the end of a run.

A rank that fails or leaves between steps is found on the host, through the process group's
key-value store, before the others enter their next step or the gather (`Liveness`): the
reference has no recovery beyond a manual restart (error.f stops a rank), and here the others
stop with an error that names the lost rank instead of waiting in a collective.
"""
import ctypes
import time

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


class RankLost(RuntimeError):
    """A rank did not check in for a step in time, or left the run; `.rank` and `.step` say
    which and when, `.left` whether it left on purpose."""

    def __init__(self, rank, step, left=False, detail=""):
        what = "left the run" if left else "did not check in"
        super().__init__(f"rank {rank} {what} at step {step!r}" + (f" ({detail})" if detail else ""))
        self.rank, self.step, self.left = rank, step, left


class Liveness:
    """Per-step check-ins of the ranks of one run through a key-value store (the process group's
    TCPStore, or any object with set / get / check).  Each rank calls `check_in(step)` once it has
    finished a step, and `wait_all(step)` before it starts the next one (or the gather): that
    returns once every rank has checked in for the step and raises RankLost as soon as one has
    left (`leave`) or after `timeout_s` without its check-in (a rank that raised, was killed or
    never got there).  A store that stops answering is reported as the loss of `store_host`, the
    rank whose process serves it (rank 0 for the process group's own store).  Keys are namespaced
    by `prefix`, so one store serves several runs."""

    def __init__(self, store, rank, world, timeout_s=30.0, prefix="fmc", poll_s=0.02, store_host=0):
        self.store, self.rank, self.world = store, int(rank), int(world)
        self.timeout_s, self.prefix, self.poll_s = float(timeout_s), str(prefix), float(poll_s)
        self.store_host = int(store_host)

    def _key(self, step, rank):
        return f"{self.prefix}/step/{step}/{rank}"

    def _left(self, rank):
        return f"{self.prefix}/left/{rank}"

    def check_in(self, step):
        self.store.set(self._key(step, self.rank), "1")

    def leave(self, step):
        """This rank stops after `step` (between steps, with nothing in flight)."""
        self.store.set(self._left(self.rank), str(step))

    def wait_all(self, step):
        pending = [r for r in range(self.world) if r != self.rank]
        deadline = time.monotonic() + self.timeout_s
        while pending:
            still = []
            for r in pending:
                try:
                    if self.store.check([self._key(step, r)]):
                        continue
                    if self.store.check([self._left(r)]):
                        after = self.store.get(self._left(r))
                        after = after.decode() if isinstance(after, bytes) else str(after)
                        raise RankLost(r, step, left=True, detail=f"after step {after}")
                except RankLost:
                    raise
                except Exception as e:  # the store itself is gone with its host
                    raise RankLost(self.store_host, step, detail=f"store unreachable: {e}") from e
                still.append(r)
            pending = still
            if pending and time.monotonic() > deadline:
                raise RankLost(pending[0], step, detail=f"no check-in within {self.timeout_s:g} s")
            if pending:
                time.sleep(self.poll_s)


def gather(results, dist_module=None, liveness=None):
    """Every rank's list of (index, result) pairs, merged and in index order, on every rank
    (torch.distributed.all_gather_object; a single process returns its own list).  With a
    Liveness, every rank checks in for the gather first, so a lost rank raises RankLost here
    instead of leaving the others in the collective."""
    if dist_module is None:
        import torch.distributed as dist_module
    if not dist_module.is_available() or not dist_module.is_initialized():
        return sorted(results, key=lambda x: x[0])
    if liveness is not None:
        liveness.check_in("gather")
        liveness.wait_all("gather")
    parts = [None] * dist_module.get_world_size()
    dist_module.all_gather_object(parts, list(results))
    merged = [r for p in parts for r in p]
    return sorted(merged, key=lambda x: x[0])
