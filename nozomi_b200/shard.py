"""Sharding a simulation over processes, one per GPU.

The reference has no multi-GPU path: its users run one independent process
per GPU (run-simulation.sh:83-86).  Here a run shards the natural way, with
one exchange step:

* Walkers.  A run of N walkers is split into contiguous walker-id ranges, one
  per rank (``shard_range``).  A rank seeds exactly its walkers of the
  unsharded run (``nz_seed_range``: the walker id is the Philox counter of the
  seeding rounds), packs them under their global ids (the walk's draws are
  keyed by walker id) and walks them with the fused kernel.  Its signal sums
  [2, ndir, nb] (FP64 sums of cos and sin) are then summed over ranks in one
  all-reduce, 2 * ndir * nb doubles.  Every walker's trajectory is the one it
  has in the unsharded run, so the reduced signal equals the unsharded
  signal up to the order of the FP64 sums, whatever the world size.
* Jobs.  A batch of independent jobs (substrates x protocols) is split whole,
  longest first onto the least-loaded rank (``shard_jobs``); no data crosses
  ranks.

Substrates, cell lists and protocol tables are replicated: each rank builds
its own.  ``reduce_sums`` is the exchange; ``AbortFlag`` lets a rank that
fails between steps tell the others through the process group's store before
their next collective, and a short process-group timeout ends a collective
that a failed rank never joins.
"""
from __future__ import annotations

import datetime

import numpy as np


def shard_range(N: int, world: int, rank: int) -> tuple[int, int]:
    """(first walker id, count) of `rank`'s shard of N walkers: contiguous,
    sizes differing by at most one, the larger shards first."""
    if world < 1 or not 0 <= rank < world or N < 0:
        raise ValueError(f"bad shard: N={N} world={world} rank={rank}")
    base, extra = divmod(int(N), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def shard_jobs(costs, world: int) -> list[list[int]]:
    """Job indices per rank: longest job first onto the least-loaded rank
    (ties to the lowest rank), so every rank computes the same assignment."""
    costs = np.asarray(costs, dtype=np.float64)
    load = np.zeros(world)
    out: list[list[int]] = [[] for _ in range(world)]
    for j in sorted(range(costs.size), key=lambda k: (-costs[k], k)):
        r = int(np.argmin(load))
        out[r].append(j)
        load[r] += costs[j]
    for r in out:
        r.sort()
    return out


def reduce_sums(t, group=None):
    """Sum a tensor of per-rank partial sums over the ranks, in place (one
    all-reduce; a no-op without an initialised process group)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


class ShardAborted(RuntimeError):
    pass


class AbortFlag:
    """A flag in the process group's store.  A rank that fails between steps
    calls ``raise_abort``; every rank calls ``check`` before its next
    collective and raises ShardAborted if any rank has failed."""

    KEY = "nozomi_b200/abort"

    def __init__(self, store):
        self.store = store

    def raise_abort(self, rank: int, why: str):
        self.store.set(self.KEY, f"rank {rank}: {why}")

    def check(self):
        if self.store.check([self.KEY]):
            raise ShardAborted(self.store.get(self.KEY).decode())


def init_process_group(backend: str, timeout_s: float = 60.0):
    """torch.distributed from the launcher's environment (RANK, WORLD_SIZE,
    MASTER_ADDR, MASTER_PORT) with a short collective timeout, so that ranks
    waiting on a rank that failed end with an error instead of hanging."""
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist.get_rank(), dist.get_world_size()


class ShardedDwiRun:
    """One rank's shard of a DWI run of N walkers (the walk of
    simulate.DwiRun on walkers [first, first + count)); ``signal`` reduces
    over ranks and normalises by N."""

    def __init__(self, dsub, gwave, dirs, amplitudes, N: int, seed: int = 0, rank: int = 0, world: int = 1,
                 targets=None, tuning=None, group=None):
        from .simulate import DwiRun
        self.N = int(N)
        self.rank, self.world, self.group = rank, world, group
        self.first, self.count = shard_range(N, world, rank)
        self.run = DwiRun(dsub, gwave, dirs, amplitudes, self.count, seed=seed, targets=targets, tuning=tuning,
                          id0=self.first)

    def prepare(self, positions=None, labels=None):
        self.run.prepare(positions, labels)
        return self

    def walk(self, events=None):
        self.run.walk(events)
        return self

    def local_sums(self):
        """This shard's [2, ndir, nb] FP64 sums (device)."""
        return self.run.signal_sums()

    def signal_sums(self):
        return reduce_sums(self.local_sums(), self.group)

    def signal(self) -> np.ndarray:
        s = self.signal_sums().cpu().numpy()
        return (s[0] + 1j * s[1]) / self.N
