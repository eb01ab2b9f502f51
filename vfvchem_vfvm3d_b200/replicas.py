"""One process per GPU, launched by torchrun: ranks from the environment, the process group, and
the max-over-ranks reduction of device timings.

The single-mesh solve does not shard (one GPU holds the whole system), so N processes run N
independent replicas with no collective on the data path; the only collectives are the barrier
around the timed region and one all-reduce (MAX) of the timings. A batch of independent meshes
(the transient transport batch) shards whole meshes across ranks with :func:`shard_meshes`.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

import numpy as np


@dataclass
class Ranks:
    rank: int = 0
    world: int = 1
    local: int = 0
    backend: str = ""
    dist: object = None  # torch.distributed once a group exists

    @property
    def active(self) -> bool:
        return self.dist is not None


def init_from_env(backend: str | None = None, timeout_s: float = 600.0) -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK from torchrun; with more than one rank a process group over
    `backend` (VFV_DIST_BACKEND, else nccl when CUDA is present, else gloo)."""
    r = Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0")))
    if r.world <= 1:
        return r
    import torch
    import torch.distributed as dist
    be = backend or os.environ.get("VFV_DIST_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")
    if be == "nccl":
        torch.cuda.set_device(r.local)
    dist.init_process_group(be, timeout=datetime.timedelta(seconds=timeout_s))
    r.backend = be
    r.dist = dist
    return r


def barrier(r: Ranks) -> None:
    if r.active:
        r.dist.barrier()


def max_over_ranks(r: Ranks, values):
    """Element-wise maximum of `values` over all ranks (the job's time is its slowest rank's)."""
    vals = [float(v) for v in values]
    if not r.active:
        return vals
    import torch
    dev = torch.device("cuda", r.local) if r.backend == "nccl" else torch.device("cpu")
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    r.dist.all_reduce(t, op=r.dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def finalize(r: Ranks) -> None:
    if r.active:
        r.dist.barrier()
        r.dist.destroy_process_group()
        r.dist = None


def shard_meshes(sizes, rank: int, world: int) -> np.ndarray:
    """Indices of the meshes rank `rank` owns: largest first, each to the least-loaded rank (ties
    to the lower rank). Deterministic, disjoint, and covering all meshes."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    load = np.zeros(world, np.int64)
    owner = np.empty(sizes.size, np.int64)
    for i in order:
        w = int(np.argmin(load))
        owner[i] = w
        load[w] += sizes[i]
    return np.nonzero(owner == rank)[0]
