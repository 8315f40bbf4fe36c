"""Multi-GPU by replicas: one process per GPU, each holding a full copy of
the scene's accelerator (and photon map) in its own HBM.

Ray queries are independent, so nothing on the query path crosses GPUs: a
batch is split into contiguous ray ranges, or whole requests are routed to a
GPU by scene.  The collectives here are plumbing around that path (scene
distribution, result collection, max-over-ranks timing) over
``torch.distributed`` (NCCL between GPUs, gloo on CPU).

The reference has no multi-process code (its queries are one ray per call
on one thread, ENCORE/src/accelerators/AccelerationStructure.h:63); this
module is what a multi-GPU caller of the engine uses.
"""
from __future__ import annotations

import numpy as np

try:
    import torch
    import torch.distributed as dist
except ImportError:  # the package's single-GPU path does not need torch
    torch = None
    dist = None


def _active() -> bool:
    return dist is not None and dist.is_available() and dist.is_initialized()


def world() -> tuple[int, int]:
    """(rank, world size); (0, 1) without an initialised process group."""
    if not _active():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


def _device():
    """Tensors for collectives live on the current CUDA device under NCCL and
    on the CPU under gloo."""
    if _active() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def ray_range(n: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous [lo, hi) share of n rays for `rank`; sizes differ by at most
    one and the shares tile [0, n) in rank order."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    base, extra = divmod(n, world_size)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def route_scenes(scene_costs, world_size: int) -> list[int]:
    """Scene affinity for serving: each scene goes to one GPU.  Greedy by
    cost (e.g. triangle count or expected rays/s), largest first, to the
    least-loaded GPU; ties go to the lower rank.  Returns the owner of each
    scene, deterministic on every rank."""
    costs = np.asarray(scene_costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return owner


def reduce_max(x: float) -> float:
    """Max over ranks (the device time of a multi-GPU step)."""
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float) -> float:
    if not _active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(units_per_rank: int, steps: int, local_ms: float) -> tuple[float, float]:
    """Whole-job throughput (units/s over all ranks) and the max-over-ranks
    total time in ms, for weak scaling (every rank does `units_per_rank`
    units per step)."""
    ms = reduce_max(local_ms)
    total_units = reduce_sum(units_per_rank * steps)
    return total_units / (ms * 1e-3), ms


def broadcast_array(a: np.ndarray | None, src: int = 0, dtype=np.float32) -> np.ndarray:
    """Sends a host array from `src` to every rank (scene triangles, photon
    records) so each builds its own replica.  Other ranks pass None."""
    if not _active():
        if a is None:
            raise ValueError("no array to broadcast without a process group")
        return np.ascontiguousarray(a, dtype=dtype)
    rank, _ = world()
    dev = _device()
    shape = torch.zeros(8, dtype=torch.int64, device=dev)
    if rank == src:
        a = np.ascontiguousarray(a, dtype=dtype)
        if a.ndim > 7:
            raise ValueError("at most 7 dimensions")
        shape[0] = a.ndim
        shape[1:1 + a.ndim] = torch.tensor(a.shape, dtype=torch.int64)
    dist.broadcast(shape, src=src)
    nd = int(shape[0])
    shp = tuple(int(s) for s in shape[1:1 + nd].tolist())
    buf = (torch.from_numpy(a.reshape(-1).view(np.uint8)).to(dev) if rank == src
           else torch.empty(int(np.prod(shp, dtype=np.int64)) * np.dtype(dtype).itemsize,
                            dtype=torch.uint8, device=dev))
    dist.broadcast(buf, src=src)
    return buf.cpu().numpy().view(dtype).reshape(shp)


def gather_records(local: np.ndarray, dst: int | None = 0) -> np.ndarray | None:
    """Concatenates each rank's records (any fixed-size numpy dtype, e.g. the
    hits of its ray range) in rank order, on `dst` (None = on every rank).
    Ranks may hold different counts."""
    if not _active():
        return local
    rank, ws = world()
    dev = _device()
    raw = np.ascontiguousarray(local).reshape(-1).view(np.uint8)
    n = torch.tensor([raw.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(ws)]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    cap = max(sizes) if sizes else 0
    mine = torch.zeros(cap, dtype=torch.uint8, device=dev)
    if raw.size:
        mine[:raw.size] = torch.from_numpy(raw).to(dev)
    parts = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(ws)]
    dist.all_gather(parts, mine)
    if dst is not None and rank != dst:
        return None
    out = np.concatenate([p.cpu().numpy()[:s] for p, s in zip(parts, sizes)])
    return out.view(local.dtype)


def intersect_sharded(acc, rays: np.ndarray, dst: int | None = 0, **kw) -> np.ndarray | None:
    """Closest hits of one batch split across the replicas: each rank traces
    its contiguous ray range on its own GPU, results are gathered in ray
    order on `dst`.  `acc` is this rank's Accelerator."""
    rank, ws = world()
    lo, hi = ray_range(len(rays), rank, ws)
    local = acc.intersect(rays[lo:hi], **kw)
    return gather_records(local, dst=dst)
