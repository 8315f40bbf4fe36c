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


class SceneRouter:
    """Multi-GPU serving by scene affinity.  Every scene is resident on one
    GPU (route_scenes, greedy by cost), each rank runs its own server
    (encore_b200.serving.Server on its GPU) over the scenes it owns, and a
    batch of requests submitted on the front-end rank is routed whole to the
    scenes' owners, served there with continuous batching, and the results
    are returned to the front end in submission order.  No ray of a request
    is split across GPUs and no kernel reads another GPU's memory: rays go
    to the owner and hits come back by point-to-point copies over the process
    group (NCCL between GPUs, gloo on CPU).

    server       this rank's server: add_scene(acc) -> id, submit(id, rays,
                 kind) -> request id, wait(request id) -> (out, info)
    build_scene  scene index -> the accelerator to make resident here (called
                 only for the scenes this rank owns)
    """

    CLOSEST, ANY = 0, 1

    def __init__(self, scene_costs, server, build_scene, front: int = 0):
        self.rank, self.world_size = world()
        self.owner = route_scenes(scene_costs, self.world_size)
        self.server = server
        self.front = front
        self.local = {s: server.add_scene(build_scene(s))
                      for s, o in enumerate(self.owner) if o == self.rank}

    @staticmethod
    def _out_bytes(kind: int, n: int) -> int:
        return n * (16 if kind == SceneRouter.CLOSEST else 1)

    def run(self, requests=None):
        """Collective: every rank calls it.  `requests` (front end only): a list
        of (scene, kind, rays), rays (n, 8) float32.  Returns, on the front
        end, the outputs in request order (enc_hit records as (n,) HIT
        arrays for closest hit, (n,) uint8 for any hit); None elsewhere."""
        from .accel import HIT_DTYPE
        rank, ws, front = self.rank, self.world_size, self.front
        if rank == front:
            meta = [(i, int(s), int(k), int(len(r))) for i, (s, k, r) in enumerate(requests)]
        else:
            meta = None
        if _active():
            box = [meta]
            dist.broadcast_object_list(box, src=front)
            meta = box[0]
        share = {r: [m for m in meta if self.owner[m[1]] == r] for r in range(ws)}
        dev = _device() if _active() else None
        # rays to their owners
        mine = share[rank]
        nmine = sum(m[3] for m in mine)
        if rank == front:
            for r in range(ws):
                if r == front or not share[r]:
                    continue
                buf = np.concatenate([np.ascontiguousarray(requests[m[0]][2], np.float32)
                                      for m in share[r]]).reshape(-1)
                dist.send(torch.from_numpy(buf).to(dev), dst=r)
            rays_of = {m[0]: np.ascontiguousarray(requests[m[0]][2], np.float32) for m in mine}
        else:
            rays_of = {}
            if mine:
                t = torch.empty(nmine * 8, dtype=torch.float32, device=dev)
                dist.recv(t, src=front)
                flat = t.cpu().numpy().reshape(-1, 8)
                off = 0
                for m in mine:
                    rays_of[m[0]] = flat[off:off + m[3]]
                    off += m[3]
        # serve this rank's share: all submitted, then all waited, so the
        # server batches them continuously
        rids = [(m, self.server.submit(self.local[m[1]], rays_of[m[0]], m[2])) for m in mine]
        outs = {m[0]: self.server.wait(rid)[0] for m, rid in rids}
        # results back to the front end, in each owner's share order
        if rank != front:
            if mine:
                buf = np.concatenate([np.ascontiguousarray(outs[m[0]]).reshape(-1).view(np.uint8)
                                      for m in mine])
                dist.send(torch.from_numpy(buf).to(dev), dst=front)
            return None
        results = [None] * len(meta)
        for m in mine:
            results[m[0]] = outs[m[0]]
        for r in range(ws):
            if r == front or not share[r]:
                continue
            nb = sum(self._out_bytes(m[2], m[3]) for m in share[r])
            t = torch.empty(nb, dtype=torch.uint8, device=dev)
            dist.recv(t, src=r)
            raw = t.cpu().numpy()
            off = 0
            for m in share[r]:
                b = self._out_bytes(m[2], m[3])
                chunk = raw[off:off + b].copy()
                results[m[0]] = chunk.view(HIT_DTYPE) if m[2] == self.CLOSEST else chunk
                off += b
        return results
