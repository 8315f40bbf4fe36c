"""The multi-GPU replica path's host logic on CPU: world_size-2 process
groups over gloo (the GPU runs use NCCL with the same calls).  Covers the
ray-range split, scene routing, max-over-ranks timing, scene broadcast,
ordered result gathering, a sharded intersect, and a rank that leaves: the
other rank's next collective ends with an error instead of waiting."""
import datetime
import os
import socket
import traceback

import numpy as np
import pytest

from encore_b200 import HIT_DTYPE, replicas


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class FakeAccel:
    """Stands in for a replica's Accelerator: 'hits' are a pure function of
    each ray, so the gathered batch can be checked ray by ray."""

    def intersect(self, rays):
        h = np.zeros(len(rays), HIT_DTYPE)
        h["tri"] = np.floor(rays[:, 0] * 1000).astype(np.int32)
        h["t"] = rays[:, 4] + rays[:, 5]
        return h


class FakeServer:
    """Stands in for a rank's serving.Server: records which scenes it holds
    and which requests it served; a request's hits are a pure function of its
    rays and its scene (so a request answered on the wrong scene or rank, or
    returned out of order, is caught)."""

    def __init__(self):
        self.scenes, self.served, self._out = [], [], {}

    def add_scene(self, acc):
        self.scenes.append(acc)
        return len(self.scenes) - 1

    def submit(self, sid, rays, kind=0):
        scene = self.scenes[sid]
        self.served.append(scene)
        rid = len(self.served)
        self._out[rid] = expected_output(scene, rays, kind)
        return rid

    def wait(self, rid):
        return self._out.pop(rid), {"status": 0}


def expected_output(scene, rays, kind):
    if kind == 0:
        h = np.zeros(len(rays), HIT_DTYPE)
        h["tri"] = np.floor(rays[:, 0] * 1000).astype(np.int32) + 100000 * scene
        h["t"] = rays[:, 4] + rays[:, 5]
        return h
    return ((np.floor(rays[:, 1] * 10).astype(np.int64) + scene) % 2).astype(np.uint8)


def routed_requests():
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(23):
        s = int(rng.integers(0, 7))
        n = int(rng.integers(0, 500))
        reqs.append((s, int(rng.integers(0, 2)), rng.random((n, 8)).astype(np.float32)))
    return reqs


def _worker(rank, ws, port, q, case):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=ws,
                                timeout=datetime.timedelta(seconds=5 if case == "leave" else 60))
        out = {}
        if case == "leave":
            if rank == 1:
                dist.destroy_process_group()
                q.put((rank, {"left": True}))
                return
            try:
                replicas.reduce_max(1.0)
                out["error"] = None
            except Exception as e:  # the collective must fail, not hang
                out["error"] = type(e).__name__
            q.put((rank, out))
            return
        out["world"] = replicas.world()
        out["max"] = replicas.reduce_max(rank + 1.0)
        out["sum"] = replicas.reduce_sum(rank + 1.0)
        out["rate"] = replicas.aggregate_rate(1000, 5, 100.0 * (rank + 1))
        tris = np.random.default_rng(5).random((777, 9)).astype(np.float32)
        got = replicas.broadcast_array(tris if rank == 0 else None, src=0)
        out["bcast_ok"] = bool(np.array_equal(got, tris))
        local = np.zeros(3 + 4 * rank, HIT_DTYPE)
        local["tri"] = np.arange(len(local)) + 100 * rank
        g = replicas.gather_records(local, dst=0)
        out["gather"] = None if g is None else g["tri"].tolist()
        g_all = replicas.gather_records(local, dst=None)
        out["gather_all_len"] = len(g_all)
        rays = np.random.default_rng(6).random((1001, 8)).astype(np.float32)
        hits = replicas.intersect_sharded(FakeAccel(), rays, dst=0)
        if rank == 0:
            want = FakeAccel().intersect(rays)
            out["sharded_ok"] = bool(np.array_equal(hits, want))
        out["owners"] = replicas.route_scenes([5, 1, 4, 4, 2, 9], ws)
        # serving by scene affinity: 7 scenes over the ranks, requests
        # submitted on rank 0 and answered by the scenes' owners
        srv = FakeServer()
        router = replicas.SceneRouter([5, 1, 4, 4, 2, 9, 3], srv, build_scene=lambda s: s)
        reqs = routed_requests() if rank == 0 else None
        res = router.run(reqs)
        out["router_owner"] = router.owner
        out["router_scenes"] = sorted(srv.scenes)
        out["router_served"] = sorted(set(srv.served))
        if rank == 0:
            out["router_ok"] = all(
                np.array_equal(np.asarray(got).view(np.uint8),
                               expected_output(s, r, k).view(np.uint8))
                for got, (s, k, r) in zip(res, reqs))
            out["router_n"] = len(res)
        res2 = router.run(reqs)  # a second batch through the same router
        if rank == 0:
            out["router_again"] = all(np.array_equal(np.asarray(a).view(np.uint8),
                                                     np.asarray(b).view(np.uint8))
                                      for a, b in zip(res, res2))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, out))
    except Exception:
        q.put((rank, {"exc": traceback.format_exc()}))


def run_ranks(case, ws=2, timeout=120):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_worker, args=(r, ws, port, q, case)) for r in range(ws)]
    for p in ps:
        p.start()
    res = {}
    try:
        for _ in range(ws):
            r, out = q.get(timeout=timeout)
            res[r] = out
    finally:
        for p in ps:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    for r, out in res.items():
        assert "exc" not in out, out["exc"]
    return res


def test_ray_range_tiles_the_batch():
    for n in (0, 1, 7, 1000, 4179838):
        for ws in (1, 2, 3, 8):
            parts = [replicas.ray_range(n, r, ws) for r in range(ws)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.ray_range(10, 2, 2)


def test_route_scenes_balances_and_is_deterministic():
    costs = [5, 1, 4, 4, 2, 9, 3]
    own = replicas.route_scenes(costs, 3)
    assert own == replicas.route_scenes(costs, 3)
    load = [sum(c for c, o in zip(costs, own) if o == r) for r in range(3)]
    assert max(load) - min(load) <= max(costs) and sorted(set(own)) == [0, 1, 2]


def test_single_process_fallbacks():
    assert replicas.world() == (0, 1)
    assert replicas.reduce_max(3.5) == 3.5
    rate, ms = replicas.aggregate_rate(100, 2, 50.0)
    assert ms == 50.0 and rate == pytest.approx(200 / 0.05)
    rays = np.random.default_rng(1).random((50, 8)).astype(np.float32)
    assert np.array_equal(replicas.intersect_sharded(FakeAccel(), rays), FakeAccel().intersect(rays))


def test_two_ranks_gloo():
    res = run_ranks("collectives")
    r0, r1 = res[0], res[1]
    assert r0["world"] == (0, 2) and r1["world"] == (1, 2)
    assert r0["max"] == r1["max"] == 2.0
    assert r0["sum"] == r1["sum"] == 3.0
    # weak scaling: 2 ranks x 1000 units x 5 steps over the slower rank's 200 ms
    for r in (r0, r1):
        rate, ms = r["rate"]
        assert ms == 200.0 and rate == pytest.approx(10000 / 0.2)
    assert r0["bcast_ok"] and r1["bcast_ok"]
    assert r0["gather"] == [0, 1, 2] + [100 + i for i in range(7)]
    assert r1["gather"] is None
    assert r0["gather_all_len"] == r1["gather_all_len"] == 10
    assert r0["sharded_ok"]
    assert r0["owners"] == r1["owners"]


def test_rank_that_leaves_ends_the_others_collective_with_an_error():
    res = run_ranks("leave", timeout=90)
    assert res[1]["left"]
    assert res[0]["error"] is not None


def test_scene_router_serves_each_request_on_its_owner_in_order():
    """Multi-GPU serving by scene affinity (world size 2, gloo): both ranks
    compute the same owners; each rank holds and serves only its own scenes;
    the front end gets every request's result, in submission order, twice."""
    res = run_ranks("ok")
    assert res[0]["router_owner"] == res[1]["router_owner"]
    owner = res[0]["router_owner"]
    for r in (0, 1):
        mine = [s for s, o in enumerate(owner) if o == r]
        assert res[r]["router_scenes"] == mine
        assert set(res[r]["router_served"]) <= set(mine)
    assert res[0]["router_ok"] and res[0]["router_n"] == 23
    assert res[0]["router_again"]
