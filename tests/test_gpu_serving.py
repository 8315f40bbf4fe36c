"""Serving (GPU): continuous batching must not change any result.  Every
request's hits are the same whether it runs alone or mixed with others that
arrive while it is on the GPU, and the same as the plain per-request call."""
import threading
import time

import numpy as np
import pytest

from encore_b200 import Accelerator, EncoreError, scenes
from encore_b200.serving import ANY, CLOSEST, Server

pytestmark = pytest.mark.gpu
SCALE = 1000.0
LIGHT = np.array([0.5, 2.0, 0.5]) * SCALE


def _pool():
    tris = [scenes.random_triangles(n, seed=50 + i, scale=SCALE)
            for i, n in enumerate([1500, 12000, 40000, 3000])]
    tris.append(scenes.heightfield(res=96, seed=57, scale=SCALE))
    return tris, [Accelerator("wbvh").build(t) for t in tris]


def _requests(tris, count, seed, max_rays=60000):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        s = int(rng.integers(0, len(tris)))
        n = int(np.exp(rng.uniform(np.log(16), np.log(max_rays))))
        u = rng.random()
        if u < 0.6:
            r = scenes.camera_rays_jittered(n, seed + 7 * i, eye=np.array([0.5, 0.5, -1.5]) * SCALE,
                                            look=np.array([0.5, 0.5, 0.5]) * SCALE)
            k = CLOSEST
        elif u < 0.9:
            r = scenes.surface_rays(tris[s], n, seed + 7 * i, "diffuse", offset=0.1)
            k = CLOSEST
        else:
            r = scenes.surface_rays(tris[s], n, seed + 7 * i, "shadow", light_center=LIGHT,
                                    light_size=0.1 * SCALE, offset=0.01 * SCALE)
            k = ANY
        reqs.append((s, k, np.ascontiguousarray(r)))
    return reqs


def test_results_identical_alone_and_in_mix(gpu):
    tris, accs = _pool()
    reqs = _requests(tris, 36, seed=900)
    srv = Server(slots=3, slot_rays=1 << 18)
    ids = [srv.add_scene(a) for a in accs]
    alone = []
    for s, k, r in reqs:
        out, info = srv.wait(srv.submit(ids[s], r, k))
        alone.append(out.copy())
        assert info["done_s"] >= info["start_s"] >= info["submit_s"]
    # plain per-request calls agree
    for (s, k, r), a in zip(reqs, alone):
        want = accs[s].intersect(r) if k == CLOSEST else accs[s].occluded(r)
        if k == CLOSEST:
            assert np.array_equal(a["tri"], want["tri"])
            assert np.array_equal(a["t"].view(np.int32), want["t"].view(np.int32))
        else:
            assert np.array_equal(a, want)
    # the mix: half submitted at once, half from a thread while those run
    rids = [None] * len(reqs)
    half = len(reqs) // 2

    def late():
        for j in range(half, len(reqs)):
            s, k, r = reqs[j]
            rids[j] = srv.submit(ids[s], r, k)
            time.sleep(0.0005)

    for j in range(half):
        s, k, r = reqs[j]
        rids[j] = srv.submit(ids[s], r, k)
    th = threading.Thread(target=late)
    th.start()
    th.join()
    for j, rid in enumerate(rids):
        out, info = srv.wait(rid)
        if reqs[j][1] == CLOSEST:
            assert np.array_equal(out.view(np.int32), alone[j].view(np.int32)), j
        else:
            assert np.array_equal(out, alone[j]), j
    srv.destroy()


def test_budget_capacity_and_cancel(gpu):
    tris, accs = _pool()
    tiny = Server(slots=1, slot_rays=1024, budget_bytes=1 << 20)
    with pytest.raises(EncoreError) as ei:
        tiny.add_scene(accs[2])
    assert ei.value.status == 5  # ENC_ERR_BUDGET
    tiny.destroy()
    srv = Server(slots=1, slot_rays=1 << 16)
    sid = srv.add_scene(accs[2])
    big = np.zeros(((1 << 16) + 1, 8), np.float32)
    with pytest.raises(EncoreError) as ei:
        srv.submit(sid, big)
    assert ei.value.status == 5
    reqs = _requests(tris[2:3], 12, seed=901, max_rays=60000)
    rids = [srv.submit(sid, r, k) for _, k, r in reqs]
    cancelled = [rid for rid in rids[-4:] if srv.cancel(rid)]
    for rid in rids:
        if rid in cancelled:
            with pytest.raises(EncoreError) as ei:
                srv.wait(rid)
            assert ei.value.status == 7  # ENC_ERR_CANCELLED
        else:
            out, info = srv.wait(rid)
            assert out is not None
    srv.destroy()


def test_empty_request_and_timeout(gpu):
    tris, accs = _pool()
    srv = Server(slots=2, slot_rays=1 << 16)
    sid = srv.add_scene(accs[0])
    out, info = srv.wait(srv.submit(sid, np.zeros((0, 8), np.float32)))
    assert len(out) == 0 and info["nrays"] == 0
    srv.destroy()
