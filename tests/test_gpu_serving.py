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


def test_request_larger_than_a_slot_is_split_and_identical(gpu):
    """A request of more rays than one slot holds runs as slot-sized pieces
    over several rounds, mixed with other requests; its hits equal the plain
    call's, and so do the small requests' around it."""
    tris, accs = _pool()
    srv = Server(slots=2, slot_rays=1 << 14)
    ids = [srv.add_scene(a) for a in accs]
    big = np.ascontiguousarray(scenes.camera_rays_jittered(
        100_000, 77, eye=np.array([0.5, 0.5, -1.5]) * SCALE, look=np.array([0.5, 0.5, 0.5]) * SCALE))
    small = _requests(tris, 10, seed=902, max_rays=12000)
    rid_big = srv.submit(ids[1], big, CLOSEST)
    rids = [srv.submit(ids[s], r, k) for s, k, r in small]
    shadow = np.ascontiguousarray(scenes.surface_rays(
        tris[1], 50_000, 78, "shadow", light_center=LIGHT, light_size=0.1 * SCALE,
        offset=0.01 * SCALE))
    rid_sh = srv.submit(ids[1], shadow, ANY)
    out, info = srv.wait(rid_big)
    want = accs[1].intersect(big)
    assert info["nrays"] == len(big)
    assert np.array_equal(out["tri"], want["tri"])
    assert np.array_equal(out["t"].view(np.int32), want["t"].view(np.int32))
    out_sh, _ = srv.wait(rid_sh)
    assert np.array_equal(out_sh, accs[1].occluded(shadow))
    for (s, k, r), rid in zip(small, rids):
        o, _ = srv.wait(rid)
        w = accs[s].intersect(r) if k == CLOSEST else accs[s].occluded(r)
        if k == CLOSEST:
            assert np.array_equal(o["tri"], w["tri"])
        else:
            assert np.array_equal(o, w)
    srv.destroy()


def test_a_stopped_piece_fails_only_its_own_request(gpu):
    """Every request has its own status: with a stack bound too shallow for
    one scene's tree, that scene's requests report ENC_ERR_WATCHDOG while the
    requests on a shallow scene in the same rounds finish normally."""
    from encore_b200 import LaunchConfig
    shallow = scenes.random_triangles(40, seed=903, scale=SCALE)
    deep = scenes.random_triangles(200_000, seed=904, scale=SCALE)
    a_sh, a_dp = Accelerator("wbvh").build(shallow), Accelerator("wbvh").build(deep)
    srv = Server(slots=1, slot_rays=1 << 18, launch=LaunchConfig(stack_depth=2))
    i_sh, i_dp = srv.add_scene(a_sh), srv.add_scene(a_dp)
    cam = dict(eye=np.array([0.5, 0.5, -1.5]) * SCALE, look=np.array([0.5, 0.5, 0.5]) * SCALE)
    r_sh = np.ascontiguousarray(scenes.camera_rays_jittered(5000, 905, **cam))
    r_dp = np.ascontiguousarray(scenes.camera_rays_jittered(5000, 906, **cam))
    rid_dp = srv.submit(i_dp, r_dp, CLOSEST)
    rid_sh = srv.submit(i_sh, r_sh, CLOSEST)
    with pytest.raises(EncoreError) as ei:
        srv.wait(rid_dp)
    assert ei.value.status == 4  # ENC_ERR_WATCHDOG
    out, info = srv.wait(rid_sh)
    assert info["status"] == 0
    want = a_sh.intersect(r_sh)
    assert np.array_equal(out["tri"], want["tri"])
    srv.destroy()
    a_sh.destroy()
    a_dp.destroy()
