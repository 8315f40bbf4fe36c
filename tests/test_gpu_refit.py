"""Accelerator update for moved geometry (GPU).

``Accelerator.update`` stands where AccelerationStructure::update stands
(ENCORE/src/accelerators/AccelerationStructure.h:51; Bvh::update,
ENCORE/src/accelerators/BVH.cpp:52-121, walks the tree and re-boxes it; the
reference Kdtree rebuilds).  Here the wide BVH keeps its shape and gets new
boxes and triangle records; the kd layout rebuilds by the reference rules.
The bar is the one every other closest-hit query meets: the same answers as
the oracle on the moved scene.
"""
import numpy as np
import pytest

from encore_b200 import Accelerator, EncoreError, scenes
from oracle import bindings as ob

pytestmark = pytest.mark.gpu
SCALE = 1000.0


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


def moved(tris: np.ndarray, seed: int, amount: float) -> np.ndarray:
    """Each triangle rigidly shifted by its own random offset, plus a global
    wave along y: every box changes, the triangle IDs stay."""
    rng = np.random.default_rng(seed)
    t = tris.reshape(-1, 3, 3).astype(np.float64).copy()
    t += rng.normal(0.0, amount, (t.shape[0], 1, 3))
    t[:, :, 1] += 0.05 * SCALE * np.sin(t[:, :, 0] / SCALE * 6.0)
    return t.reshape(-1, 9).astype(np.float32)


def rays_for(seed: int) -> np.ndarray:
    return np.concatenate([
        scenes.camera_rays(96, 96, eye=np.array([0.5, 0.5, -1.5]) * SCALE,
                           look=np.array([0.5, 0.5, 0.5]) * SCALE),
        scenes.random_sphere_rays(6000, seed=seed, hi=(SCALE, SCALE, SCALE))])


def assert_matches_brute(tris, rays, got):
    want = ob.port_brute(tris, rays, clamp=True)
    mism, classes = ob.classify(tris, rays, got, want)
    assert "unexplained" not in classes, list(zip(mism.tolist(), classes))
    assert len([c for c in classes if c != "tie"]) <= 3, classes
    m = (got["tri"] == want["tri"]) & (want["tri"] >= 0)
    assert np.array_equal(bits(got["t"][m]), bits(want["t"][m]))
    assert np.array_equal(bits(got["u"][m]), bits(want["u"][m]))
    assert np.array_equal(bits(got["v"][m]), bits(want["v"][m]))


@pytest.mark.parametrize("width", [2, 4, 8])
def test_wbvh_refit_matches_brute_force_on_moved_scene(gpu, width):
    a = scenes.random_triangles(5000, seed=501, scale=SCALE)
    b = moved(a, seed=502, amount=0.02 * SCALE)
    rays = rays_for(503)
    acc = Accelerator("wbvh", width=width).build(a)
    nodes_before = acc.info()["nnodes"]
    acc.update(b)
    assert acc.info()["nnodes"] == nodes_before  # same tree, new boxes
    assert_matches_brute(b, rays, acc.intersect(rays))
    # the refit tree answers like a fresh build on the moved scene, up to ties
    fresh = Accelerator("wbvh", width=width).build(b).intersect(rays)
    got = acc.intersect(rays)
    diff = np.nonzero(got["tri"] != fresh["tri"])[0]
    assert np.array_equal(bits(got["t"][diff]), bits(fresh["t"][diff]))


def test_wbvh_refit_survives_scrambled_geometry(gpu):
    """Triangles moved to arbitrary new places (every leaf box now spans the
    scene) still give exact answers: refit trades speed, never results."""
    a = scenes.random_triangles(3000, seed=511, scale=SCALE)
    b = a[np.random.default_rng(512).permutation(len(a))]
    rays = rays_for(513)
    acc = Accelerator("wbvh").build(a).update(b)
    assert_matches_brute(b, rays, acc.intersect(rays))
    acc.check()


def test_wbvh_refit_round_trip_restores_answers(gpu):
    a = scenes.heightfield(res=48, seed=521, scale=SCALE)
    rays = rays_for(522)
    acc = Accelerator("wbvh").build(a)
    before = acc.intersect(rays)
    acc.update(moved(a, seed=523, amount=0.05 * SCALE)).update(a)
    after = acc.intersect(rays)
    assert np.array_equal(after["tri"], before["tri"])
    assert np.array_equal(bits(after["t"]), bits(before["t"]))


def test_any_hit_after_refit(gpu):
    a = scenes.heightfield(res=48, seed=531, scale=SCALE)
    b = moved(a, seed=532, amount=0.01 * SCALE)
    pts = np.random.default_rng(533).random((6000, 3)).astype(np.float32) * SCALE
    pts[:, 1] *= 0.3
    sh = scenes.shadow_rays(pts, seed=534, light_center=np.array([0.5, 2.0, 0.5]) * SCALE,
                            light_size=0.1 * SCALE, offset=0.01 * SCALE)
    want = ob.port_occluded(b, sh, clamp=True)
    for width in (4, 8):
        got = Accelerator("wbvh", width=width).build(a).update(b).occluded(sh)
        assert np.array_equal(got, want), width


def test_kdtree_update_is_reference_rebuild(gpu):
    """The kd layout rebuilds by the reference rules: bit-exact with the
    oracle's kd restatement built on the moved scene."""
    a = scenes.random_triangles(8000, seed=541, scale=SCALE)
    b = moved(a, seed=542, amount=0.03 * SCALE)
    rays = rays_for(543)
    acc = Accelerator("kdtree").build(a).update(b)
    got = acc.intersect(rays)
    want = ob.PortKd(b).closest(rays, clamp=True)
    assert np.array_equal(got["tri"], want["tri"])
    m = want["tri"] >= 0
    assert np.array_equal(bits(got["t"][m]), bits(want["t"][m]))
    lo = acc.info()["scene_lo"]
    assert np.allclose(lo, b.reshape(-1, 3).min(axis=0), rtol=0, atol=1e-3 * SCALE)


def test_update_rejects_a_different_triangle_count(gpu):
    a = scenes.random_triangles(500, seed=551, scale=SCALE)
    for kind in ("wbvh", "kdtree"):
        acc = Accelerator(kind).build(a)
        with pytest.raises(EncoreError) as ei:
            acc.update(a[:-1])
        assert ei.value.status == 1
        # the accelerator is unchanged and still answers
        rays = scenes.random_sphere_rays(500, seed=552, hi=(SCALE, SCALE, SCALE))
        assert_matches_brute(a, rays, acc.intersect(rays))


@pytest.mark.parametrize("kind,width", [("wbvh", 8), ("wbvh", 4), ("kdtree", 8)])
def test_saved_and_loaded_accelerator_answers_identically(gpu, kind, width):
    """enc_accel_serialize / enc_accel_deserialize: the loaded accelerator
    (no host build) gives every hit bit for bit, and a wide BVH loaded from
    its image refits like the original."""
    tris = scenes.random_triangles(30000, seed=95, scale=1000.0)
    rays = np.concatenate([
        scenes.camera_rays(96, 96, eye=np.array([0.5, 0.5, -1.5]) * 1000.0,
                           look=np.array([0.5, 0.5, 0.5]) * 1000.0),
        scenes.random_sphere_rays(20000, seed=96, hi=(1000.0, 1000.0, 1000.0))])
    acc = Accelerator(kind, width=width).build(tris)
    img = acc.save()
    acc2 = Accelerator.load(img)
    assert acc2.info()["nnodes"] == acc.info()["nnodes"]
    a, b = acc.intersect(rays), acc2.intersect(rays)
    assert np.array_equal(a.view(np.int32), b.view(np.int32))
    assert np.array_equal(acc.occluded(rays), acc2.occluded(rays))
    assert acc2.save() == img
    if kind == "wbvh":
        moved = tris + np.float32(3.0)
        acc.update(moved)
        acc2.update(moved)
        assert np.array_equal(acc.intersect(rays).view(np.int32), acc2.intersect(rays).view(np.int32))
    acc.destroy()
    acc2.destroy()
