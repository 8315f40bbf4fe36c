"""Generates the golden vectors in tests/golden/ from the reference itself.

The reference publishes no test vectors, so these fixtures are outputs of the
reference's own CPU code (Kdtree, Bvh, BasicAS, PhotonMap), compiled from its
sources by oracle/Makefile into oracle/_ref/libencore_ref.so, on seeded
synthetic inputs.  Inputs are stored with the outputs so a fixture stays
valid if a generator changes.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from encore_b200 import scenes  # noqa: E402
from oracle import bindings as ob  # noqa: E402

OUT = Path(__file__).resolve().parent


def hits_fields(prefix: str, h: np.ndarray) -> dict:
    return {f"{prefix}_tri": h["tri"], f"{prefix}_t": h["t"], f"{prefix}_u": h["u"],
            f"{prefix}_v": h["v"]}


def random_scene_fixture(scale: float) -> None:
    tris = scenes.random_triangles(2000, seed=11, scale=scale)
    cam = scenes.camera_rays(64, 64, eye=np.array([0.5, 0.5, -1.5]) * scale,
                             look=np.array([0.5, 0.5, 0.5]) * scale)
    sph = scenes.random_sphere_rays(1024, seed=12, lo=(0.0, 0.0, 0.0), hi=(scale, scale, scale))
    rays = np.concatenate([cam, sph]).astype(np.float32)
    kd, _ = ob.ref_closest(tris, rays, kind=0)
    bvh, _ = ob.ref_closest(tris, rays, kind=1)
    basic, _ = ob.ref_closest(tris, rays, kind=2)
    # shadow rays from kd hits toward the light (IsInShadow form)
    h = kd["tri"] >= 0
    pts = scenes.hit_points(tris, rays[h], kd["tri"][h], kd["u"][h], kd["v"][h])
    sh = scenes.shadow_rays(pts, seed=13, light_center=np.array([0.5, 2.0, 0.5]) * scale,
                            light_size=0.1 * scale, offset=0.01 * scale)
    occ = ob.ref_occluded(tris, sh, kind=0)
    name = f"random2k_x{int(scale)}.npz"
    np.savez_compressed(OUT / name, tris=tris, rays=rays, shadow_rays=sh, kd_occluded=occ,
                        **hits_fields("kd", kd), **hits_fields("bvh", bvh),
                        **hits_fields("basic", basic))
    print(name, "kd hits", int((kd["tri"] >= 0).sum()), "occluded", int(occ.sum()))


def heightfield_fixture() -> None:
    scale = 1000.0
    tris = scenes.heightfield(res=64, seed=21, scale=scale)
    prim = scenes.camera_rays(32, 32, eye=np.array([0.5, 1.3, 0.5]) * scale,
                              look=np.array([0.5, 0.0, 0.5]) * scale, up=(0.0, 0.0, 1.0),
                              fov_deg=40.0)
    kd0, _ = ob.ref_closest(tris, prim, kind=0)
    sec = scenes.diffuse_rays(tris, prim, kd0["tri"], kd0["u"], kd0["v"], per_hit=2, seed=22,
                              offset=1e-4 * scale)
    rays = np.concatenate([prim, sec]).astype(np.float32)
    kd, _ = ob.ref_closest(tris, rays, kind=0)
    np.savez_compressed(OUT / "heightfield64_x1000.npz", tris=tris, rays=rays, **hits_fields("kd", kd))
    print("heightfield64_x1000.npz kd hits", int((kd["tri"] >= 0).sum()), "of", len(rays))


def photon_fixture(scale: float, ignore_normal: bool) -> None:
    rng = np.random.default_rng(31)
    tris = scenes.random_triangles(300, seed=32, scale=scale)
    nrm = scenes.tri_normals_ref(tris)
    t = tris.reshape(-1, 3, 3).astype(np.float64)

    def points_on(ids):
        r1 = rng.random(len(ids))
        r2 = rng.random(len(ids))
        s = np.sqrt(r1)
        a, b = 1 - s, s * (1 - r2)
        c = s * r2
        p = a[:, None] * t[ids, 0] + b[:, None] * t[ids, 1] + c[:, None] * t[ids, 2]
        return p.astype(np.float32)

    pid = rng.integers(0, len(tris), size=20000)
    pos = points_on(pid)
    pn = nrm[pid]
    power = np.full((len(pid), 3), 1.0 / len(pid), dtype=np.float32)
    qid = rng.integers(0, len(tris), size=400)
    qpos = points_on(qid)
    qn = nrm[qid]
    lib = ob.reference()
    import ctypes as C
    k, md = 50, np.float32(0.02 * scale)
    out = {}
    for caustic in (0, 1):
        bs = C.c_double()
        h = lib.encref_pmap_create(pos.ctypes.data, pn.ctypes.data, power.ctypes.data, len(pos),
                                   caustic, C.byref(bs))
        lib.encref_set_ignore_normal(int(ignore_normal))
        rgb = np.empty((len(qpos), 3), np.float32)
        lib.encref_pmap_radiance(h, qpos.ctypes.data, qn.ctypes.data, len(qpos), k, md,
                                 rgb.ctypes.data, 0)
        idx = np.empty((len(qpos), k), np.int32)
        d2 = np.empty((len(qpos), k), np.float32)
        cnt = np.empty(len(qpos), np.int32)
        lib.encref_pmap_nearest(h, qpos.ctypes.data, qn.ctypes.data, len(qpos), k, md,
                                idx.ctypes.data, d2.ctypes.data, cnt.ctypes.data, 0)
        lib.encref_set_ignore_normal(0)
        lib.encref_pmap_destroy(h)
        out[f"rgb_c{caustic}"] = rgb
        out[f"idx_c{caustic}"] = idx
        out[f"d2_c{caustic}"] = d2
        out[f"count_c{caustic}"] = cnt
    name = f"photons20k_x{int(scale)}_{'ignore' if ignore_normal else 'normal'}.npz"
    np.savez_compressed(OUT / name, pos=pos, nrm=pn, power=power, qpos=qpos, qnrm=qn,
                        k=np.int32(k), max_dist=md, ignore_normal=np.int32(ignore_normal), **out)
    print(name, "mean count", float(out["count_c0"].mean()))


CAMERAS = [
    # eye, look, up, vertical fov, width, height
    ((0.5, 0.5, -1.5), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 45.0, 64, 48),
    ((500.0, 1300.0, 500.0), (500.0, 0.0, 500.0), (0.0, 0.0, 1.0), 40.0, 33, 65),
    ((500.0, 500.0, -1500.0), (500.0, 500.0, 500.0), (0.0, 1.0, 0.0), 45.0, 128, 128),
    ((-2.0, 3.0, 4.0), (0.25, 0.0, -0.5), (0.3, 1.0, 0.1), 60.0, 40, 30),
]


def camera_surface_fixture() -> None:
    """Eye rays from the reference's Camera basis and Vector3 arithmetic
    (the formula of RayTracer::CalcEyeRaySamples), and the hit point and
    normal the reference's TrianglePrim::intersect stores for the Kdtree's
    hits on the random2k x1000 scene."""
    out = {}
    for i, (eye, look, up, fov, w, h) in enumerate(CAMERAS):
        out[f"cam{i}_params"] = np.array([*eye, *look, *up, fov, w, h], np.float64)
        out[f"cam{i}_rays"] = ob.ref_camera_rays(eye, look, up, fov, w, h)
    g = np.load(OUT / "random2k_x1000.npz")
    tris, rays, ids = g["tris"], g["rays"], g["kd_tri"]
    pos, nrm = ob.ref_hit_surface(tris, rays, ids)
    out.update(ncams=np.int32(len(CAMERAS)), surf_ids=ids, surf_pos=pos, surf_nrm=nrm)
    np.savez_compressed(OUT / "camera_surface.npz", **out)
    print("camera_surface.npz", len(CAMERAS), "cameras,", int((ids >= 0).sum()), "surfaces")


FIXTURES = {
    "random2k_x1": lambda: random_scene_fixture(1.0),
    "random2k_x1000": lambda: random_scene_fixture(1000.0),
    "heightfield64_x1000": heightfield_fixture,
    "photons20k_x1_ignore": lambda: photon_fixture(1.0, ignore_normal=True),
    "photons20k_x1000_normal": lambda: photon_fixture(1000.0, ignore_normal=False),
    "camera_surface": camera_surface_fixture,
}


if __name__ == "__main__":
    # python tests/golden/make_golden.py [fixture ...]   (no names: all of them)
    if ob.reference() is None:
        sys.exit("oracle/_ref/libencore_ref.so missing: run `make -C oracle ref` first")
    for name in (sys.argv[1:] or list(FIXTURES)):
        FIXTURES[name]()
