"""A scene file through the whole path (GPU): loaded by the engine's
front-end, built, traced from the scene's own CAMERA, shadow-tested toward
its RECT_LIGHT, then animated frame by frame with refits (the loop of
DynamicScene::UpdateFrame, ENCORE/src/scene/DynamicScene.cpp:25-36).  The
scene is a Cornell-style box written by the test (unit-quad walls scaled to
100, a random mesh inside)."""
import numpy as np
import pytest

from encore_b200 import Accelerator, scene_io, scenes
from oracle import bindings as ob
from tests.scene_files import mesh, write_ply

pytestmark = pytest.mark.gpu


def cornell(tmp_path):
    models = tmp_path / "models"
    models.mkdir()
    quad = np.array([[0, 0, 0], [0, 0, 1], [1, 0, 1], [1, 0, 0]], np.float32)
    faces = np.array([[0, 1, 2], [2, 3, 0]])
    write_ply(models / "floor.ply", quad, faces)
    write_ply(models / "wall.ply", quad[:, [1, 2, 0]], faces)   # a quad in x = 0 (yz plane)
    write_ply(models / "back.ply", quad[:, [0, 2, 1]], faces)   # a quad in z = 0 (xy plane)
    v, f = mesh(31, nv=400, nf=800)
    write_ply(models / "blob.ply", v, f)
    (tmp_path / "cornell.txt").write_text("""* box of walls, a ceiling light and a mesh *
CAMERA 0 0 170 0 0 0 0 1 0 45 1 0.1 1000
MATERIAL 0.9 0.9 0.9 0 0 0 0 0 0 0 0 0 0
RECT_LIGHT 1.0 1.0 1.0
MATERIAL 0.7 0.7 0.7 0 0 0 0.1 0.1 0.1 0 0 0 0
MODEL models/floor.ply 0 -50 0 100 0 0 1 0
MODEL models/floor.ply 0 50 0 100 0 0 1 0
MODEL models/wall.ply 50 0 0 100 0 0 1 0
MODEL models/wall.ply -50 0 0 100 0 0 1 0
MODEL models/back.ply 0 0 -50 100 0 0 1 0
MATERIAL 0.36 0.36 0.6 0 0 0 0.05 0.05 0.05 0 0 0 0
MODEL models/blob.ply 0 -20 0 40 30 0 1 0
""")
    return scene_io.load_scene(tmp_path / "cornell.txt", model_dir=tmp_path)


def test_scene_file_camera_and_light(gpu, tmp_path):
    sc = cornell(tmp_path)
    d = sc.desc
    assert d["ntris"] == 2 + 5 * 2 + 800
    rays = scenes.camera_rays(128, 128, eye=d["cam_eye"], look=d["cam_look"], up=d["cam_up"],
                              fov_deg=d["cam_fov_deg"], near=d["cam_near"])
    for kind in ("wbvh", "kdtree"):
        acc = Accelerator(kind).build(sc.tris)
        got = acc.intersect(rays)
        want = (ob.PortKd(sc.tris).closest(rays, clamp=True) if kind == "kdtree"
                else ob.port_brute(sc.tris, rays, clamp=True))
        if kind == "kdtree":
            assert np.array_equal(got["tri"], want["tri"])
        else:
            mism, classes = ob.classify(sc.tris, rays, got, want)
            assert "unexplained" not in classes
            assert len([c for c in classes if c != "tie"]) <= 3
        # every eye ray inside the closed box hits something
        assert (got["tri"] >= 0).mean() > 0.95
    # shadow rays from the visible points toward the ceiling light
    acc = Accelerator("wbvh").build(sc.tris)
    h = acc.intersect(rays)
    m = h["tri"] >= 0
    pts = scenes.hit_points(sc.tris, rays[m], h["tri"][m], h["u"][m], h["v"][m])
    L = sc.lights[0]
    sh = scenes.shadow_rays(pts, seed=32, light_center=np.asarray(L["center"]), light_size=L["size"],
                            offset=0.01)
    assert np.array_equal(acc.occluded(sh), ob.port_occluded(sc.tris, sh, clamp=True))


def test_animated_frames_refit(gpu, tmp_path):
    """The mesh inside the box moves each frame; the accelerator is refit,
    never rebuilt, and answers like brute force on every frame."""
    sc = cornell(tmp_path)
    d = sc.desc
    rays = scenes.camera_rays(96, 96, eye=d["cam_eye"], look=d["cam_look"], up=d["cam_up"],
                              fov_deg=d["cam_fov_deg"], near=d["cam_near"])
    moving = sc.material_of_tri == sc.material_of_tri.max()
    acc = Accelerator("wbvh").build(sc.tris)
    tris = sc.tris.copy()
    for frame in range(4):
        tris[moving] = sc.tris[moving] + np.tile(np.float32([8.0 * frame, 3.0 * frame, 0.0]), 3)
        acc.update(tris)
        got = acc.intersect(rays)
        want = ob.port_brute(tris, rays, clamp=True)
        mism, classes = ob.classify(tris, rays, got, want)
        assert "unexplained" not in classes, frame
        assert len([c for c in classes if c != "tie"]) <= 3, frame
