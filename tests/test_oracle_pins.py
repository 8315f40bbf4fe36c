"""Pins the C oracle (oracle/encore_oracle.c) to the reference.

Golden vectors in tests/golden/ were produced by the reference's own CPU code
(tests/golden/make_golden.py).  When oracle/_ref/libencore_ref.so is present
the oracle is also compared with it live on fresh inputs.
"""
from pathlib import Path

import numpy as np
import pytest

from encore_b200 import scenes
from oracle import bindings as ob

GOLD = Path(__file__).resolve().parent / "golden"


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


def assert_hits_equal(h, tri, t, u, v):
    assert np.array_equal(h["tri"], tri)
    m = tri >= 0
    assert np.array_equal(bits(h["t"][m]), bits(t[m]))
    assert np.array_equal(bits(h["u"][m]), bits(u[m]))
    assert np.array_equal(bits(h["v"][m]), bits(v[m]))


@pytest.mark.parametrize("name", ["random2k_x1.npz", "random2k_x1000.npz", "heightfield64_x1000.npz"])
def test_kd_port_matches_reference_golden(name):
    g = np.load(GOLD / name)
    kd = ob.PortKd(g["tris"])
    h = kd.closest(g["rays"], clamp=True)
    assert_hits_equal(h, g["kd_tri"], g["kd_t"], g["kd_u"], g["kd_v"])


@pytest.mark.parametrize("name", ["random2k_x1.npz", "random2k_x1000.npz"])
def test_brute_port_matches_reference_basicas(name):
    g = np.load(GOLD / name)
    h = ob.port_brute(g["tris"], g["rays"], clamp=True)
    assert_hits_equal(h, g["basic_tri"], g["basic_t"], g["basic_u"], g["basic_v"])


def test_x1000_predicate_is_geometric_on_golden():
    # At x1000 the reference Kdtree, Bvh and BasicAS agree and match brute force.
    g = np.load(GOLD / "random2k_x1000.npz")
    assert np.array_equal(g["kd_tri"], g["basic_tri"])
    assert np.array_equal(g["kd_tri"], g["bvh_tri"])


def test_unit_scale_candidate_sets_differ_on_golden():
    # At unit scale the clamped predicate accepts off-triangle "hits", so each
    # reference accelerator returns a different closest hit on some rays.
    g = np.load(GOLD / "random2k_x1.npz")
    assert (g["kd_tri"] != g["basic_tri"]).sum() > 0


def test_occluded_port_matches_reference_golden_x1000():
    g = np.load(GOLD / "random2k_x1000.npz")
    occ = ob.port_occluded(g["tris"], g["shadow_rays"], clamp=True)
    assert np.array_equal(occ, g["kd_occluded"])


@pytest.mark.parametrize("name", ["photons20k_x1_ignore.npz", "photons20k_x1000_normal.npz"])
@pytest.mark.parametrize("caustic", [0, 1])
def test_gather_port_matches_reference_golden(name, caustic):
    g = np.load(GOLD / name)
    k, md, ign = int(g["k"]), float(g["max_dist"]), bool(g["ignore_normal"])
    rgb, cnt, idx, d2 = ob.port_gather(g["pos"], g["nrm"], g["power"], g["qpos"], g["qnrm"], k,
                                       md, ignore_normal=ign, caustic=bool(caustic),
                                       with_sets=True)
    assert np.array_equal(cnt, g[f"count_c{caustic}"])
    ref_idx = g[f"idx_c{caustic}"]
    for i in range(len(cnt)):
        a = set(idx[i, :cnt[i]].tolist())
        b = set(ref_idx[i, :cnt[i]].tolist())
        assert a == b, f"query {i}: k-nearest sets differ"
    ref_rgb = g[f"rgb_c{caustic}"].astype(np.float64)
    np.testing.assert_allclose(rgb, ref_rgb, rtol=1e-4, atol=1e-12)


def test_kd_port_matches_live_reference(ref_lib):
    for scale in (1.0, 1000.0):
        tris = scenes.random_triangles(5000, seed=77, scale=scale)
        rays = np.concatenate([
            scenes.camera_rays(96, 96, eye=np.array([0.5, 0.5, -1.5]) * scale,
                               look=np.array([0.5, 0.5, 0.5]) * scale),
            scenes.random_sphere_rays(3000, seed=78, hi=(scale, scale, scale))])
        ref, _ = ob.ref_closest(tris, rays, kind=0)
        h = ob.PortKd(tris).closest(rays, clamp=True)
        assert_hits_equal(h, ref["tri"], ref["t"], ref["u"], ref["v"])


def test_f64_oracle_agrees_with_fp32_at_x1000():
    g = np.load(GOLD / "random2k_x1000.npz")
    f64 = ob.port_f64(g["tris"], g["rays"])
    assert np.array_equal(f64["tri"], g["kd_tri"])
    m = f64["tri"] >= 0
    np.testing.assert_allclose(f64["t"][m], g["kd_t"][m], rtol=1e-5)


# ---- f2: ray generation and hit surfaces ------------------------------------

def _camera_cases():
    g = np.load(GOLD / "camera_surface.npz")
    for i in range(int(g["ncams"])):
        p = g[f"cam{i}_params"]
        yield (tuple(p[0:3]), tuple(p[3:6]), tuple(p[6:9]), float(p[9]), int(p[10]),
               int(p[11])), g[f"cam{i}_rays"]


def test_camera_restatement_matches_reference_golden():
    """scenes.camera_rays (the host restatement of RayTracer::CalcEyeRaySamples
    with Camera::CalcCamVectors) equals, bit for bit, the rays the reference's
    own Camera and Vector3 code produced (tests/golden/camera_surface.npz)."""
    for (eye, look, up, fov, w, h), want in _camera_cases():
        got = scenes.camera_rays(w, h, eye=np.array(eye), look=np.array(look), up=up, fov_deg=fov)
        assert np.array_equal(bits(got[:, :7]), bits(want[:, :7])), (eye, look, up)
        assert np.all(np.isinf(got[:, 7])) and np.all(np.isinf(want[:, 7]))


def test_camera_golden_matches_live_reference(ref_lib):
    for (eye, look, up, fov, w, h), want in _camera_cases():
        live = ob.ref_camera_rays(eye, look, up, fov, w, h)
        assert np.array_equal(bits(live), bits(want))


def test_surface_restatement_matches_reference_golden():
    """Hit point v0 + (v1-v0)*alpha + (v2-v0)*beta and normal
    Normalize(Cross(edge1, edge2)) restated in FP32 equal what the reference's
    TrianglePrim::intersect stored for the Kdtree's hits."""
    g = np.load(GOLD / "random2k_x1000.npz")
    s = np.load(GOLD / "camera_surface.npz")
    ids, u, v = g["kd_tri"], g["kd_u"], g["kd_v"]
    h = ids >= 0
    t = g["tris"].reshape(-1, 3, 3)[ids[h]]
    e1 = (t[:, 1] - t[:, 0]).astype(np.float32)
    e2 = (t[:, 2] - t[:, 0]).astype(np.float32)
    p = ((t[:, 0] + e1 * u[h][:, None]) + e2 * v[h][:, None]).astype(np.float32)
    n = scenes.normalize_ref(scenes.cross_ref(e1, e2))
    assert np.array_equal(bits(p), bits(s["surf_pos"][h]))
    assert np.array_equal(bits(n), bits(s["surf_nrm"][h]))
    assert np.all(np.isnan(s["surf_pos"][~h]))


def test_surface_golden_matches_live_reference(ref_lib):
    g = np.load(GOLD / "random2k_x1000.npz")
    s = np.load(GOLD / "camera_surface.npz")
    pos, nrm = ob.ref_hit_surface(g["tris"], g["rays"], g["kd_tri"])
    assert np.array_equal(bits(pos), bits(s["surf_pos"]))
    assert np.array_equal(bits(nrm), bits(s["surf_nrm"]))
