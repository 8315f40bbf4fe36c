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
