import numpy as np

from encore_b200 import scenes


def test_random_triangles_deterministic_and_sized():
    a = scenes.random_triangles(1000, seed=3)
    b = scenes.random_triangles(1000, seed=3)
    assert a.shape == (1000, 9) and a.dtype == np.float32
    assert np.array_equal(a, b)
    t = a.reshape(-1, 3, 3).astype(np.float64)
    c = t.mean(axis=1)
    d = np.linalg.norm(t - c[:, None, :], axis=2)
    assert d.max() < 0.1  # vertices lie within 0.05 of the generating centroid


def test_heightfield_triangle_count_and_amplitude():
    h = scenes.heightfield(res=32, seed=1)
    assert h.shape == (2 * 32 * 32, 9)
    y = h.reshape(-1, 3)[:, 1]
    assert 0.0 <= y.min() and y.max() <= 0.2 + 1e-6
    assert np.array_equal(h, scenes.heightfield(res=32, seed=1))


def test_heightfield_full_size_is_2m_triangles():
    assert 2 * 1024 * 1024 == 2_097_152


def test_camera_rays_unit_directions():
    r = scenes.camera_rays(16, 8, eye=(0.5, 0.5, -1.5), look=(0.5, 0.5, 0.5))
    assert r.shape == (128, 8)
    n = np.linalg.norm(r[:, 4:7].astype(np.float64), axis=1)
    assert np.allclose(n, 1.0, atol=1e-5)
    assert np.all(r[:, 6] > 0)  # looking down +z


def test_cross_ref_clamps_small_components():
    c = scenes.cross_ref(np.array([1e-2, 0, 0], np.float32), np.array([0, 5e-2, 0], np.float32))
    assert c[2] == 0.0  # 5e-4 < 0.001 -> clamped
