"""Device-side ray and photon generation (GPU): eye rays bit-exact with the
reference's own camera (RayTracer::CalcEyeRaySamples over Camera's basis),
hit surfaces bit-exact with what the reference's TrianglePrim::intersect
stores, diffuse rays with randDirectionSuperN's distribution, photon paths
well formed and reproducible, and the photon-map pipeline's radiance within
1e-4 of the FP64 oracle."""
import numpy as np
import pytest

from encore_b200 import Accelerator, PhotonMap, scenes, wavefront
from oracle import bindings as ob

pytestmark = pytest.mark.gpu
SCALE = 1000.0


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


GOLD = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def _camera_cases():
    g = np.load(GOLD / "camera_surface.npz")
    return [(g[f"cam{i}_params"], g[f"cam{i}_rays"]) for i in range(int(g["ncams"]))]


@pytest.mark.parametrize("case", range(4))
def test_camera_rays_bit_exact_with_reference(gpu, case):
    """camera_kernel against eye rays that the reference's own Camera basis and
    Vector3 arithmetic produced (tests/golden/camera_surface.npz, made by
    tests/golden/make_golden.py from the compiled reference)."""
    import torch
    p, want = _camera_cases()[case]
    eye, look, up, fov, w, h = tuple(p[0:3]), tuple(p[3:6]), tuple(p[6:9]), float(p[9]), int(p[10]), int(p[11])
    d = torch.empty((w * h, 8), dtype=torch.float32, device="cuda")
    wavefront.camera_rays(eye, look, up, fov, w, h, d)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    assert np.array_equal(bits(got[:, :7]), bits(want[:, :7]))
    assert np.all(np.isinf(got[:, 7]))


def test_hit_surface_bit_exact_with_reference(gpu):
    """surface_kernel on the reference Kdtree's hits (random2k x1000 golden)
    against the hit point and normal the reference's TrianglePrim::intersect
    stored for them."""
    import torch
    g = np.load(GOLD / "random2k_x1000.npz")
    s = np.load(GOLD / "camera_surface.npz")
    tris = g["tris"]
    n = len(g["rays"])
    hits = np.zeros(n, ob.HIT)
    hits["tri"], hits["t"], hits["u"], hits["v"] = g["kd_tri"], g["kd_t"], g["kd_u"], g["kd_v"]
    acc = Accelerator("wbvh").build(tris)
    d_hits = _t(hits.view(np.int32).reshape(-1, 4))
    d_pos = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    d_nrm = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    wavefront.hit_surface(acc, d_hits, n, d_pos, d_nrm)
    torch.cuda.synchronize()
    pos, nrm = d_pos.cpu().numpy(), d_nrm.cpu().numpy()
    h = hits["tri"] >= 0
    assert h.sum() > 500
    assert np.array_equal(bits(pos[h]), bits(s["surf_pos"][h]))
    assert np.array_equal(bits(nrm[h]), bits(s["surf_nrm"][h]))
    assert np.all(np.isnan(pos[~h]))
    acc.destroy()


def test_diffuse_rays_follow_the_reference_lobe(gpu):
    """diffuse_kernel's directions have randDirectionSuperN's distribution
    (Common.cpp:144-182): cos^2(theta) about the facing normal uniform on
    [0.001, 1), azimuth uniform.  A flat two-triangle floor seen from above
    gives every hit the normal +y, so theta and the azimuth are read directly;
    chi-square over 20 bins each (19 degrees of freedom: 99.99th percentile
    about 49), and the mean of cos(theta) against its exact value."""
    import torch
    s = 1000.0
    floor = np.array([[0, 0, 0, s, 0, 0, s, 0, s], [0, 0, 0, s, 0, s, 0, 0, s]], np.float32)
    acc = Accelerator("wbvh").build(floor)
    w = h = 256
    d_prim = torch.empty((w * h, 8), dtype=torch.float32, device="cuda")
    wavefront.camera_rays((0.5 * s, 2.0 * s, 0.5 * s), (0.5 * s, 0.0, 0.5 * s), (0.0, 0.0, 1.0), 25.0,
                          w, h, d_prim)
    d_hits = torch.empty((w * h, 4), dtype=torch.int32, device="cuda")
    acc.intersect_device(d_prim, w * h, d_hits)
    k = 4
    d_out = torch.empty((w * h * k, 8), dtype=torch.float32, device="cuda")
    wavefront.diffuse_rays(acc, d_prim, d_hits, w * h, k, 2024, 0.1, d_out)
    torch.cuda.synchronize()
    hit = np.repeat(d_hits[:, 0].cpu().numpy() >= 0, k)
    assert hit.all()
    d = d_out.cpu().numpy()[:, 4:7].astype(np.float64)
    ct = d[:, 1]  # the facing normal is +y (the camera is above the floor)
    assert ct.min() >= np.sqrt(0.001) - 1e-6
    n = len(ct)
    lo = 0.001
    mean_ct = (2.0 / 3.0) * (1 - lo ** 1.5) / (1 - lo)
    assert abs(ct.mean() - mean_ct) < 5 * np.sqrt((0.5 * (1 + lo) - mean_ct ** 2) / n)
    edges = np.linspace(lo, 1.0, 21)
    obs, _ = np.histogram(ct ** 2, bins=edges)
    exp = n / 20.0
    assert ((obs - exp) ** 2 / exp).sum() < 60.0
    phi = np.arctan2(d[:, 2], d[:, 0])
    obs, _ = np.histogram(phi, bins=np.linspace(-np.pi, np.pi, 21))
    assert ((obs - exp) ** 2 / exp).sum() < 60.0
    acc.destroy()


def test_diffuse_rays_well_formed_and_seeded(gpu):
    import torch
    tris = scenes.heightfield(res=64, seed=62, scale=SCALE)
    prim = scenes.camera_rays(64, 64, eye=np.array([0.5, 1.3, 0.5]) * SCALE,
                              look=np.array([0.5, 0.0, 0.5]) * SCALE, up=(0.0, 0.0, 1.0), fov_deg=50.0)
    acc = Accelerator("wbvh").build(tris)
    hits = acc.intersect(prim)
    d_prim, d_hits = _t(prim), _t(hits.view(np.int32).reshape(-1, 4))
    n, k = len(prim), 3
    outs = []
    for _ in range(2):
        d_out = torch.empty((n * k, 8), dtype=torch.float32, device="cuda")
        wavefront.diffuse_rays(acc, d_prim, d_hits, n, k, 77, 0.1, d_out)
        torch.cuda.synchronize()
        outs.append(d_out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    r = outs[0].reshape(n, k, 8)
    h = hits["tri"] >= 0
    d = r[h, :, 4:7].reshape(-1, 3)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    # every secondary leaves on the side the primary came from
    t = tris.reshape(-1, 3, 3)[hits["tri"][h]].astype(np.float64)
    g = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    g *= -np.sign(np.sum(g * prim[h, 4:7], axis=1))[:, None]
    assert np.all(np.sum(np.repeat(g, k, axis=0) * d, axis=1) > -1e-4)
    assert np.all(r[~h, :, 7] == 0)  # misses give empty rays
    # secondaries traced from the surface: no self hit at their own triangle at t ~ 0
    sec = np.ascontiguousarray(r[h].reshape(-1, 8))
    sh = acc.intersect(sec)
    assert np.all(sh["t"][sh["tri"] >= 0] > 0.05)


def test_photon_tracing_counts_and_reproducibility(gpu):
    import torch
    tris = scenes.random_triangles(10000, seed=63, scale=SCALE)
    acc = Accelerator("wbvh").build(tris)
    nph, cap = 100_000, 400_000
    res = []
    for _ in range(2):
        bufs = [torch.empty((cap, 3), dtype=torch.float32, device="cuda") for _ in range(3)]
        m = wavefront.trace_photons(acc, np.array([0.5, 2.0, 0.5]) * SCALE, 0.1 * SCALE, nph, *bufs,
                                    max_bounces=3, albedo=0.7, seed=5, emit_offset=0.01 * SCALE,
                                    bounce_offset=0.001 * SCALE)
        res.append((m, [b[:m].cpu().numpy() for b in bufs]))
    (m1, (p1, n1, w1)), (m2, (p2, n2, w2)) = res
    # the light sits at height 2 above the unit cube: most of its cosine lobe
    # misses the scene, about a fifth of the photons land
    assert m1 == m2 and m1 > nph // 10
    # photon paths are seeded per photon: the same set whatever the storage order
    o1, o2 = np.lexsort(p1.T), np.lexsort(p2.T)
    assert np.array_equal(p1[o1], p2[o2]) and np.array_equal(n1[o1], n2[o2])
    assert np.all(w1 == np.float32(1.0 / nph))
    lo, hi = tris.reshape(-1, 3).min(0), tris.reshape(-1, 3).max(0)
    assert np.all((p1 >= lo - 1) & (p1 <= hi + 1))
    # at most 1 + 3 hits per emitted photon
    assert m1 <= 4 * nph


def test_photon_pipeline_radiance_matches_fp64_oracle(gpu):
    import torch
    tris = scenes.random_triangles(10000, seed=64, scale=SCALE)
    acc = Accelerator("wbvh").build(tris)
    nph, cap = 200_000, 800_000
    bufs = [torch.empty((cap, 3), dtype=torch.float32, device="cuda") for _ in range(3)]
    m = wavefront.trace_photons(acc, np.array([0.5, 2.0, 0.5]) * SCALE, 0.1 * SCALE, nph, *bufs,
                                seed=9, emit_offset=0.01 * SCALE, bounce_offset=0.001 * SCALE)
    pm = wavefront.photon_map_from_device(bufs[0], bufs[1], bufs[2], m)
    w, h = 96, 96
    d_rays = torch.empty((w * h, 8), dtype=torch.float32, device="cuda")
    wavefront.camera_rays(np.array([0.5, 0.5, -1.5]) * SCALE, np.array([0.5, 0.5, 0.5]) * SCALE,
                          (0.0, 1.0, 0.0), 45.0, w, h, d_rays)
    d_hits = torch.empty((w * h, 4), dtype=torch.int32, device="cuda")
    acc.intersect_device(d_rays, w * h, d_hits)
    d_q = torch.empty((w * h, 3), dtype=torch.float32, device="cuda")
    d_n = torch.empty((w * h, 3), dtype=torch.float32, device="cuda")
    wavefront.hit_surface(acc, d_hits, w * h, d_q, d_n)
    torch.cuda.synchronize()
    ok = d_hits[:, 0].cpu().numpy() >= 0
    q, qn = d_q.cpu().numpy()[ok], d_n.cpu().numpy()[ok]
    rgb = pm.get_radiance_estimate(50, 0.02 * SCALE, q, qn)
    pos, nrm, pw = (b[:m].cpu().numpy() for b in bufs)
    want, cnt = ob.port_gather(pos, nrm, pw, q, qn, 50, 0.02 * SCALE)
    assert (cnt > 0).mean() > 0.5
    np.testing.assert_allclose(rgb, want, rtol=1e-4, atol=1e-12)
