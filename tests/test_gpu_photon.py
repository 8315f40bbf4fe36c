"""Parity of the CUDA photon gather with the reference PhotonMap (GPU).

Bars: the k-nearest set equals the reference's (as a set; ties at exactly
equal squared distance would be listed); radiance within 1e-4 relative of the
FP64 host oracle and of the reference's own FP32 estimate.
"""
from pathlib import Path

import numpy as np
import pytest

from encore_b200 import EncoreError, PhotonMap
from oracle import bindings as ob

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
RTOL = 1e-4


@pytest.mark.parametrize("name", ["photons20k_x1_ignore.npz", "photons20k_x1000_normal.npz"])
@pytest.mark.parametrize("caustic", [0, 1])
def test_gather_matches_reference_golden(gpu, name, caustic):
    g = np.load(GOLD / name)
    k, md, ign = int(g["k"]), float(g["max_dist"]), bool(g["ignore_normal"])
    pm = PhotonMap(len(g["pos"]), caustic=bool(caustic))
    pm.add_photons(g["pos"], g["nrm"], g["power"])
    idx, d2, cnt = pm.get_nearest_n_photons(k, md, g["qpos"], g["qnrm"], ignore_normal=ign)
    assert np.array_equal(cnt, g[f"count_c{caustic}"])
    ref_idx = g[f"idx_c{caustic}"]
    for i in range(len(cnt)):
        assert set(idx[i, :cnt[i]].tolist()) == set(ref_idx[i, :cnt[i]].tolist()), i
        assert np.all(np.diff(d2[i, :cnt[i]]) >= 0)  # ascending
        assert np.all(idx[i, cnt[i]:] == -1)
    rgb = pm.get_radiance_estimate(k, md, g["qpos"], g["qnrm"], ignore_normal=ign)
    np.testing.assert_allclose(rgb, g[f"rgb_c{caustic}"], rtol=RTOL, atol=1e-12)
    f64, _ = ob.port_gather(g["pos"], g["nrm"], g["power"], g["qpos"], g["qnrm"], k, md,
                            ignore_normal=ign, caustic=bool(caustic))
    np.testing.assert_allclose(rgb, f64, rtol=RTOL, atol=1e-12)


@pytest.mark.parametrize("k", [1, 7, 32, 33, 50, 64, 100, 200, 256])
def test_gather_k_sweep_matches_fp64_oracle(gpu, k):
    rng = np.random.default_rng(k)
    n = 60000
    pos = rng.random((n, 3), dtype=np.float32)
    nrm = np.tile(np.array([[0, 1, 0]], np.float32), (n, 1))
    nrm[::3] = (1, 0, 0)  # a third of the photons fail the normal filter
    pw = rng.random((n, 3), dtype=np.float32) / n
    q = rng.random((2000, 3), dtype=np.float32)
    qn = np.tile(np.array([[0, 1, 0]], np.float32), (2000, 1))
    for caustic in (False, True):
        pm = PhotonMap(n, caustic=caustic)
        pm.add_photons(pos, nrm, pw)
        rgb = pm.get_radiance_estimate(k, 0.05, q, qn)
        want, cnt = ob.port_gather(pos, nrm, pw, q, qn, k, 0.05, caustic=caustic)
        np.testing.assert_allclose(rgb, want, rtol=RTOL, atol=1e-12)
        idx, d2, gcnt = pm.get_nearest_n_photons(k, 0.05, q, qn)
        assert np.array_equal(gcnt, cnt)


@pytest.mark.parametrize("n", [65537, 67584])
@pytest.mark.parametrize("k", [1, 50, 100])
def test_gather_paired_leaves_match_fp64_oracle(gpu, n, k):
    # The build splits down to leaves of at most 32 photons, so leaves hold
    # between 16 and 32. Only just above 16 * 2^d do leaves of 16 appear,
    # two of which the gather tests in one warp step. 65,537 photons give
    # 4,096 leaves of 16 (one of 17); 67,584 give 16s and 17s half and half,
    # so some sibling pairs fit in a step and some do not.
    rng = np.random.default_rng(n + k)
    pos = rng.random((n, 3), dtype=np.float32)
    nrm = np.tile(np.array([[0, 1, 0]], np.float32), (n, 1))
    nrm[::4] = (0, 0, 1)
    pw = rng.random((n, 3), dtype=np.float32) / n
    q = rng.random((2000, 3), dtype=np.float32)
    qn = np.tile(np.array([[0, 1, 0]], np.float32), (2000, 1))
    for caustic in (False, True):
        pm = PhotonMap(n, caustic=caustic)
        pm.add_photons(pos, nrm, pw)
        rgb = pm.get_radiance_estimate(k, 0.06, q, qn)
        want, cnt = ob.port_gather(pos, nrm, pw, q, qn, k, 0.06, caustic=caustic)
        np.testing.assert_allclose(rgb, want, rtol=RTOL, atol=1e-12)
        idx, d2, gcnt = pm.get_nearest_n_photons(k, 0.06, q, qn)
        assert np.array_equal(gcnt, cnt)


def test_gather_edge_cases(gpu):
    pm = PhotonMap(10)
    pm.balance_and_construct()  # empty map
    q = np.zeros((3, 3), np.float32)
    qn = np.zeros((3, 3), np.float32)
    assert np.all(pm.get_radiance_estimate(50, 1.0, q, qn) == 0)
    pm2 = PhotonMap(4)
    taken = pm2.add_photons(np.zeros((6, 3), np.float32), np.zeros((6, 3), np.float32),
                            np.ones((6, 3), np.float32))
    assert taken == 4 and pm2.full()  # AddPhoton drops photons beyond capacity
    rgb = pm2.get_radiance_estimate(50, 1.0, q, qn)
    assert np.allclose(rgb, 4.0)
    assert np.all(pm2.get_radiance_estimate(0, 1.0, q, qn) == 0)  # N = 0
    with pytest.raises(EncoreError):
        pm2.get_radiance_estimate(300, 1.0, q, qn)  # k above the built limit


def test_nan_normals_never_match(gpu):
    # H10: with the reference filter, NaN normals compare unequal, so nothing is found
    n = 1000
    pos = np.random.default_rng(1).random((n, 3), dtype=np.float32)
    nrm = np.full((n, 3), np.nan, np.float32)
    pm = PhotonMap(n)
    pm.add_photons(pos, nrm, np.ones((n, 3), np.float32))
    q = pos[:10]
    assert np.all(pm.get_radiance_estimate(50, 1.0, q, nrm[:10]) == 0)
    assert np.all(pm.get_radiance_estimate(50, 1.0, q, nrm[:10], ignore_normal=True) > 0)


def test_saved_and_loaded_photon_map_answers_identically(gpu):
    """enc_photonmap_serialize / _deserialize: the loaded map (no host
    balance) gives the same radiance and k-nearest sets bit for bit."""
    rng = np.random.default_rng(97)
    n = 30000
    pos = rng.random((n, 3), dtype=np.float32) * 1000
    nrm = np.tile(np.array([[0, 1, 0]], np.float32), (n, 1))
    pw = rng.random((n, 3), dtype=np.float32)
    q = rng.random((2000, 3), dtype=np.float32) * 1000
    qn = np.tile(np.array([[0, 1, 0]], np.float32), (2000, 1))
    for caustic in (False, True):
        pm = PhotonMap(n, caustic=caustic)
        pm.add_photons(pos, nrm, pw)
        a = pm.get_radiance_estimate(50, 60.0, q, qn)
        ia, da, ca = pm.get_nearest_n_photons(50, 60.0, q, qn)
        img = pm.save()
        pm2 = PhotonMap.load(img)
        assert pm2.caustic == caustic and pm2.count() == n
        b = pm2.get_radiance_estimate(50, 60.0, q, qn)
        ib, db, cb = pm2.get_nearest_n_photons(50, 60.0, q, qn)
        assert np.array_equal(a.view(np.int32), b.view(np.int32))
        assert np.array_equal(ia, ib) and np.array_equal(ca, cb)
        assert pm2.save() == img
