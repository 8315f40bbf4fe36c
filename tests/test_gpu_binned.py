"""Binned closest hit (enc_intersect_closest_device_binned, GPU): the batch is
counting-sorted by a key of origin cell and direction cell before the
traversal, and the hits must be the unbinned launch's bit for bit -- binning
changes only which rays share a warp, never a ray's result -- and both must
match the oracle."""
import numpy as np
import pytest

from encore_b200 import Accelerator, BinConfig, EncoreError, scenes
from oracle import bindings as ob

pytestmark = pytest.mark.gpu


def _dev_hits(acc, rays, binning=None, device=0):
    import torch
    n = len(rays)
    d_rays = torch.from_numpy(np.ascontiguousarray(rays)).to(device)
    d_plain = torch.full((max(n, 1), 4), -7, dtype=torch.int32, device=device)
    d_bin = torch.full((max(n, 1), 4), -9, dtype=torch.int32, device=device)
    acc.intersect_device(d_rays, n, d_plain)
    scratch = torch.empty(acc.bin_scratch_bytes(n, binning), dtype=torch.uint8, device=device)
    acc.intersect_device_binned(d_rays, n, d_bin, scratch, binning)
    acc.check()
    return d_plain[:n].cpu().numpy(), d_bin[:n].cpu().numpy()


@pytest.fixture(scope="module")
def field():
    tris = scenes.heightfield(res=128, seed=3, scale=1000.0)
    acc = Accelerator("wbvh").build(tris)
    prim = scenes.camera_rays(128, 128, eye=np.array([0.5, 1.3, 0.5]) * 1000.0,
                              look=np.array([0.5, 0.0, 0.5]) * 1000.0, up=(0.0, 0.0, 1.0),
                              fov_deg=40.0)
    ph = acc.intersect(prim)
    sec = scenes.diffuse_rays(tris, prim, ph["tri"], ph["u"], ph["v"], per_hit=3, seed=4,
                              offset=0.1)
    rays = np.concatenate([prim, sec])
    rays = np.ascontiguousarray(rays[np.random.default_rng(5).permutation(len(rays))])
    return tris, rays, acc


@pytest.mark.parametrize("cfg", [None, BinConfig(10, 6), BinConfig(16, 0), BinConfig(0, 12),
                                 BinConfig(1, 0), BinConfig(12, 8), BinConfig(12, 0, 0.05),
                                 BinConfig(9, 9, 0.2)])
def test_binned_equals_plain_and_oracle(gpu, field, cfg):
    tris, rays, acc = field
    plain, binned = _dev_hits(acc, rays, cfg)
    assert np.array_equal(plain, binned)
    sub = np.arange(0, len(rays), 7)
    want = ob.port_brute(tris, rays[sub], clamp=True)
    got = binned[sub]
    mism, classes = ob.classify(tris, rays[sub], got.view(ob.HIT).reshape(-1), want)
    # shared-edge ties, and brute-force hits that are clamp artefacts outside
    # their triangle's box (no tree reaches them)
    assert set(classes) <= {"tie", "edge", "want_false_positive"}, classes
    assert len(mism) <= len(sub) // 500 + 2


@pytest.mark.parametrize("n", [1, 31, 33, 1000, 4097])
def test_binned_ragged_sizes(gpu, field, n):
    tris, rays, acc = field
    plain, binned = _dev_hits(acc, rays[:n])
    assert np.array_equal(plain, binned)


def test_binned_random_triangles_unit_scale(gpu):
    """The CPU-runnable plain case at unit scale (clamp artefacts included):
    binning must not change a single result."""
    tris = scenes.random_triangles(10000, seed=0, scale=1.0)
    rays = scenes.camera_rays(256, 256, eye=np.array([0.5, 0.5, -1.5]),
                              look=np.array([0.5, 0.5, 0.5]))
    sph = scenes.random_sphere_rays(20000, seed=9)
    rays = np.concatenate([rays, sph])
    acc = Accelerator("wbvh").build(tris)
    plain, binned = _dev_hits(acc, rays, BinConfig(8, 8))
    assert np.array_equal(plain, binned)
    acc.destroy()


def test_binned_argument_errors(gpu, field):
    import torch
    tris, rays, acc = field
    n = 1000
    d_rays = torch.from_numpy(rays[:n]).to(0)
    d_hits = torch.empty((n, 4), dtype=torch.int32, device=0)
    need = acc.bin_scratch_bytes(n)
    small = torch.empty(need - 256, dtype=torch.uint8, device=0)
    with pytest.raises(EncoreError):
        acc.intersect_device_binned(d_rays, n, d_hits, small)
    big = torch.empty(need + 256, dtype=torch.uint8, device=0)
    with pytest.raises(EncoreError):  # not 256-byte aligned
        acc.intersect_device_binned(d_rays, n, d_hits, big[16:])
    with pytest.raises(EncoreError):  # more than 20 key bits
        acc.bin_scratch_bytes(n, BinConfig(16, 8))
    acc.intersect_device_binned(d_rays, 0, d_hits, big)  # empty batch: nothing to do


def test_binned_kd_parity_mode_is_unchanged(gpu, field):
    """The kd-tree parity mode walks the binned order too; every hit is the
    unbinned walk's (and so the reference Kdtree's) bit for bit."""
    tris, rays, acc = field
    kd = Accelerator("kdtree").build(tris)
    plain, binned = _dev_hits(kd, rays)
    assert np.array_equal(plain, binned)
    kd.destroy()


def test_bin_then_ordered_trace_equals_plain(gpu, field):
    """enc_bin_rays + enc_intersect_closest_device_ordered (the binned call in
    two halves) and any permutation given directly give the plain hits."""
    import torch
    tris, rays, acc = field
    n = len(rays)
    d_rays = torch.from_numpy(rays).to(0)
    d_plain = torch.empty((n, 4), dtype=torch.int32, device=0)
    acc.intersect_device(d_rays, n, d_plain)
    scratch = torch.empty(acc.bin_scratch_bytes(n), dtype=torch.uint8, device=0)
    order = acc.bin_rays(d_rays, n, scratch)
    d_hits = torch.full((n, 4), -5, dtype=torch.int32, device=0)
    acc.intersect_device_ordered(d_rays, n, order, d_hits)
    acc.check()
    assert torch.equal(d_hits, d_plain)
    # the permutation is one: every ray index exactly once
    base = scratch.data_ptr()
    off = order - base
    perm = scratch[off:off + 4 * n].view(torch.int32).cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(n))
    rev = torch.arange(n - 1, -1, -1, dtype=torch.int32, device=0)
    d_rev = torch.full((n, 4), -5, dtype=torch.int32, device=0)
    acc.intersect_device_ordered(d_rays, n, rev, d_rev)
    acc.check()
    assert torch.equal(d_rev, d_plain)


def test_ordered_trace_skips_and_reports_entries_outside_the_batch(gpu, field):
    import torch
    tris, rays, acc = field
    n = 2000
    d_rays = torch.from_numpy(rays[:n]).to(0)
    d_plain = torch.empty((n, 4), dtype=torch.int32, device=0)
    acc.intersect_device(d_rays, n, d_plain)
    order = torch.arange(n, dtype=torch.int32, device=0)
    order[7] = n + 5  # outside the batch: skipped, reported, never read
    d_hits = torch.full((n, 4), -5, dtype=torch.int32, device=0)
    acc.intersect_device_ordered(d_rays, n, order, d_hits)
    with pytest.raises(EncoreError):
        acc.check()
    acc.check()  # the report is cleared by the check that returned it
    got, want = d_hits.cpu().numpy(), d_plain.cpu().numpy()
    keep = np.ones(n, bool)
    keep[7] = False
    assert np.array_equal(got[keep], want[keep])
    assert np.all(got[7] == -5)
