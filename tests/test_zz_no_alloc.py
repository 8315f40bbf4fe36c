"""enc_intersect_closest_noalloc: the closest-hit entry point for callers that
must not allocate device memory while answering queries (their framework owns
the device memory, or their frame loop cannot take an allocation's device-wide
synchronisation).  Its scratch is a fixed array inside the library, so its
results must equal those of the allocating entry point, enc_intersect_closest,
and the oracle's, on consecutive calls that reuse that array; and once the
accelerator is built, its calls must not change the device's free memory.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from encore_b200 import _lib, scenes
from encore_b200.accel import HIT_DTYPE
from oracle import bindings as ob

pytestmark = pytest.mark.gpu


def _build(lib, tris):
    scene = C.c_void_p()
    assert lib.enc_scene_create(tris.ctypes.data, len(tris), C.byref(scene)) == _lib.ENC_OK
    acc = C.c_void_p()
    opts = _lib.BuildOpts(_lib.ENC_ACCEL_WBVH, 8, 3, _lib.ENC_PRED_REFERENCE)
    assert lib.enc_accel_build(scene, C.byref(opts), 0, C.byref(acc)) == _lib.ENC_OK
    lib.enc_scene_destroy(scene)
    return acc


def test_noalloc_matches_allocating_entry_point_on_two_calls(gpu):
    lib = _lib.load()
    scale = 1000.0
    tris = np.ascontiguousarray(scenes.random_triangles(20000, seed=1201, scale=scale))
    acc = _build(lib, tris)
    try:
        batches = [
            np.ascontiguousarray(scenes.camera_rays(
                192, 192, eye=np.array([0.5, 0.5, -1.5]) * scale,
                look=np.array([0.5, 0.5, 0.5]) * scale)),
            np.ascontiguousarray(scenes.random_sphere_rays(
                50000, seed=1202, hi=(scale, scale, scale))),
        ]
        for rays in batches:  # two calls in a row through the shared scratch
            n = len(rays)
            assert n <= 65536
            want = np.empty(n, HIT_DTYPE)
            assert lib.enc_intersect_closest(acc, rays.ctypes.data, n, want.ctypes.data, None,
                                             None) == _lib.ENC_OK
            got = np.empty(n, HIT_DTYPE)
            st = lib.enc_intersect_closest_noalloc(acc, rays.ctypes.data, n, got.ctypes.data, None)
            assert st == _lib.ENC_OK, lib.enc_last_error()
            assert (want["tri"] >= 0).sum() > n // 10
            # the same kernel on the same inputs: identical, bit for bit
            assert np.array_equal(got["tri"], want["tri"])
            for f in ("t", "u", "v"):
                assert np.array_equal(got[f].view(np.int32), want[f].view(np.int32))
            # and the oracle's brute force with the reference predicate agrees
            # on a sample, up to shared-edge ties
            sub = np.arange(0, n, 13)
            oracle = ob.port_brute(tris, rays[sub], clamp=True)
            mism, classes = ob.classify(tris, rays[sub], got[sub], oracle)
            assert set(classes) <= {"tie", "edge"}, classes
    finally:
        lib.enc_accel_destroy(acc)


def test_noalloc_calls_leave_free_device_memory_unchanged(gpu):
    """enc_accel_build sets up the fixed scratch (its module loaded, its
    kernel run once), so the query calls that follow allocate nothing:
    cudaMemGetInfo's free bytes are the same before and after them."""
    import torch
    lib = _lib.load()
    torch.cuda.init()
    torch.cuda.mem_get_info(0)  # the context exists before the first reading
    scale = 1000.0
    tris = np.ascontiguousarray(scenes.random_triangles(5000, seed=1204, scale=scale))
    acc = _build(lib, tris)
    try:
        rays = np.ascontiguousarray(scenes.random_sphere_rays(
            30000, seed=1205, hi=(scale, scale, scale)))
        hits = np.empty(len(rays), HIT_DTYPE)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        for _ in range(2):
            st = lib.enc_intersect_closest_noalloc(acc, rays.ctypes.data, len(rays),
                                                   hits.ctypes.data, None)
            assert st == _lib.ENC_OK, lib.enc_last_error()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, (free0, free1)
        assert (hits["tri"] >= 0).any()
    finally:
        lib.enc_accel_destroy(acc)


def test_noalloc_rejects_batches_above_its_scratch(gpu):
    lib = _lib.load()
    tris = np.ascontiguousarray(scenes.random_triangles(100, seed=1203))
    acc = _build(lib, tris)
    try:
        n = 65537
        rays = np.zeros((n, 8), np.float32)
        hits = np.empty(n, HIT_DTYPE)
        st = lib.enc_intersect_closest_noalloc(acc, rays.ctypes.data, n, hits.ctypes.data, None)
        assert st == _lib.ENC_ERR_INVALID_ARG
        assert b"ENC_NOALLOC_MAX_RAYS" in lib.enc_last_error()
    finally:
        lib.enc_accel_destroy(acc)
