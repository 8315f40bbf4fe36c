"""Host API mirroring the reference's accelerator interface.

``Accelerator`` stands where ``AccelerationStructure`` stands in the reference
(ENCORE/src/accelerators/AccelerationStructure.h:33-67): ``build`` takes the
scene's triangles in primitive-list order (the triangle index is the ID the
reference recovers from HitInfo::hitObject, Model.cpp:255-264) and
``intersect`` answers closest-hit queries.  Because one ray per call is the
wrong granularity for a GPU, ``intersect`` takes a batch; a batch of one is
the reference's call.  ``occluded`` is the shadow test of
PhotonMapperCPU::IsInShadow (PhotonMapperCPU.cpp:1192-1207).

Rays are (N, 8) float32 rows (ox, oy, oz, tmin, dx, dy, dz, tmax) in host
memory (numpy, or pinned torch tensors) or device memory (torch CUDA tensors
for the ``*_device`` forms).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, ptr

HIT_DTYPE = np.dtype([("tri", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])

KIND = {"wbvh": _lib.ENC_ACCEL_WBVH, "kdtree": _lib.ENC_ACCEL_KDTREE}
PRED = {"reference": _lib.ENC_PRED_REFERENCE, "noclamp": _lib.ENC_PRED_NOCLAMP}


@dataclass
class BinConfig:
    """Ray binning ahead of the closest-hit launch (enc_bin_opts): key bits of
    the origin cell and of the direction cell (both 0 = the tuned default),
    and the probe distance as a fraction of the scene diagonal (0 = bin the
    origin itself)."""
    origin_bits: int = 0
    dir_bits: int = 0
    probe_frac: float = 0.0

    def c(self) -> _lib.BinOpts:
        return _lib.BinOpts(self.origin_bits, self.dir_bits, self.probe_frac)


@dataclass
class LaunchConfig:
    block_threads: int = 0
    blocks_per_sm: int = 0
    chunk: int = 0
    stack_depth: int = 0

    def c(self) -> _lib.LaunchOpts:
        return _lib.LaunchOpts(self.block_threads, self.blocks_per_sm, self.chunk, self.stack_depth)


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _as_rays(rays: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(rays, dtype=np.float32)
    if r.ndim != 2 or r.shape[1] != 8:
        raise ValueError("rays must be (N, 8) float32: ox oy oz tmin dx dy dz tmax")
    return r


def rays_from_origin_dir(o: np.ndarray, d: np.ndarray, tmin: float = 0.0,
                         tmax: float = np.inf) -> np.ndarray:
    """Packs reference-style rays (origin, direction; t > 0) into (N, 8)."""
    n = o.shape[0]
    r = np.empty((n, 8), dtype=np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


class Accelerator:
    """Device-resident accelerator over one triangle scene."""

    def __init__(self, kind: str = "wbvh", width: int = 8, max_leaf_tris: int = 3,
                 predicate: str = "reference", device: int = 0):
        self.lib = _lib.load()
        self.opts = _lib.BuildOpts(KIND[kind], width, max_leaf_tris, PRED[predicate])
        self.device = device
        self.kind = kind
        self.handle = None
        self.ntris = 0

    # AccelerationStructure::build (AccelerationStructure.h:47)
    def build(self, tris: np.ndarray) -> "Accelerator":
        t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        self.destroy()
        scene = C.c_void_p()
        check(self.lib.enc_scene_create(ptr(t), t.shape[0], C.byref(scene)), "enc_scene_create")
        try:
            h = C.c_void_p()
            check(self.lib.enc_accel_build(scene, C.byref(self.opts), self.device, C.byref(h)),
                  "enc_accel_build")
        finally:
            self.lib.enc_scene_destroy(scene)
        self.handle = h
        self.ntris = t.shape[0]
        return self

    # AccelerationStructure::update (AccelerationStructure.h:51)
    def update(self, tris: np.ndarray) -> "Accelerator":
        """The same triangles at new positions: refit (wide BVH) or rebuild (kd)."""
        t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
        check(self.lib.enc_accel_refit(self.handle, ptr(t), t.shape[0]), "enc_accel_refit")
        return self

    def save(self) -> bytes:
        """The accelerator as a byte image (enc_accel_serialize)."""
        size = C.c_size_t()
        check(self.lib.enc_accel_serialize(self.handle, None, 0, C.byref(size)),
              "enc_accel_serialize")
        buf = np.empty(size.value, np.uint8)
        check(self.lib.enc_accel_serialize(self.handle, ptr(buf), size.value, C.byref(size)),
              "enc_accel_serialize")
        return buf.tobytes()

    @classmethod
    def load(cls, image: bytes, device: int = 0) -> "Accelerator":
        """An accelerator from a byte image saved by save(), uploaded to
        `device` without a host build (enc_accel_deserialize)."""
        acc = cls.__new__(cls)
        acc.lib = _lib.load()
        acc.device = device
        acc.handle = None
        buf = np.frombuffer(image, dtype=np.uint8)
        h = C.c_void_p()
        check(acc.lib.enc_accel_deserialize(ptr(buf), buf.size, device, C.byref(h)),
              "enc_accel_deserialize")
        acc.handle = h
        info = acc.info()
        acc.kind = "wbvh" if info["kind"] == _lib.ENC_ACCEL_WBVH else "kdtree"
        acc.ntris = info["ntris"]
        acc.opts = _lib.BuildOpts(info["kind"], info["width"], 0, info["predicate"])
        return acc

    def info(self) -> dict:
        i = _lib.AccelInfo()
        check(self.lib.enc_accel_info_get(self.handle, C.byref(i)), "enc_accel_info_get")
        return {f: (list(getattr(i, f)) if f.startswith("scene_") else getattr(i, f))
                for f, _ in i._fields_}

    # AccelerationStructure::intersect (AccelerationStructure.h:63), batched
    def intersect(self, rays: np.ndarray, launch: LaunchConfig | None = None,
                  stream=None, out: np.ndarray | None = None) -> np.ndarray:
        r = _as_rays(rays) if isinstance(rays, np.ndarray) else rays
        n = r.shape[0]
        hits = out if out is not None else np.empty(n, dtype=HIT_DTYPE)
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_closest(self.handle, ptr(r), n, ptr(hits), C.byref(lo),
                                             _stream_ptr(stream)), "enc_intersect_closest")
        return hits

    # AccelerationStructure::intersect on the reference's Ray payload: (N, 6)
    # float32 origin and direction, no distance bounds (a hit needs t > 0)
    def intersect_od(self, rays, launch: LaunchConfig | None = None, stream=None,
                     out: np.ndarray | None = None) -> np.ndarray:
        if isinstance(rays, np.ndarray):
            r = np.ascontiguousarray(rays, dtype=np.float32)
            if r.ndim != 2 or r.shape[1] != 6:
                raise ValueError("rays must be (N, 6) float32: ox oy oz dx dy dz")
        else:
            r = rays
        n = r.shape[0]
        hits = out if out is not None else np.empty(n, dtype=HIT_DTYPE)
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_closest_od(self.handle, ptr(r), n, ptr(hits), C.byref(lo),
                                                _stream_ptr(stream)), "enc_intersect_closest_od")
        return hits

    def occluded(self, rays: np.ndarray, launch: LaunchConfig | None = None, stream=None,
                 out: np.ndarray | None = None) -> np.ndarray:
        r = _as_rays(rays) if isinstance(rays, np.ndarray) else rays
        n = r.shape[0]
        occ = out if out is not None else np.empty(n, dtype=np.uint8)
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_any(self.handle, ptr(r), n, ptr(occ), C.byref(lo),
                                         _stream_ptr(stream)), "enc_intersect_any")
        return occ

    # device-buffer forms (torch CUDA tensors or raw pointers); asynchronous
    def intersect_device(self, d_rays, n: int, d_hits, launch: LaunchConfig | None = None,
                         stream=None) -> None:
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_closest_device(self.handle, ptr(d_rays), n, ptr(d_hits),
                                                    C.byref(lo), _stream_ptr(stream)),
              "enc_intersect_closest_device")

    def bin_scratch_bytes(self, n: int, binning: BinConfig | None = None) -> int:
        out = C.c_size_t()
        b = (binning or BinConfig()).c()
        check(self.lib.enc_bin_scratch_bytes(n, C.byref(b), C.byref(out)),
              "enc_bin_scratch_bytes")
        return out.value

    def intersect_device_binned(self, d_rays, n: int, d_hits, d_scratch,
                                binning: BinConfig | None = None,
                                launch: LaunchConfig | None = None, stream=None) -> None:
        """Closest hit with the batch binned first (identical hits); d_scratch
        is a device buffer of at least bin_scratch_bytes(n) bytes (a torch
        uint8 CUDA tensor, whose storage the caching allocator aligns to 512
        bytes)."""
        lo = (launch or LaunchConfig()).c()
        b = (binning or BinConfig()).c()
        nbytes = d_scratch.numel() * d_scratch.element_size() if hasattr(d_scratch, "numel") \
            else int(getattr(d_scratch, "nbytes", 0))
        check(self.lib.enc_intersect_closest_device_binned(
            self.handle, ptr(d_rays), n, ptr(d_hits), ptr(d_scratch), nbytes, C.byref(b),
            C.byref(lo), _stream_ptr(stream)), "enc_intersect_closest_device_binned")

    def bin_rays(self, d_rays, n: int, d_scratch, binning: BinConfig | None = None,
                 stream=None) -> int:
        """Enqueues the binning pass alone; returns the device address of the
        permutation (inside d_scratch) for intersect_device_ordered."""
        b = (binning or BinConfig()).c()
        nbytes = d_scratch.numel() * d_scratch.element_size()
        order = C.c_void_p()
        check(self.lib.enc_bin_rays(self.handle, ptr(d_rays), n, ptr(d_scratch), nbytes,
                                    C.byref(b), C.byref(order), _stream_ptr(stream)),
              "enc_bin_rays")
        return order.value or 0

    def intersect_device_ordered(self, d_rays, n: int, d_order, d_hits,
                                 launch: LaunchConfig | None = None, stream=None) -> None:
        """Closest hit taking ray d_order[q] as the q-th ray of the queue."""
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_closest_device_ordered(
            self.handle, ptr(d_rays), n, ptr(d_order), ptr(d_hits), C.byref(lo),
            _stream_ptr(stream)), "enc_intersect_closest_device_ordered")

    def occluded_device(self, d_rays, n: int, d_occ, launch: LaunchConfig | None = None,
                        stream=None) -> None:
        lo = (launch or LaunchConfig()).c()
        check(self.lib.enc_intersect_any_device(self.handle, ptr(d_rays), n, ptr(d_occ),
                                                C.byref(lo), _stream_ptr(stream)),
              "enc_intersect_any_device")

    def check(self, stream=None) -> None:
        check(self.lib.enc_accel_check(self.handle, _stream_ptr(stream)), "enc_accel_check")

    def count_visits(self, d_rays, n: int, d_visits, stream=None) -> None:
        check(self.lib.enc_accel_count_visits(self.handle, ptr(d_rays), n, ptr(d_visits),
                                              _stream_ptr(stream)), "enc_accel_count_visits")

    def destroy(self) -> None:
        if self.handle:
            self.lib.enc_accel_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
