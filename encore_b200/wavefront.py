"""Device-side ray and photon generation (wavefront stages around the
traversal kernels): eye rays, hit surfaces, diffuse secondaries, photon
tracing.  All buffers are CUDA tensors; calls are asynchronous on `stream`
except photon tracing, which returns the stored count."""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check, ptr
from .accel import Accelerator, _stream_ptr
from .photon_map import PhotonMap


def camera_rays(eye, look, up, fov_deg: float, width: int, height: int, d_rays,
                jitter_seed: int = 0, stream=None) -> None:
    """width*height eye rays into d_rays (float32, (width*height, 8))."""
    cam = _lib.Camera((C.c_float * 3)(*eye), (C.c_float * 3)(*look), (C.c_float * 3)(*up),
                      fov_deg, width, height, jitter_seed)
    check(_lib.load().enc_camera_rays_device(C.byref(cam), ptr(d_rays), _stream_ptr(stream)),
          "enc_camera_rays_device")


def hit_surface(acc: Accelerator, d_hits, n: int, d_pos, d_nrm, stream=None) -> None:
    check(_lib.load().enc_hit_surface_device(acc.handle, ptr(d_hits), n, ptr(d_pos), ptr(d_nrm),
                                             _stream_ptr(stream)), "enc_hit_surface_device")


def diffuse_rays(acc: Accelerator, d_rays, d_hits, n: int, per_hit: int, seed: int, offset: float,
                 d_out, stream=None) -> None:
    check(_lib.load().enc_diffuse_rays_device(acc.handle, ptr(d_rays), ptr(d_hits), n, per_hit,
                                              seed, offset, ptr(d_out), _stream_ptr(stream)),
          "enc_diffuse_rays_device")


def trace_photons(acc: Accelerator, light_center, light_size: float, nphotons: int,
                  d_pos, d_nrm, d_pow, max_bounces: int = 3, albedo: float = 0.7, seed: int = 1,
                  emit_offset: float = 0.01, bounce_offset: float = 0.001, stream=None) -> int:
    """Emits and traces photons; returns how many were stored (<= capacity =
    rows of d_pos)."""
    o = _lib.PhotonOpts((C.c_float * 3)(*light_center), light_size, nphotons, max_bounces, albedo,
                        seed, emit_offset, bounce_offset)
    stored = C.c_uint32()
    check(_lib.load().enc_photons_trace_device(acc.handle, C.byref(o), ptr(d_pos), ptr(d_nrm),
                                               ptr(d_pow), int(d_pos.shape[0]), C.byref(stored),
                                               _stream_ptr(stream)), "enc_photons_trace_device")
    return stored.value


def trace_photon_maps(acc: Accelerator, light_center, light_size: float, nphotons: int,
                      direct, indirect, max_bounces: int = 3, albedo: float = 0.7, seed: int = 1,
                      emit_offset: float = 0.01, bounce_offset: float = 0.001,
                      shadow_offset: float = 0.0, fill_indirect: bool = False,
                      stream=None) -> tuple[int, int, int]:
    """The reference's direct / indirect map split (enc_photons_trace_maps_device).
    `direct` and `indirect` are (pos, nrm, pow, tag) tuples of CUDA tensors
    ((cap, 3) float32 x 3 and (cap,) int32, or None for no tags).  Returns
    (stored direct, stored indirect, paths emitted)."""
    def store(t):
        pos, nrm, pw, tag = t
        return _lib.PhotonStore(ptr(pos), ptr(nrm), ptr(pw), ptr(tag), int(pos.shape[0]))
    o = _lib.PhotonOpts((C.c_float * 3)(*light_center), light_size, nphotons, max_bounces, albedo,
                        seed, emit_offset, bounce_offset)
    sd, si = store(direct), store(indirect)
    stored = (C.c_uint32 * 2)()
    emitted = C.c_uint32()
    check(_lib.load().enc_photons_trace_maps_device(
        acc.handle, C.byref(o), shadow_offset, int(fill_indirect), C.byref(sd), C.byref(si),
        stored, C.byref(emitted), _stream_ptr(stream)), "enc_photons_trace_maps_device")
    return stored[0], stored[1], emitted.value


def photon_map_from_device(d_pos, d_nrm, d_pow, n: int, caustic: bool = False,
                           device: int = 0) -> PhotonMap:
    pm = PhotonMap(n, caustic=caustic, device=device)
    h = C.c_void_p()
    check(_lib.load().enc_photonmap_create_device(ptr(d_pos), ptr(d_nrm), ptr(d_pow), n,
                                                  int(caustic), device, C.byref(h)),
          "enc_photonmap_create_device")
    pm.handle = h
    pm._count = n
    return pm
