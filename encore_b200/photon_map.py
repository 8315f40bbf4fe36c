"""Host API mirroring the reference's PhotonMap (ENCORE/src/renderers/PhotonMap.h:28-105).

``PhotonMap(n).add_photons(...)`` + ``balance_and_construct()`` stand for
AddPhoton x n and BalanceAndConstruct; ``get_nearest_n_photons`` and
``get_radiance_estimate`` answer GetNearestNPhotons / GetRadianceEstimate for
a batch of query points (a batch of one is the reference's call).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr


def _f32(a, cols=3):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != cols:
        raise ValueError(f"expected (N, {cols}) float32")
    return a


class PhotonMap:
    def __init__(self, max_photon_count: int, caustic: bool = False, device: int = 0):
        self.lib = _lib.load()
        self.max_photons = int(max_photon_count)
        self.caustic = caustic
        self.device = device
        self._pos: list[np.ndarray] = []
        self._nrm: list[np.ndarray] = []
        self._pow: list[np.ndarray] = []
        self._count = 0
        self.handle = None

    # PhotonMap::AddPhoton (PhotonMap.cpp:46-53): photons beyond the capacity are dropped
    def add_photons(self, pos, normal, power) -> int:
        pos, normal, power = _f32(pos), _f32(normal), _f32(power)
        room = self.max_photons - self._count
        take = max(0, min(room, pos.shape[0]))
        if take:
            self._pos.append(pos[:take])
            self._nrm.append(normal[:take])
            self._pow.append(power[:take])
            self._count += take
            self._destroy()
        return take

    def full(self) -> bool:
        return self._count == self.max_photons

    def count(self) -> int:
        return self._count

    # PhotonMap::BalanceAndConstruct (PhotonMap.cpp:167-175)
    def balance_and_construct(self) -> "PhotonMap":
        if self.handle is not None:
            return self
        z = np.zeros((0, 3), np.float32)
        pos = np.concatenate(self._pos) if self._pos else z
        nrm = np.concatenate(self._nrm) if self._nrm else z
        pw = np.concatenate(self._pow) if self._pow else z
        h = C.c_void_p()
        check(self.lib.enc_photonmap_create(ptr(pos), ptr(nrm), ptr(pw), pos.shape[0],
                                            int(self.caustic), self.device, C.byref(h)),
              "enc_photonmap_create")
        self.handle = h
        return self

    def save(self) -> bytes:
        """The balanced map as a byte image (enc_photonmap_serialize)."""
        self.balance_and_construct()
        size = C.c_size_t()
        check(self.lib.enc_photonmap_serialize(self.handle, None, 0, C.byref(size)),
              "enc_photonmap_serialize")
        buf = np.empty(size.value, np.uint8)
        check(self.lib.enc_photonmap_serialize(self.handle, ptr(buf), size.value, C.byref(size)),
              "enc_photonmap_serialize")
        return buf.tobytes()

    @classmethod
    def load(cls, image: bytes, device: int = 0) -> "PhotonMap":
        """A map from a byte image saved by save(), with no host balance."""
        buf = np.frombuffer(image, dtype=np.uint8)
        lib = _lib.load()
        h = C.c_void_p()
        check(lib.enc_photonmap_deserialize(ptr(buf), buf.size, device, C.byref(h)),
              "enc_photonmap_deserialize")
        caustic = bool(int.from_bytes(image[12:16], "little"))
        n = int.from_bytes(image[16:20], "little")
        pm = cls(n, caustic=caustic, device=device)
        pm.handle = h
        pm._count = n
        return pm

    def _flags(self, ignore_normal: bool) -> int:
        return _lib.ENC_GATHER_IGNORE_NORMAL if ignore_normal else 0

    # PhotonMap::GetRadianceEstimate (PhotonMap.cpp:121-164), batched
    def get_radiance_estimate(self, n: int, max_distance: float, location, normal,
                              ignore_normal: bool = False, stream=None) -> np.ndarray:
        self.balance_and_construct()
        q, qn = _f32(location), _f32(normal)
        rgb = np.empty((q.shape[0], 3), np.float32)
        check(self.lib.enc_photonmap_radiance(self.handle, ptr(q), ptr(qn), q.shape[0], n,
                                              max_distance, self._flags(ignore_normal), ptr(rgb),
                                              stream), "enc_photonmap_radiance")
        return rgb

    def get_radiance_estimate_device(self, n: int, max_distance: float, d_q, d_n, nq: int, d_rgb,
                                     ignore_normal: bool = False, stream=None) -> None:
        self.balance_and_construct()
        check(self.lib.enc_photonmap_radiance_device(self.handle, ptr(d_q), ptr(d_n), nq, n,
                                                     max_distance, self._flags(ignore_normal),
                                                     ptr(d_rgb), stream),
              "enc_photonmap_radiance_device")

    def count_visits(self, n: int, max_distance: float, d_q, d_n, nq: int, d_rgb, d_visits,
                     ignore_normal: bool = False, stream=None) -> None:
        """The device radiance estimate with per-query work counters (4 words
        per query: child boxes tested, photons tested, normals read, photons
        found), for the bytes-per-query roofline."""
        self.balance_and_construct()
        check(self.lib.enc_photonmap_count_visits(self.handle, ptr(d_q), ptr(d_n), nq, n,
                                                  max_distance, self._flags(ignore_normal),
                                                  ptr(d_rgb), ptr(d_visits), stream),
              "enc_photonmap_count_visits")

    def check(self, stream=None) -> None:
        """Waits for `stream` and raises if a gather on this map stopped at
        its loop bound (the device form does not read the status itself)."""
        stream = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(self.lib.enc_photonmap_check(self.handle, stream), "enc_photonmap_check")

    # PhotonMap::GetNearestNPhotons (PhotonMap.cpp:76-94), batched; ascending distance
    def get_nearest_n_photons(self, n: int, max_distance: float, location, normal,
                              ignore_normal: bool = False):
        self.balance_and_construct()
        q, qn = _f32(location), _f32(normal)
        nq = q.shape[0]
        idx = np.empty((nq, n), np.int32)
        d2 = np.empty((nq, n), np.float32)
        cnt = np.empty(nq, np.int32)
        check(self.lib.enc_photonmap_nearest(self.handle, ptr(q), ptr(qn), nq, n, max_distance,
                                             self._flags(ignore_normal), ptr(idx), ptr(d2),
                                             ptr(cnt), None), "enc_photonmap_nearest")
        return idx, d2, cnt

    def _destroy(self) -> None:
        if self.handle:
            self.lib.enc_photonmap_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass
