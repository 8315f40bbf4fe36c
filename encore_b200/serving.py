"""Serving: resident scenes, continuous batching of ray-batch requests
(enc_server_* in the C ABI).  The reference has no counterpart; it answers one
ray per call from one thread."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr
from .accel import HIT_DTYPE, Accelerator, LaunchConfig

CLOSEST = 0
ANY = 1


class Server:
    def __init__(self, device: int = 0, slots: int = 6, slot_rays: int = 4 << 20,
                 budget_bytes: int = 120 * 10**9, launch: LaunchConfig | None = None):
        self.lib = _lib.load()
        o = _lib.ServerOpts(device, slots, slot_rays, budget_bytes, (launch or LaunchConfig()).c())
        h = C.c_void_p()
        check(self.lib.enc_server_create(C.byref(o), C.byref(h)), "enc_server_create")
        self.handle = h
        self._live: dict[int, tuple] = {}  # keeps request buffers alive until waited
        self._scenes: list[Accelerator] = []

    def add_scene(self, acc: Accelerator) -> int:
        sid = C.c_uint32()
        check(self.lib.enc_server_add_scene(self.handle, acc.handle, C.byref(sid)),
              "enc_server_add_scene")
        self._scenes.append(acc)
        return sid.value

    def submit(self, scene: int, rays: np.ndarray, kind: int = CLOSEST,
               out: np.ndarray | None = None) -> int:
        """Queues a request; returns its id.  rays/out should be pinned host
        memory (e.g. numpy views of pinned torch tensors) for overlap."""
        n = rays.shape[0]
        if out is None:
            out = np.empty(n, HIT_DTYPE) if kind == CLOSEST else np.empty(n, np.uint8)
        rid = C.c_uint64()
        check(self.lib.enc_server_submit(self.handle, scene, kind, ptr(rays), n, ptr(out),
                                         C.byref(rid)), "enc_server_submit")
        self._live[rid.value] = (rays, out)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0):
        """Blocks until the request is done; returns (result array, info dict)."""
        info = _lib.RequestInfo()
        st = self.lib.enc_server_wait(self.handle, rid, timeout, C.byref(info))
        if st == _lib.ENC_ERR_NOT_READY:
            return None, None
        rays, out = self._live.pop(rid)
        d = {f: getattr(info, f) for f, _ in info._fields_}
        if st != _lib.ENC_OK:
            raise _lib.EncoreError(st, "enc_server_wait", f"request {rid} failed")
        return out, d

    def cancel(self, rid: int) -> bool:
        return self.lib.enc_server_cancel(self.handle, rid) == _lib.ENC_OK

    def now(self) -> float:
        return self.lib.enc_server_now()

    def destroy(self) -> None:
        if self.handle:
            self.lib.enc_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
