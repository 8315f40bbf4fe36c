"""Multi-scene batched launch: many scenes' ray batches in one persistent
kernel launch, optionally replayed from a CUDA graph (enc_batch_* in the C
ABI).  The reference traces one ray per call and has no counterpart."""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from . import _lib
from ._lib import check, ptr
from .accel import Accelerator, LaunchConfig, _stream_ptr


class BatchLaunch:
    """items: (accelerator, device rays (N, 8) f32, device hits (N, 4) i32)."""

    def __init__(self, items: Sequence[tuple], launch: LaunchConfig | None = None):
        self.lib = _lib.load()
        arr = (_lib.BatchItem * len(items))()
        self._keep = []
        for i, (acc, d_rays, d_hits) in enumerate(items):
            if not isinstance(acc, Accelerator):
                raise TypeError("items[i][0] must be an Accelerator")
            n = int(d_rays.shape[0])
            arr[i] = _lib.BatchItem(acc.handle, ptr(d_rays), ptr(d_hits), n, 0)
            self._keep.append((acc, d_rays, d_hits))
        self.nrays = sum(int(t[1].shape[0]) for t in items)
        lo = (launch or LaunchConfig()).c()
        h = C.c_void_p()
        check(self.lib.enc_batch_create(arr, len(items), C.byref(lo), C.byref(h)),
              "enc_batch_create")
        self.handle = h

    def launch(self, stream=None) -> None:
        check(self.lib.enc_batch_launch(self.handle, _stream_ptr(stream)), "enc_batch_launch")

    def launch_graph(self, stream=None) -> None:
        check(self.lib.enc_batch_launch_graph(self.handle, _stream_ptr(stream)),
              "enc_batch_launch_graph")

    def check(self, stream=None) -> None:
        check(self.lib.enc_batch_check(self.handle, _stream_ptr(stream)), "enc_batch_check")

    def destroy(self) -> None:
        if self.handle:
            self.lib.enc_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
