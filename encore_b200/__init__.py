"""encore_b200: a B200-native ray-query engine with the accelerator API of
endy/ENCORE (build over a triangle scene, closest-hit / any-hit intersect of
ray batches, photon-map k-nearest gather).

The compute path is the CUDA library ``libencore_b200.so`` (sources in
``csrc/``, C ABI in ``include/encore_b200.h``); this package is its host-side
binding.  There is no CPU fallback: without the library every call raises.
"""
from .accel import HIT_DTYPE, Accelerator, BinConfig, LaunchConfig, rays_from_origin_dir  # noqa: F401
from .photon_map import PhotonMap  # noqa: F401
from ._lib import EncoreError  # noqa: F401

__all__ = ["Accelerator", "BinConfig", "LaunchConfig", "PhotonMap", "HIT_DTYPE", "EncoreError",
           "rays_from_origin_dir"]
