"""Scene front-end: the reference's PLY model loader and scene-file parser.

``load_ply`` stands where ``Model(filename, center, size, angle, axis, ...)``
stands (ENCORE/src/scene/Model.cpp:34-107: loadPLY, then centerModel) and
``load_scene`` where ``Scene::load`` stands (ENCORE/src/scene/Scene.cpp:78-209).
Both run in the engine library (host code); the triangles they return are in
the reference's primitive-list order, ready for ``Accelerator.build``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from os import PathLike, fspath

import numpy as np

from . import _lib
from ._lib import check


def _xform(center, size, angle, axis) -> _lib.ModelXform:
    return _lib.ModelXform((C.c_float * 3)(*center), size, angle, (C.c_float * 3)(*axis))


def _tris_of(lib, h) -> np.ndarray:
    n = C.c_uint32()
    check(lib.enc_scene_tris(h, None, 0, C.byref(n)), "enc_scene_tris")
    out = np.empty((n.value, 9), np.float32)
    check(lib.enc_scene_tris(h, out.ctypes.data, n.value, None), "enc_scene_tris")
    return out


def load_ply(path: str | PathLike, center=(0.0, 0.0, 0.0), size: float = 1.0, angle: float = 0.0,
             axis=(0.0, 1.0, 0.0)) -> np.ndarray:
    """A PLY mesh scaled to ``size`` on its longest side, centred on
    ``center`` and rotated ``angle`` degrees about ``axis``; (N, 9) float32."""
    lib = _lib.load()
    h = C.c_void_p()
    xf = _xform(center, size, angle, axis)
    check(lib.enc_scene_load_ply(fspath(path).encode(), C.byref(xf), C.byref(h)),
          "enc_scene_load_ply")
    try:
        return _tris_of(lib, h)
    finally:
        lib.enc_scene_destroy(h)


@dataclass
class SceneFile:
    tris: np.ndarray                 # (N, 9) float32, primitive-list order
    prim_of_tri: np.ndarray          # (N,) int32: the reference's primitive index
    material_of_tri: np.ndarray      # (N,) int32: index into materials, -1 = default
    materials: np.ndarray            # (M, 13) float32: MATERIAL's values in file order
    lights: list = field(default_factory=list)  # dicts: kind, center, size, color
    desc: dict = field(default_factory=dict)    # counts, camera, background


def load_scene(path: str | PathLike, model_dir: str | PathLike | None = None) -> SceneFile:
    """Parses a scene file; relative MODEL paths resolve against
    ``model_dir`` (None = the working directory, as the reference does)."""
    lib = _lib.load()
    h = C.c_void_p()
    md = fspath(model_dir).encode() if model_dir is not None else None
    check(lib.enc_scene_load_file(fspath(path).encode(), md, C.byref(h)), "enc_scene_load_file")
    try:
        tris = _tris_of(lib, h)
        n = tris.shape[0]
        prim = np.empty(n, np.int32)
        mat = np.empty(n, np.int32)
        check(lib.enc_scene_prims(h, prim.ctypes.data, mat.ctypes.data, n), "enc_scene_prims")
        nm = C.c_uint32()
        check(lib.enc_scene_materials(h, None, 0, C.byref(nm)), "enc_scene_materials")
        mats = np.empty((nm.value, 13), np.float32)
        check(lib.enc_scene_materials(h, mats.ctypes.data, nm.value, None), "enc_scene_materials")
        nl = C.c_uint32()
        check(lib.enc_scene_lights(h, None, 0, C.byref(nl)), "enc_scene_lights")
        arr = (_lib.SceneLight * max(1, nl.value))()
        check(lib.enc_scene_lights(h, arr, nl.value, None), "enc_scene_lights")
        lights = [{"kind": "rect" if L.kind == _lib.ENC_LIGHT_RECT else "point",
                   "center": tuple(L.center), "size": L.size, "color": tuple(L.color)}
                  for L in arr[:nl.value]]
        d = _lib.SceneDesc()
        check(lib.enc_scene_desc_get(h, C.byref(d)), "enc_scene_desc_get")
        desc = {f: (tuple(getattr(d, f)) if f.startswith(("cam_eye", "cam_look", "cam_up", "background"))
                    else getattr(d, f)) for f, _ in d._fields_}
        return SceneFile(tris, prim, mat, mats, lights, desc)
    finally:
        lib.enc_scene_destroy(h)
