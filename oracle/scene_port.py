"""CPU restatement of the reference's model and scene-file loaders.

Test infrastructure: imported only by tests/.  It is the checker for the
engine's loader (encore_b200/csrc/scene_io.cpp) on files the tests write
themselves; on the reference's own meshes the tests also check it against
the compiled reference (oracle/_ref, ``bindings.ref_model_load``).

Follows, in float32 with the reference's operation order:
  Model::loadPLY            ENCORE/src/scene/Model.cpp:396-482 (ascii only,
                            line based: the first three numbers of a vertex
                            line, the 2nd-4th numbers of a face line)
  Model::centerModel        ENCORE/src/scene/Model.cpp:109-141
  Model::getCenterMatrix    ENCORE/src/scene/Model.cpp:143-173
  Model::rotate             ENCORE/src/scene/Model.cpp:175-202 (cos/sin of the
                            float angle through the C library's cosf/sinf)
  Scene::load               ENCORE/src/scene/Scene.cpp:184-209
  Scene::HandleSceneVariable ENCORE/src/scene/Scene.cpp:78-183
  RectangleLight            ENCORE/src/scene/RectangleLight.cpp (constructor:
                            the 30 x 30 quad at y = 49.99999, triangles
                            (v0, v1, v2) and (v2, v3, v0))
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

f32 = np.float32
_libm = C.CDLL("libm.so.6")
_libm.cosf.restype = C.c_float
_libm.cosf.argtypes = [C.c_float]
_libm.sinf.restype = C.c_float
_libm.sinf.argtypes = [C.c_float]


def load_ply_ascii(path) -> tuple[np.ndarray, np.ndarray]:
    """(vertices (V, 3) float32, faces (F, 3) int64) as loadPLY reads them."""
    text = open(path, "rb").read().decode("latin-1")
    if not text.startswith("ply"):
        raise ValueError("not a PLY file")
    t = text.find("element") + 7
    t = text.find("vertex", t) + 7
    s = text.find("\n", t)
    nv = int(text[t:s].strip().split()[0])
    t = text.find("element", s) + 7
    t = text.find("face", t) + 5
    s = text.find("\n", t)
    nf = int(text[t:s].strip().split()[0])
    body = text[text.find("\n", text.find("end_header", t)) + 1:].split("\n")
    v = np.empty((nv, 3), np.float32)
    for i in range(nv):
        w = body[i].split()
        v[i] = [f32(float(w[0])), f32(float(w[1])), f32(float(w[2]))]
    f = np.empty((nf, 3), np.int64)
    for i in range(nf):
        w = body[nv + i].split()
        f[i] = [int(w[1]), int(w[2]), int(w[3])]
    return v, f


def rotation(angle: float, u) -> np.ndarray:
    R = np.zeros(16, np.float32)
    R[[0, 5, 10, 15]] = 1
    rad = f32(float(angle) / 180.0 * math.pi)  # in double, as (float)(angle/180.0*M_PI)
    if -0.0000001 <= float(rad) <= 0.0000001:
        return R
    c = f32(_libm.cosf(float(rad)))
    s = f32(_libm.sinf(float(rad)))
    k = f32(1) - c
    ux, uy, uz = (f32(x) for x in u)
    R[0] = c + k * ux * ux
    R[4] = k * uy * ux - s * uz
    R[8] = k * uz * ux + s * uy
    R[1] = k * ux * uy + s * uz
    R[5] = c + k * uy * uy
    R[9] = k * uz * uy - s * ux
    R[2] = k * ux * uz - s * uy
    R[6] = k * uy * uz + s * ux
    R[10] = c + k * uz * uz
    return R


def center_model(v: np.ndarray, center, size: float, angle: float, axis) -> np.ndarray:
    # running bounds start at FLT_MAX / FLT_MIN (POS_INF / NEG_INF, Common.h:28-29)
    lo = np.minimum(v.min(axis=0), np.finfo(np.float32).max)
    hi = np.maximum(v.max(axis=0), np.finfo(np.float32).tiny)
    ln = hi - lo
    longest = ln[0] if ln[0] > max(ln[1], ln[2]) else (ln[1] if ln[1] > ln[2] else ln[2])
    scale = f32(size) / longest
    mid = (hi + lo) * f32(0.5)
    off = mid * scale - np.asarray(center, np.float32)
    m = rotation(angle, axis)
    m[12] = -off[0] * m[0] - off[1] * m[4] - off[2] * m[8]
    m[13] = -off[0] * m[1] - off[1] * m[5] - off[2] * m[9]
    m[14] = -off[0] * m[2] - off[1] * m[6] - off[2] * m[10]
    m[[0, 1, 2, 4, 5, 6, 8, 9, 10]] *= scale
    x, y, z = v[:, 0], v[:, 1], v[:, 2]
    out = np.empty_like(v)
    out[:, 0] = x * m[0] + y * m[4] + z * m[8] + m[12]
    out[:, 1] = x * m[1] + y * m[5] + z * m[9] + m[13]
    out[:, 2] = x * m[2] + y * m[6] + z * m[10] + m[14]
    return out


def load_model(path, center, size, angle, axis) -> np.ndarray:
    v, f = load_ply_ascii(path)
    v = center_model(v, center, size, angle, axis)
    return v[f].reshape(-1, 9)


RECT_LIGHT_TRIS = np.array([[15, 49.99999, 15, -15, 49.99999, 15, -15, 49.99999, -15],
                            [-15, 49.99999, -15, 15, 49.99999, -15, 15, 49.99999, 15]],
                           np.float32)


def load_scene(path, model_dir=None, model_loader=load_model) -> dict:
    """Triangles in primitive-list order, with each triangle's primitive and
    material index, the materials, lights and camera of a scene file."""
    words = []
    for line in open(path, encoding="latin-1"):
        for w in line.split():
            if w.startswith("*"):
                break  # the rest of the line is a comment
            words.append(w)
    tris, prim, mat = [], [], []
    materials, lights = [], []
    nprims = 0
    camera = None
    material = -1
    it = iter(words)

    def nums(k):
        return [f32(float(next(it))) for _ in range(k)]

    for var in it:
        if var == "BACKGROUND_COLOR":
            nums(4)
        elif var == "POINT_LIGHT":
            p = nums(6)
            lights.insert(0, {"kind": "point", "center": tuple(p[:3]), "size": 0.0,
                              "color": tuple(p[3:])})
        elif var == "RECT_LIGHT":
            c = nums(3)
            tris.append(RECT_LIGHT_TRIS)
            prim += [nprims, nprims]
            mat += [material, material]
            nprims += 1
            lights.append({"kind": "rect", "center": (0.0, f32(49.99999), 0.0), "size": 30.0,
                           "color": tuple(c)})
        elif var == "MATERIAL":
            materials.append(nums(13))
            material = len(materials) - 1
        elif var == "SPHERE":
            nums(9)
            nprims += 1
        elif var == "CAMERA":
            camera = nums(13)
        elif var == "MODEL":
            fname = next(it)
            c = nums(3)
            size, angle = nums(2)
            ax = nums(3)
            p = fname if model_dir is None or os.path.isabs(fname) else os.path.join(model_dir, fname)
            t = model_loader(p, c, size, angle, ax)
            tris.append(t)
            prim += list(range(nprims, nprims + len(t)))
            mat += [material] * len(t)
            nprims += len(t)
    return {
        "tris": np.concatenate(tris) if tris else np.zeros((0, 9), np.float32),
        "prim_of_tri": np.asarray(prim, np.int32),
        "material_of_tri": np.asarray(mat, np.int32),
        "materials": np.asarray(materials, np.float32).reshape(-1, 13),
        "lights": lights,
        "camera": camera,
        "nprims": nprims,
    }
