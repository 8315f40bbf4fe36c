"""PLY meshes and scene files written by the tests (the engine's scene
front-end reads them; the oracle's restatement checks it)."""
import struct
from pathlib import Path

import numpy as np


def mesh(seed, nv=60, nf=100):
    """Vertices on a 1/1024 grid (exact in decimal, so ascii and binary files
    hold the same floats) and random faces."""
    rng = np.random.default_rng(seed)
    v = (rng.integers(-40000, 40000, (nv, 3)) / 1024.0).astype(np.float32)
    f = rng.integers(0, nv, (nf, 3))
    return v, f


def write_ply(path, v, f, fmt="ascii", extra_vertex_props=False, quads=False, crlf=False,
              trailing_newline=True):
    nl = "\r\n" if crlf else "\n"
    props = ["property float x", "property float y", "property float z"]
    if extra_vertex_props:
        props += ["property float confidence", "property float intensity"]
    head = ["ply", f"format {fmt} 1.0", "comment written by the tests",
            f"element vertex {len(v)}", *props, f"element face {len(f)}",
            "property list uchar int vertex_indices", "end_header"]
    data = nl.join(head) + nl
    if fmt == "ascii":
        lines = []
        for p in v:
            s = " ".join(f"{float(x):.10f}" for x in p)
            lines.append(s + (" 0.5 1.0 " if extra_vertex_props else " "))
        for k, tri in enumerate(f):
            idx = list(tri) + ([int(tri[0])] if quads else [])
            lines.append(f"{len(idx)} " + " ".join(str(int(i)) for i in idx))
        data += nl.join(lines) + (nl if trailing_newline else "")
        Path(path).write_bytes(data.encode())
        return
    end = "<" if fmt == "binary_little_endian" else ">"
    out = bytearray(data.encode())
    for p in v:
        out += struct.pack(end + "3f", *map(float, p))
        if extra_vertex_props:
            out += struct.pack(end + "2f", 0.5, 1.0)
    for tri in f:
        idx = list(tri) + ([int(tri[0])] if quads else [])
        out += struct.pack(end + "B", len(idx)) + struct.pack(end + f"{len(idx)}i", *map(int, idx))
    Path(path).write_bytes(bytes(out))


def write_scene(tmp_path):
    rng = np.random.default_rng(21)
    models = tmp_path / "models"
    models.mkdir()
    quad = np.array([[0, 0, 0], [0, 0, 1], [1, 0, 1], [1, 0, 0]], np.float32)
    write_ply(models / "wall.ply", quad, np.array([[0, 1, 2], [2, 3, 0]]))
    v, f = mesh(22, nv=200, nf=400)
    write_ply(models / "blob.ply", v, f, extra_vertex_props=True)
    text = f"""*a scene written by the tests*
CAMERA 0 0 170 0 0 0 0 1 0 45 1 0.1 1000
MATERIAL 0.9 0.9 0.9 0 0 0 0 0 0 0 0 0 0
RECT_LIGHT 1.0 1.0 1.0
MATERIAL 0.7 0.7 0.7 0 0 0 0.1 0.1 0.1 0 0 0 0
* floor *
MODEL models/wall.ply 0 -50 0 100 0 0 1 0
MODEL models/wall.ply 0 50 0 100 0 0 1 0   *ceiling
POINT_LIGHT 1 2 3 0.5 0.5 0.5
SPHERE 20 -29.9 20 20 1 0 0 1 0
*MODEL models/blob.ply 0 0 0 10 0 0 1 0
BACKGROUND_COLOR 0 0 0 1
MATERIAL 0.36 0.36 0.6 0 0 0 0.05 0.05 0.05 0 0 0 0
MODEL models/blob.ply 5 -20 {rng.integers(1, 9)} 40 25 0 1 0
NOT_A_COMMAND
"""
    p = tmp_path / "scene.txt"
    p.write_text(text)
    return p
