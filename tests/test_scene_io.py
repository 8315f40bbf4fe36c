"""Scene front-end (host code, no GPU): the engine's PLY loader and
scene-file parser against the oracle's restatement on files written here,
and against the reference's own Model::load on the reference's meshes when
the reference tree and its compiled loader are present.

Bar: bit-exact vertex coordinates, the same triangle count and order, the
same primitive and material index per triangle.
"""
import os
from pathlib import Path

import numpy as np
import pytest

from encore_b200 import EncoreError, scene_io
from oracle import bindings as ob
from oracle import scene_port
from tests.scene_files import mesh, write_ply, write_scene

REF_MODELS = ob.REFERENCE_DIR


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


XFORMS = [((0, 0, 0), 1.0, 0.0, (0, 1, 0)), ((0, -30, 0), 60.0, 20.0, (0, 1, 0)),
          ((10, -30, 5), 25.0, -30.0, (0, 1, 0)), ((1, 2, 3), 50.0, 33.0, (0.3, 0.8, 0.1))]


@pytest.mark.parametrize("xf", XFORMS)
def test_ascii_ply_matches_oracle(tmp_path, xf):
    v, f = mesh(11)
    p = tmp_path / "m.ply"
    write_ply(p, v, f, extra_vertex_props=True)
    got = scene_io.load_ply(p, *xf)
    want = scene_port.load_model(p, *xf)
    assert got.shape == (len(f), 9)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian"])
def test_binary_ply_reads_like_ascii(tmp_path, fmt):
    v, f = mesh(12)
    write_ply(tmp_path / "a.ply", v, f)
    write_ply(tmp_path / "b.ply", v, f, fmt=fmt, extra_vertex_props=True)
    xf = XFORMS[3]
    assert np.array_equal(bits(scene_io.load_ply(tmp_path / "a.ply", *xf)),
                          bits(scene_io.load_ply(tmp_path / "b.ply", *xf)))


def test_ply_line_endings_and_polygon_faces(tmp_path):
    v, f = mesh(13)
    write_ply(tmp_path / "a.ply", v, f)
    write_ply(tmp_path / "b.ply", v, f, crlf=True, quads=True, trailing_newline=False)
    a = scene_io.load_ply(tmp_path / "a.ply")
    b = scene_io.load_ply(tmp_path / "b.ply")  # a polygon contributes its first three indices
    assert np.array_equal(bits(a), bits(b))
    assert np.array_equal(bits(b), bits(scene_port.load_model(tmp_path / "b.ply", *XFORMS[0])))


def test_ply_errors(tmp_path):
    v, f = mesh(14)
    bad = f.copy()
    bad[5, 1] = len(v)  # out of range
    write_ply(tmp_path / "idx.ply", v, bad)
    (tmp_path / "not.ply").write_text("hello\n")
    write_ply(tmp_path / "short.ply", v, f)
    data = (tmp_path / "short.ply").read_bytes()
    (tmp_path / "short.ply").write_bytes(data[: len(data) // 2])
    for name in ("idx.ply", "not.ply", "short.ply", "missing.ply"):
        with pytest.raises(EncoreError) as ei:
            scene_io.load_ply(tmp_path / name)
        assert ei.value.status == 1, name


def test_scene_file_matches_oracle(tmp_path):
    p = write_scene(tmp_path)
    got = scene_io.load_scene(p, model_dir=tmp_path)
    want = scene_port.load_scene(p, model_dir=str(tmp_path))
    assert np.array_equal(bits(got.tris), bits(want["tris"]))
    assert np.array_equal(got.prim_of_tri, want["prim_of_tri"])
    assert np.array_equal(got.material_of_tri, want["material_of_tri"])
    assert np.array_equal(got.materials, want["materials"])
    assert got.desc["nprims"] == want["nprims"] == 2 + 2 + 1 + 1 + 400
    assert got.desc["nspheres"] == 1 and got.desc["nunknown"] == 1
    assert got.desc["has_camera"] == 1
    assert np.allclose(got.desc["cam_eye"], want["camera"][:3])
    assert [L["kind"] for L in got.lights] == [L["kind"] for L in want["lights"]] == ["point", "rect"]
    for g, w in zip(got.lights, want["lights"]):
        assert np.allclose(g["center"], w["center"]) and np.allclose(g["color"], w["color"])
    # the rect light's two triangles are one primitive, listed first
    assert got.prim_of_tri[0] == got.prim_of_tri[1] == 0


def test_scene_file_relative_to_working_directory(tmp_path):
    p = write_scene(tmp_path)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        got = scene_io.load_scene(p.name)
    finally:
        os.chdir(cwd)
    assert got.tris.shape[0] == 2 + 2 + 2 + 400


def test_scene_file_errors(tmp_path):
    (tmp_path / "a.txt").write_text("MATERIAL 1 2 three 4 5 6 7 8 9 10 11 12 13\n")
    (tmp_path / "b.txt").write_text("MODEL missing.ply 0 0 0 1 0 0 1 0\n")
    (tmp_path / "c.txt").write_text("CAMERA 0 0 170\n")
    (tmp_path / "d.txt").write_text("MODEL mesh.obj 0 0 0 1 0 0 1 0\n")
    for name in ("a.txt", "b.txt", "c.txt", "d.txt", "none.txt"):
        with pytest.raises(EncoreError) as ei:
            scene_io.load_scene(tmp_path / name, model_dir=tmp_path)
        assert ei.value.status == 1, name


# ---- the reference's own meshes and scenes (only where the reference tree
# ---- and oracle/_ref/libencore_ref.so are present) --------------------------

needs_ref = pytest.mark.skipif(not (REF_MODELS / "models").is_dir() or ob.reference() is None,
                               reason="reference tree or its compiled loader absent")

REF_MESHES = ["cornell_floor.ply", "box.ply", "tallbox.ply", "bunny4.ply", "bunny3.ply",
              "dragon4.ply"]


@needs_ref
@pytest.mark.parametrize("name", REF_MESHES)
def test_ply_matches_reference_model_load(name):
    path = REF_MODELS / "models" / "bwl" / name
    for xf in XFORMS:
        want = ob.ref_model_load(path, *xf)
        got = scene_io.load_ply(path, *xf)
        assert np.array_equal(bits(got), bits(want)), (name, xf)
        # and the oracle's restatement agrees with the reference
        assert np.array_equal(bits(scene_port.load_model(path, *xf)), bits(want)), (name, xf)


def _ref_scenes():
    d = REF_MODELS / "environment" / "scenes"
    if not d.is_dir():
        return []
    out = []
    for p in sorted(d.glob("*.txt")):
        models = [w for line in p.read_text(errors="replace").splitlines()
                  for w in line.split()[1:2] if line.startswith("MODEL")]
        if all((REF_MODELS / m).exists() for m in models):
            out.append(p.name)
    return out


@needs_ref
@pytest.mark.parametrize("name", _ref_scenes()[:6])
def test_reference_scene_files(name):
    """The reference's scene files, each MODEL checked against the
    reference's own Model::load."""
    p = REF_MODELS / "environment" / "scenes" / name
    got = scene_io.load_scene(p, model_dir=REF_MODELS)
    want = scene_port.load_scene(p, model_dir=str(REF_MODELS), model_loader=ob.ref_model_load)
    assert np.array_equal(bits(got.tris), bits(want["tris"]))
    assert np.array_equal(got.prim_of_tri, want["prim_of_tri"])
    assert np.array_equal(got.material_of_tri, want["material_of_tri"])
