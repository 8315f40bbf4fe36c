"""The C-ABI library loads and exports every symbol include/encore_b200.h
declares (no compute calls: these run without a GPU)."""
import re
from pathlib import Path

from encore_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "encore_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:enc_status|int32_t|double|const char\*)\s+(enc_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "enc_accel_build" in syms and "enc_intersect_closest" in syms
    assert "enc_photonmap_radiance" in syms


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_abi_version():
    assert _lib.load().enc_abi_version() == 1


def test_errors_without_device_are_reported_not_raised():
    import ctypes as C
    lib = _lib.load()
    s = C.c_void_p()
    assert lib.enc_scene_create(None, 0, C.byref(s)) == _lib.ENC_OK
    a = C.c_void_p()
    # empty scene is rejected before any device call
    assert lib.enc_accel_build(s, None, 0, C.byref(a)) == _lib.ENC_ERR_INVALID_ARG
    assert b"no triangles" in lib.enc_last_error()
    lib.enc_scene_destroy(s)
    assert lib.enc_accel_build(None, None, 0, C.byref(a)) == _lib.ENC_ERR_INVALID_ARG
    # the host-buffer queries check their arguments before any device call
    rays = (C.c_float * 6)()
    hits = (C.c_int32 * 4)()
    for fn in (lib.enc_intersect_closest, lib.enc_intersect_closest_od):
        assert fn(None, rays, 1, hits, None, None) == _lib.ENC_ERR_INVALID_ARG
        assert b"null argument" in lib.enc_last_error()


def test_deserialize_rejects_malformed_images_before_any_device_call():
    """enc_accel_deserialize checks the header and every section size first:
    garbage, a foreign magic and a truncated image are ENC_ERR_INVALID_ARG
    with no device involved."""
    import ctypes as C
    import numpy as np
    lib = _lib.load()
    out = C.c_void_p()
    junk = np.zeros(128, np.uint8)
    assert lib.enc_accel_deserialize(junk.ctypes.data, junk.size, 0, C.byref(out)) == _lib.ENC_ERR_INVALID_ARG
    assert b"not a serialised accelerator" in lib.enc_last_error()
    short = np.frombuffer(b"ENCACC01", np.uint8).copy()
    assert lib.enc_accel_deserialize(short.ctypes.data, short.size, 0, C.byref(out)) == _lib.ENC_ERR_INVALID_ARG
    # a well-formed header whose sections are missing
    hdr = np.zeros(120, np.uint8)  # sizeof the header
    hdr[:8] = np.frombuffer(b"ENCACC01", np.uint8)
    hdr[8:12] = np.array([1], np.uint32).view(np.uint8)
    assert lib.enc_accel_deserialize(hdr.ctypes.data, hdr.size, 0, C.byref(out)) == _lib.ENC_ERR_INVALID_ARG
    assert not out.value


def test_photonmap_deserialize_rejects_malformed_images():
    import ctypes as C
    import numpy as np
    lib = _lib.load()
    out = C.c_void_p()
    junk = np.zeros(256, np.uint8)
    assert lib.enc_photonmap_deserialize(junk.ctypes.data, junk.size, 0, C.byref(out)) == _lib.ENC_ERR_INVALID_ARG
    assert b"not a serialised photon map" in lib.enc_last_error()
    assert lib.enc_photonmap_deserialize(junk.ctypes.data, 8, 0, C.byref(out)) == _lib.ENC_ERR_INVALID_ARG
    assert not out.value


def test_ray_payload_shapes_are_checked_before_any_call():
    """intersect takes (N, 8) rays and intersect_od (N, 6): the wrong width is
    a ValueError raised on the host, before the library is called."""
    import numpy as np
    import pytest
    from encore_b200 import Accelerator
    acc = Accelerator.__new__(Accelerator)
    acc.lib = _lib.load()
    acc.handle = None
    with pytest.raises(ValueError, match="6"):
        acc.intersect_od(np.zeros((4, 8), np.float32))
    with pytest.raises(ValueError, match="8"):
        acc.intersect(np.zeros((4, 6), np.float32))
