"""ctypes access to the two oracles.  Test infrastructure: imported only by
tests/, __graft_entry__.smoke() and the CPU arm of bench.py.

* port()      : oracle/_ref/libencore_oracle.so, the C restatement in oracle/*.c
* reference() : oracle/_ref/libencore_ref.so, the reference's own CPU code
                compiled from its sources by oracle/Makefile (None if absent)
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE = Path(__file__).resolve().parent
PORT_SO = ORACLE / "_ref" / "libencore_oracle.so"
REF_SO = ORACLE / "_ref" / "libencore_ref.so"

HIT = np.dtype([("tri", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
P = C.c_void_p

_port = None
_ref = None


def port():
    global _port
    if _port is None:
        if not PORT_SO.exists():
            subprocess.run(["make", "-C", str(ORACLE), "port"], check=True, capture_output=True)
        lib = C.CDLL(str(PORT_SO))
        lib.eo_tri_test.argtypes = [P, P, C.c_int, P, P, P]
        lib.eo_tri_test.restype = C.c_int
        lib.eo_tri_test_batch.argtypes = [P, P, P, C.c_long, C.c_int, P, P, P, P]
        lib.eo_closest_brute.argtypes = [P, C.c_int, P, C.c_long, C.c_int, P, C.c_int]
        lib.eo_occluded_brute.argtypes = [P, C.c_int, P, C.c_long, C.c_int, P, C.c_int]
        lib.eo_closest_f64.argtypes = [P, C.c_int, P, C.c_long, P, C.c_int]
        lib.eo_pairs_f64.argtypes = [P, P, P, C.c_long, P, P]
        lib.eo_kd_build.restype = P
        lib.eo_kd_build.argtypes = [P, C.c_int, P, P, P]
        lib.eo_kd_closest.argtypes = [P, P, C.c_long, C.c_int, P, C.c_int]
        lib.eo_kd_free.argtypes = [P]
        lib.eo_pmap_build.restype = P
        lib.eo_pmap_build.argtypes = [P, P, P, C.c_long]
        lib.eo_pmap_gather.argtypes = [P, P, P, C.c_long, C.c_int, C.c_float, C.c_int, C.c_int,
                                       P, P, P, P, C.c_int]
        lib.eo_pmap_free.argtypes = [P]
        _port = lib
    return _port


def reference():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        lib = C.CDLL(str(REF_SO))
        lib.encref_scene_create.restype = P
        lib.encref_scene_create.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_double)]
        lib.encref_scene_destroy.argtypes = [P]
        lib.encref_closest.argtypes = [P, P, C.c_long, P, P, P, P, C.c_int]
        lib.encref_occluded.argtypes = [P, P, C.c_long, P, C.c_int]
        lib.encref_pmap_create.restype = P
        lib.encref_pmap_create.argtypes = [P, P, P, C.c_long, C.c_int, C.POINTER(C.c_double)]
        lib.encref_pmap_destroy.argtypes = [P]
        lib.encref_set_ignore_normal.argtypes = [C.c_int]
        lib.encref_pmap_radiance.argtypes = [P, P, P, C.c_long, C.c_int, C.c_float, P, C.c_int]
        lib.encref_pmap_nearest.argtypes = [P, P, P, C.c_long, C.c_int, C.c_float, P, P, P, C.c_int]
        lib.encref_hardware_threads.restype = C.c_int
        lib.encref_model_load.restype = C.c_long
        lib.encref_model_load.argtypes = [C.c_char_p, P, C.c_float, C.c_float, P, P, C.c_long]
        _ref = lib
    return _ref


# ---- convenience wrappers --------------------------------------------------

def _c(a):
    return np.ascontiguousarray(a)


def port_brute(tris, rays, clamp=True, nthreads=0):
    lib = port()
    tris, rays = _c(tris), _c(rays)
    out = np.empty(rays.shape[0], HIT)
    lib.eo_closest_brute(tris.ctypes.data, tris.shape[0], rays.ctypes.data, rays.shape[0],
                         int(clamp), out.ctypes.data, nthreads)
    return out


def port_occluded(tris, rays, clamp=True, nthreads=0):
    lib = port()
    tris, rays = _c(tris), _c(rays)
    out = np.empty(rays.shape[0], np.uint8)
    lib.eo_occluded_brute(tris.ctypes.data, tris.shape[0], rays.ctypes.data, rays.shape[0],
                          int(clamp), out.ctypes.data, nthreads)
    return out


def port_f64(tris, rays, nthreads=0):
    lib = port()
    tris, rays = _c(tris), _c(rays)
    out = np.empty(rays.shape[0], HIT)
    lib.eo_closest_f64(tris.ctypes.data, tris.shape[0], rays.ctypes.data, rays.shape[0],
                       out.ctypes.data, nthreads)
    return out


def pairs_f64(tris, rays, ids):
    """FP64 geometric test of each ray against one triangle (-1 = none)."""
    lib = port()
    tris, rays = _c(tris), _c(rays)
    ids = _c(np.asarray(ids, dtype=np.int32))
    hit = np.empty(len(ids), np.uint8)
    t = np.empty(len(ids), np.float64)
    lib.eo_pairs_f64(tris.ctypes.data, rays.ctypes.data, ids.ctypes.data, len(ids),
                     hit.ctypes.data, t.ctypes.data)
    return hit.astype(bool), t


def tri_test(tris, rays, ids, clamp=True):
    """The FP32 reference predicate for ray i against triangle ids[i]:
    (accepted, t, alpha, beta)."""
    lib = port()
    tris, rays = _c(tris), _c(rays)
    ids = _c(np.asarray(ids, dtype=np.int32))
    n = len(ids)
    acc = np.zeros(n, np.uint8)
    t, a, b = (np.zeros(n, np.float32) for _ in range(3))
    lib.eo_tri_test_batch(tris.ctypes.data, rays.ctypes.data, ids.ctypes.data, n, int(clamp),
                          acc.ctypes.data, t.ctypes.data, a.ctypes.data, b.ctypes.data)
    return acc.astype(bool), t, a, b


def classify(tris, rays, got, want):
    """Mismatch classes between two closest-hit results on the same rays:
    'tie' (both triangles accepted by the FP32 predicate with the same t),
    'want_false_positive' / 'got_false_positive' (that side's triangle is not
    hit geometrically in FP64: a clamp artefact of the reference predicate),
    'grazing' (|t_got - t_want| <= 1e-5 relative), 'unexplained'.
    Returns (indices of mismatches, list of class names)."""
    mism = np.nonzero(got["tri"] != want["tri"])[0]
    if len(mism) == 0:
        return mism, []
    r = rays[mism]
    gh, gt = pairs_f64(tris, r, got["tri"][mism])
    wh, wt = pairs_f64(tris, r, want["tri"][mism])
    ga, gtt, _, _ = tri_test(tris, r, got["tri"][mism])
    wa, wtt, _, _ = tri_test(tris, r, want["tri"][mism])
    classes = []
    for j in range(len(mism)):
        g_id, w_id = got["tri"][mism[j]], want["tri"][mism[j]]
        if g_id >= 0 and w_id >= 0 and ga[j] and wa[j] and gtt[j] == wtt[j]:
            classes.append("tie")
        elif w_id >= 0 and not wh[j]:
            classes.append("want_false_positive")
        elif g_id >= 0 and not gh[j]:
            classes.append("got_false_positive")
        elif g_id >= 0 and w_id >= 0 and abs(float(got["t"][mism[j]]) - float(want["t"][mism[j]])) <= 1e-5 * abs(float(want["t"][mism[j]])):
            classes.append("grazing")
        else:
            classes.append("unexplained")
    return mism, classes


class PortKd:
    def __init__(self, tris):
        self.lib = port()
        self.tris = _c(tris)
        md, nn, ni = C.c_int(), C.c_long(), C.c_long()
        self.h = self.lib.eo_kd_build(self.tris.ctypes.data, self.tris.shape[0], C.byref(md),
                                      C.byref(nn), C.byref(ni))
        self.max_depth, self.nnodes, self.nitems = md.value, nn.value, ni.value

    def closest(self, rays, clamp=True, nthreads=0):
        rays = _c(rays)
        out = np.empty(rays.shape[0], HIT)
        self.lib.eo_kd_closest(self.h, rays.ctypes.data, rays.shape[0], int(clamp),
                               out.ctypes.data, nthreads)
        return out

    def __del__(self):
        try:
            self.lib.eo_kd_free(self.h)
        except Exception:
            pass


def port_gather(pos, nrm, power, qpos, qnrm, k, max_dist, ignore_normal=False, caustic=False,
                with_sets=False, nthreads=0):
    lib = port()
    pos, nrm, power, qpos, qnrm = map(lambda a: _c(a.astype(np.float32)), (pos, nrm, power, qpos, qnrm))
    h = lib.eo_pmap_build(pos.ctypes.data, nrm.ctypes.data, power.ctypes.data, pos.shape[0])
    nq = qpos.shape[0]
    rgb = np.empty((nq, 3), np.float64)
    idx = np.empty((nq, k), np.int32) if with_sets else None
    d2 = np.empty((nq, k), np.float32) if with_sets else None
    cnt = np.empty(nq, np.int32)
    lib.eo_pmap_gather(h, qpos.ctypes.data, qnrm.ctypes.data, nq, k, max_dist, int(ignore_normal),
                       int(caustic), rgb.ctypes.data, idx.ctypes.data if with_sets else None,
                       d2.ctypes.data if with_sets else None, cnt.ctypes.data, nthreads)
    lib.eo_pmap_free(h)
    return (rgb, cnt, idx, d2) if with_sets else (rgb, cnt)


def ref_closest(tris, rays, kind=0, nthreads=0):
    """kind 0 = Kdtree, 1 = Bvh, 2 = BasicAS.  rays (N, 8); tmin/tmax ignored."""
    lib = reference()
    tris = _c(tris)
    r6 = _c(np.concatenate([rays[:, 0:3], rays[:, 4:7]], axis=1).astype(np.float32))
    bs = C.c_double()
    h = lib.encref_scene_create(tris.ctypes.data, tris.shape[0], kind, C.byref(bs))
    n = r6.shape[0]
    out = np.zeros(n, HIT)
    tid = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    a = np.empty(n, np.float32)
    b = np.empty(n, np.float32)
    lib.encref_closest(h, r6.ctypes.data, n, tid.ctypes.data, t.ctypes.data, a.ctypes.data,
                       b.ctypes.data, nthreads)
    lib.encref_scene_destroy(h)
    out["tri"], out["t"], out["u"], out["v"] = tid, t, a, b
    return out, bs.value


def ref_occluded(tris, rays, kind=0, nthreads=0):
    lib = reference()
    tris = _c(tris)
    r7 = _c(np.concatenate([rays[:, 0:3], rays[:, 4:7], rays[:, 7:8]], axis=1).astype(np.float32))
    bs = C.c_double()
    h = lib.encref_scene_create(tris.ctypes.data, tris.shape[0], kind, C.byref(bs))
    out = np.empty(r7.shape[0], np.uint8)
    lib.encref_occluded(h, r7.ctypes.data, r7.shape[0], out.ctypes.data, nthreads)
    lib.encref_scene_destroy(h)
    return out


def ref_model_load(path, center, size, angle, axis):
    """The reference's Model::load + centerModel on a mesh file: (N, 9) float32
    in primitive-list order (needs oracle/_ref/libencore_ref.so)."""
    lib = reference()
    c = np.ascontiguousarray(center, np.float32)
    ax = np.ascontiguousarray(axis, np.float32)
    b = str(path).encode()
    n = lib.encref_model_load(b, c.ctypes.data, size, angle, ax.ctypes.data, None, 0)
    out = np.empty((n, 9), np.float32)
    lib.encref_model_load(b, c.ctypes.data, size, angle, ax.ctypes.data, out.ctypes.data, n)
    return out
