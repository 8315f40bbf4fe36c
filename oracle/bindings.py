"""ctypes access to the two oracles.  Test infrastructure: imported only by
tests/, __graft_entry__.smoke() and the CPU arm of bench.py.

* port()      : oracle/_ref/libencore_oracle.so, the C restatement in oracle/*.c
* reference() : oracle/_ref/libencore_ref.so, the reference's own CPU code
                compiled from its sources by oracle/Makefile (None if absent)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ORACLE = Path(__file__).resolve().parent
PORT_SO = ORACLE / "_ref" / "libencore_oracle.so"
REF_SO = ORACLE / "_ref" / "libencore_ref.so"
# The reference's source tree (read only, to compile oracle/_ref and to read
# its shipped meshes and scene files): $ENCORE_REFERENCE_DIR, else the
# location oracle/Makefile defaults to.
REFERENCE_DIR = Path(os.environ.get("ENCORE_REFERENCE_DIR", "/root/reference/ENCORE"))

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
        lib.eo_kd_tested.argtypes = [P, P, P, C.c_long, C.c_int, P, C.c_int]
        lib.eo_kd_leaves_at.argtypes = [P, P, C.c_float, P, C.c_int]
        lib.eo_kd_leaves_at.restype = C.c_int
        lib.eo_kd_leaf_has.argtypes = [P, C.c_int32, C.c_int32]
        lib.eo_kd_leaf_has.restype = C.c_int
        lib.eo_kd_walk.argtypes = [P, P, C.c_int, P, P, P, C.c_int]
        lib.eo_kd_walk.restype = C.c_int
        lib.eo_pmap_build.restype = P
        lib.eo_pmap_build.argtypes = [P, P, P, C.c_long]
        lib.eo_pmap_gather.argtypes = [P, P, P, C.c_long, C.c_int, C.c_float, C.c_int, C.c_int,
                                       P, P, P, P, C.c_int]
        lib.eo_pmap_free.argtypes = [P]
        lib.eo_photon_trace.argtypes = [P, C.c_int, P, C.c_int, C.c_int, C.c_float, C.c_int, P, P,
                                        P, P, C.c_int]
        lib.eo_photon_trace.restype = C.c_int
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
        lib.encref_camera_rays.argtypes = [P, P, P, C.c_float, C.c_float, C.c_float, C.c_int,
                                           C.c_int, P]
        lib.encref_hit_surface.argtypes = [P, P, P, C.c_long, P, P]
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


def share_vertex(tris, a, b):
    """True where triangles a[i] and b[i] (both >= 0) have a vertex with the
    same three float coordinates (neighbours across an edge or a corner)."""
    t = np.asarray(tris, np.float32).reshape(-1, 3, 3)
    va = t[np.maximum(a, 0)][:, :, None, :]
    vb = t[np.maximum(b, 0)][:, None, :, :]
    same = np.all(va == vb, axis=-1).any(axis=(1, 2))
    return same & (a >= 0) & (b >= 0)


CLASS_NAMES = ("tie", "edge", "want_false_positive", "got_false_positive", "grazing",
               "closer_untested", "unexplained", "split_plane_nan")


def classify(tris, rays, got, want, kd=None):
    """Mismatch classes between two closest-hit results on the same rays
    (got = the engine, want = the reference), first match wins:
    'tie'   both triangles accepted by the FP32 predicate with the same t (a
            shared edge met in a different order, H7);
    'edge'  both accepted by the FP32 predicate, t within 1e-5 relative, and
            the two triangles share a vertex: the ray crosses their common
            edge or corner, and FP32 rounding decides which side accepts it;
    'want_false_positive' / 'got_false_positive'  that side's triangle is not
            hit geometrically in FP64 (a Cross() clamp artefact);
    'grazing'  |t_got - t_want| <= 1e-5 relative, both geometric;
    'split_plane_nan'  (only with kd): as closer_untested, for a ray whose
            origin lies exactly on a kd split plane and whose direction has
            an exactly zero component (the reference's Normalize snaps
            components below 0.001 to 0, H2): along that axis
            Kdtree::intersect forms tplane = (split - o) * (1 / 0) = 0 * inf
            = NaN (Kdtree.cpp:712), and its walk's [tmin, tmax] bookkeeping
            passes over the cells that hold the hit;
    'closer_untested'  (only with kd = the reference's kd walk, a PortKd):
            got's hit is geometric in FP64 and closer than want's (or want
            misses), and the kd walk never tests got's triangle -- its cells
            along the ray do not list it (a triangle that only touches a
            cell's face is not distributed into it, Kdtree.cpp:579-585);
    'unexplained'  anything else.
    Returns (indices of mismatches, list of class names)."""
    mism = np.nonzero(got["tri"] != want["tri"])[0]
    if len(mism) == 0:
        return mism, []
    r = rays[mism]
    gid, wid = got["tri"][mism], want["tri"][mism]
    gh, gt = pairs_f64(tris, r, gid)
    wh, wt = pairs_f64(tris, r, wid)
    ga, gtt, _, _ = tri_test(tris, r, gid)
    wa, wtt, _, _ = tri_test(tris, r, wid)
    nb = share_vertex(tris, gid, wid)
    untested = np.zeros(len(mism), bool)
    if kd is not None:
        untested = ~kd.tested(r, gid)
    classes = []
    for j in range(len(mism)):
        g_id, w_id = gid[j], wid[j]
        tg, tw = float(got["t"][mism[j]]), float(want["t"][mism[j]])
        close = g_id >= 0 and w_id >= 0 and abs(tg - tw) <= 1e-5 * abs(tw)
        if g_id >= 0 and w_id >= 0 and ga[j] and wa[j] and gtt[j] == wtt[j]:
            classes.append("tie")
        elif close and ga[j] and wa[j] and nb[j]:
            classes.append("edge")
        elif w_id >= 0 and not wh[j]:
            classes.append("want_false_positive")
        elif g_id >= 0 and not gh[j]:
            classes.append("got_false_positive")
        elif close:
            classes.append("grazing")
        elif (kd is not None and g_id >= 0 and gh[j] and (w_id < 0 or tg < tw)
              and untested[j]):
            rr = r[j]
            in_plane = bool(np.any(rr[4:7] == 0)) and len(kd.leaves_at(rr[0:3], 0.0)) > 1
            classes.append("split_plane_nan" if in_plane else "closer_untested")
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

    def leaves_at(self, p, eps=0.0):
        """Leaves whose cells contain point p (both sides of a split within eps)."""
        pt = np.ascontiguousarray(p, np.float32)
        out = np.empty(256, np.int32)
        n = self.lib.eo_kd_leaves_at(self.h, pt.ctypes.data, float(eps), out.ctypes.data, 256)
        return out[:n]

    def leaf_has(self, leaf, tri_id):
        return bool(self.lib.eo_kd_leaf_has(self.h, int(leaf), int(tri_id)))

    def walk(self, ray, clamp=True, max_leaves=4096):
        """The leaves one ray's reference walk visits: (leaves, tmin, tmax)."""
        r = np.ascontiguousarray(ray, np.float32)
        lv = np.empty(max_leaves, np.int32)
        t0 = np.empty(max_leaves, np.float32)
        t1 = np.empty(max_leaves, np.float32)
        n = self.lib.eo_kd_walk(self.h, r.ctypes.data, int(clamp), lv.ctypes.data,
                                t0.ctypes.data, t1.ctypes.data, max_leaves)
        return lv[:n], t0[:n], t1[:n]

    def tested(self, rays, ids, clamp=True, nthreads=0):
        """Per ray: does the reference kd walk test triangle ids[i] at all?"""
        rays = _c(rays)
        ids = _c(np.asarray(ids, dtype=np.int32))
        out = np.zeros(rays.shape[0], np.uint8)
        self.lib.eo_kd_tested(self.h, rays.ctypes.data, ids.ctypes.data, rays.shape[0],
                              int(clamp), out.ctypes.data, nthreads)
        return out.astype(bool)

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


def ref_camera_rays(eye, look, up, fov_deg, width, height, near=1.0):
    """Eye rays from the reference's own Camera basis and Vector3 arithmetic
    (ref_harness.cpp:encref_camera_rays): (width*height, 8) float32."""
    lib = reference()
    e, l, u = (np.ascontiguousarray(x, np.float32) for x in (eye, look, up))
    out = np.empty((width * height, 8), np.float32)
    lib.encref_camera_rays(e.ctypes.data, l.ctypes.data, u.ctypes.data, float(fov_deg),
                           float(np.float32(width / height)), float(near), int(width),
                           int(height), out.ctypes.data)
    return out


def ref_hit_surface(tris, rays, ids):
    """Hit point and normal that the reference's TrianglePrim::intersect stores
    for ray i against triangle ids[i] (NaN where none): two (n, 3) arrays."""
    lib = reference()
    tris, rays = _c(np.asarray(tris, np.float32)), _c(np.asarray(rays, np.float32))
    ids = _c(np.asarray(ids, dtype=np.int32))
    n = len(ids)
    pos = np.empty((n, 3), np.float32)
    nrm = np.empty((n, 3), np.float32)
    lib.encref_hit_surface(tris.ctypes.data, rays.ctypes.data, ids.ctypes.data, n,
                           pos.ctypes.data, nrm.ctypes.data)
    return pos, nrm


class _PhotonOpts(C.Structure):
    _fields_ = [("light_center", C.c_float * 3), ("light_size", C.c_float),
                ("nphotons", C.c_uint32), ("max_bounces", C.c_uint32), ("albedo", C.c_float),
                ("seed", C.c_uint32), ("emit_offset", C.c_float), ("bounce_offset", C.c_float)]


class _PhotonOut(C.Structure):
    _fields_ = [("pos", P), ("nrm", P), ("pow", P), ("tag", P), ("capacity", C.c_uint32)]


def port_photon_trace(tris, light_center, light_size, nphotons, max_bounces=3, albedo=0.7,
                      seed=1, emit_offset=0.01, bounce_offset=0.001, clamp=True, split=False,
                      shadow_offset=0.0, fill=False, caps=(1 << 20, 1 << 20), nthreads=0):
    """The oracle's photon tracer (encore_oracle.c:eo_photon_trace).  Returns a
    list of one or two stores, each a dict of pos, nrm, pow (n, 3) and tag
    (n,), plus the number of paths emitted."""
    lib = port()
    tris = _c(np.asarray(tris, np.float32))
    o = _PhotonOpts((C.c_float * 3)(*light_center), light_size, nphotons, max_bounces, albedo,
                    seed, emit_offset, bounce_offset)
    stores, outs = [], []
    for m in range(2 if split else 1):
        cap = int(caps[m])
        d = {"pos": np.zeros((cap, 3), np.float32), "nrm": np.zeros((cap, 3), np.float32),
             "pow": np.zeros((cap, 3), np.float32), "tag": np.zeros(cap, np.uint32)}
        stores.append(d)
        outs.append(_PhotonOut(d["pos"].ctypes.data, d["nrm"].ctypes.data, d["pow"].ctypes.data,
                               d["tag"].ctypes.data, cap))
    stored = (C.c_uint32 * 2)()
    emitted = C.c_uint32()
    rc = lib.eo_photon_trace(tris.ctypes.data, tris.shape[0], C.byref(o), int(clamp), int(split),
                             float(shadow_offset), int(fill), C.byref(outs[0]),
                             C.byref(outs[1]) if split else None, stored, C.byref(emitted),
                             nthreads)
    if rc:
        raise RuntimeError("oracle photon tracer: a shadow ray left 32 surfaces")
    for m, d in enumerate(stores):
        k = stored[m]
        for key in d:
            d[key] = d[key][:k]
    return stores, emitted.value
