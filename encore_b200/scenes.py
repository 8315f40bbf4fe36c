"""Seeded synthetic scenes, rays and photons for the workloads the engine is
measured on.  All arrays are FP32 and generated with numpy's PCG64, so they
are identical on every machine for a given seed.

Workloads (sizes as named by the workload, `scale` multiplies every
coordinate; scale 1000 is the size at which the reference's Cross() clamp of
|c| < 0.001 does not act on ordinary geometry):

* random_triangles  : N triangles, centroids uniform in [0,1]^3, each vertex =
                      centroid + L*u with L ~ U[0.005, 0.05] and u uniform on
                      the unit sphere.
* heightfield       : a 1024x1024 quad grid (2,097,152 triangles) over [0,1]^2
                      in x/z, y = 0.2 * fBm (6 octaves of seeded value noise).
* camera_rays       : pinhole eye rays, one per pixel centre, formed as
                      RayTracer::CalcEyeRaySamples does (RayTracer.cpp:489-525)
                      with the camera basis of Camera::CalcCamVectors
                      (Camera.cpp:157-166) and the clamping Normalize/Cross.
* diffuse_rays      : cosine-weighted directions about the hit triangle's
                      normal, from primary hit points.
* shadow_rays       : from hit points toward a random point on a 0.1 x 0.1
                      area light at height 2.0, origin offset 0.01 along the
                      direction and tmax = distance to the light, as
                      PhotonMapperCPU::IsInShadow forms them (:1192-1207).

Rays are (N, 8) float32: ox, oy, oz, tmin, dx, dy, dz, tmax.
"""
from __future__ import annotations

import numpy as np

F32 = np.float32
EPS = F32(0.001)  # ENC_EPSILON, Vector3.h:18-20
PI_F = F32(3.14159)  # Common.h:36


# ---------------------------------------------------------------------------
# FP32 vector helpers with the reference's semantics (Vector3.h / .cpp)

def _clamp(v: np.ndarray) -> np.ndarray:
    v = v.copy()
    v[(v > -EPS) & (v < EPS)] = F32(0)
    return v


def cross_ref(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Cross() with ClampfloatoZero (Vector3.h:148-161), FP32, last axis = xyz."""
    a = a.astype(F32, copy=False)
    b = b.astype(F32, copy=False)
    x = a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1]
    y = -(a[..., 0] * b[..., 2] - a[..., 2] * b[..., 0])
    z = a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]
    return _clamp(np.stack([x, y, z], axis=-1).astype(F32))


def normalize_ref(v: np.ndarray) -> np.ndarray:
    """Normalize(): divide by sqrt of the FP32 sum of squares, then clamp
    (Vector3.cpp:105-124)."""
    v = v.astype(F32, copy=False)
    m2 = (v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2]
    m = np.sqrt(m2.astype(np.float64)).astype(F32)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = (v / m[..., None]).astype(F32)
    return _clamp(out)


def tri_normals_ref(tris: np.ndarray) -> np.ndarray:
    """Geometric normal as the reference stores it on a hit:
    Normalize(Cross(edge1, edge2)) (TrianglePrim.cpp:236-238)."""
    t = tris.reshape(-1, 3, 3).astype(F32)
    e1 = t[:, 1] - t[:, 0]
    e2 = t[:, 2] - t[:, 0]
    return normalize_ref(cross_ref(e1, e2))


# ---------------------------------------------------------------------------
# scenes

def random_triangles(n: int, seed: int = 0, scale: float = 1.0) -> np.ndarray:
    """(n, 9) float32 triangle soup; see module docstring."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3))
    L = rng.uniform(0.005, 0.05, size=(n, 3, 1))
    u = rng.normal(size=(n, 3, 3))
    u /= np.linalg.norm(u, axis=2, keepdims=True)
    v = (c + L * u) * scale
    return v.reshape(n, 9).astype(F32)


def _value_noise(x: np.ndarray, z: np.ndarray, freq: int, rng: np.random.Generator) -> np.ndarray:
    lat = rng.random((freq + 2, freq + 2))
    gx = x * freq
    gz = z * freq
    ix = np.floor(gx).astype(np.int64)
    iz = np.floor(gz).astype(np.int64)
    fx = gx - ix
    fz = gz - iz
    sx = fx * fx * (3 - 2 * fx)
    sz = fz * fz * (3 - 2 * fz)
    a = lat[ix, iz]
    b = lat[ix + 1, iz]
    c = lat[ix, iz + 1]
    d = lat[ix + 1, iz + 1]
    return (a * (1 - sx) + b * sx) * (1 - sz) + (c * (1 - sx) + d * sx) * sz


def heightfield(res: int = 1024, seed: int = 0, scale: float = 1.0, amplitude: float = 0.2,
                octaves: int = 6) -> np.ndarray:
    """(2*res*res, 9) float32 heightfield triangles, row-major quads, two
    triangles per quad: (v00, v10, v11) and (v00, v11, v01)."""
    rng = np.random.default_rng(seed)
    t = np.linspace(0.0, 1.0, res + 1)
    X, Z = np.meshgrid(t, t, indexing="ij")
    h = np.zeros_like(X)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        h += amp * _value_noise(X, Z, 4 * 2 ** o, rng)
        total += amp
        amp *= 0.5
    Y = amplitude * h / total
    V = np.stack([X, Y, Z], axis=-1) * scale  # (res+1, res+1, 3)
    v00 = V[:-1, :-1].reshape(-1, 3)
    v10 = V[1:, :-1].reshape(-1, 3)
    v11 = V[1:, 1:].reshape(-1, 3)
    v01 = V[:-1, 1:].reshape(-1, 3)
    t1 = np.concatenate([v00, v10, v11], axis=1)
    t2 = np.concatenate([v00, v11, v01], axis=1)
    tris = np.stack([t1, t2], axis=1).reshape(-1, 9)
    return tris.astype(F32)


# ---------------------------------------------------------------------------
# rays

def camera_rays(width: int, height: int, eye, look, up=(0.0, 1.0, 0.0), fov_deg: float = 45.0,
                near: float = 1.0) -> np.ndarray:
    """One ray per pixel centre; rows from the bottom of the image
    (Vr = -H + 2H y / rows, RayTracer.cpp:505-506)."""
    eye = np.asarray(eye, dtype=F32)
    look = np.asarray(look, dtype=F32)
    up = np.asarray(up, dtype=F32)
    n = (eye - look).astype(F32)
    u = cross_ref(up, n)
    n = normalize_ref(n)
    u = normalize_ref(u)
    v = cross_ref(n, u)
    # H = near * tan(angle * (PI / 360.0)) evaluated in double, as the float
    # angle times the double constant promotes (RayTracer.cpp:495)
    H = F32(near * np.tan(np.float64(F32(fov_deg)) * (float(PI_F) / 360.0)))
    W = F32(H * F32(width / height))
    cols = np.arange(width, dtype=F32) + F32(0.5)
    rows = np.arange(height, dtype=F32) + F32(0.5)
    Uc = (-W + (W * (F32(2) * cols) / F32(width))).astype(F32)
    Vr = (-H + (H * (F32(2) * rows) / F32(height))).astype(F32)
    R, Cc = np.meshgrid(Vr, Uc, indexing="ij")  # (height, width)
    dn = (n * F32(-near)).astype(F32)
    d = (dn[None, None, :] + u[None, None, :] * Cc[..., None]).astype(F32)
    d = (d + v[None, None, :] * R[..., None]).astype(F32)
    d = normalize_ref(d.reshape(-1, 3))
    rays = np.zeros((d.shape[0], 8), dtype=F32)
    rays[:, 0:3] = eye
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def random_sphere_rays(n: int, seed: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)) -> np.ndarray:
    """Origins uniform in the box, directions uniform on the unit sphere."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), dtype=F32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def hit_points(tris: np.ndarray, rays: np.ndarray, tri_id: np.ndarray, u: np.ndarray,
               v: np.ndarray) -> np.ndarray:
    """v0 + (v1 - v0) * alpha + (v2 - v0) * beta (TrianglePrim.cpp:239) for hits."""
    t = tris.reshape(-1, 3, 3)[tri_id]
    p = t[:, 0] + (t[:, 1] - t[:, 0]) * u[:, None] + (t[:, 2] - t[:, 0]) * v[:, None]
    return p.astype(F32)


def _orient(nrm: np.ndarray, d: np.ndarray) -> np.ndarray:
    s = np.sign(np.sum(nrm * d, axis=1))
    s[s == 0] = 1
    return (-nrm * s[:, None]).astype(F32)  # normal facing back toward the incoming ray


def cosine_directions(nrm: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Cosine-weighted unit directions about unit normals (n, 3)."""
    n = nrm.shape[0]
    r1 = rng.random(n)
    r2 = rng.random(n)
    phi = 2 * np.pi * r1
    sr = np.sqrt(r2)
    local = np.stack([np.cos(phi) * sr, np.sin(phi) * sr, np.sqrt(1 - r2)], axis=1)
    a = np.where(np.abs(nrm[:, 0:1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(a, nrm)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(nrm, t)
    d = local[:, 0:1] * t + local[:, 1:2] * b + local[:, 2:3] * nrm
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def diffuse_rays(tris: np.ndarray, prim_rays: np.ndarray, tri_id: np.ndarray, u: np.ndarray,
                 v: np.ndarray, per_hit: int, seed: int, offset: float) -> np.ndarray:
    """`per_hit` cosine-weighted secondaries from each primary hit; origins
    pushed `offset` along the facing normal."""
    hit = tri_id >= 0
    ids = tri_id[hit]
    p = hit_points(tris, prim_rays[hit], ids, u[hit], v[hit]).astype(np.float64)
    t = tris.reshape(-1, 3, 3)[ids].astype(np.float64)
    nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = _orient(nrm, prim_rays[hit, 4:7].astype(np.float64)).astype(np.float64)
    rng = np.random.default_rng(seed)
    p = np.repeat(p, per_hit, axis=0)
    nrm = np.repeat(nrm, per_hit, axis=0)
    d = cosine_directions(nrm, rng)
    rays = np.zeros((p.shape[0], 8), dtype=F32)
    rays[:, 0:3] = p + offset * nrm
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def shadow_rays(points: np.ndarray, seed: int, light_center, light_size: float,
                offset: float) -> np.ndarray:
    """Rays from surface points to uniform points on a square light facing -y.
    origin = point + offset * direction, tmax = |light point - surface point|
    (the reference uses offset 0.01 in unit-scene units)."""
    rng = np.random.default_rng(seed)
    n = points.shape[0]
    lc = np.asarray(light_center, dtype=np.float64)
    lp = np.empty((n, 3))
    lp[:, 0] = lc[0] + (rng.random(n) - 0.5) * light_size
    lp[:, 1] = lc[1]
    lp[:, 2] = lc[2] + (rng.random(n) - 0.5) * light_size
    p = points.astype(np.float64)
    d = lp - p
    dist = np.linalg.norm(d, axis=1)
    d /= dist[:, None]
    rays = np.zeros((n, 8), dtype=F32)
    rays[:, 0:3] = p + offset * d
    rays[:, 4:7] = d
    rays[:, 7] = dist
    return rays


# ---------------------------------------------------------------------------
# photons

def emit_from_light(n: int, seed: int, center, size: float) -> np.ndarray:
    """Photon rays from a square light facing -y with a cosine (Lambert) lobe,
    the distribution RectangleLight::EmitPhoton draws (RectangleLight.cpp:172-185)."""
    rng = np.random.default_rng(seed)
    c = np.asarray(center, dtype=np.float64)
    o = np.empty((n, 3))
    o[:, 0] = c[0] + (rng.random(n) - 0.5) * size
    o[:, 1] = c[1]
    o[:, 2] = c[2] + (rng.random(n) - 0.5) * size
    nrm = np.tile(np.array([[0.0, -1.0, 0.0]]), (n, 1))
    d = cosine_directions(nrm, rng)
    rays = np.zeros((n, 8), dtype=F32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def camera_rays_jittered(n: int, seed: int, eye, look, up=(0.0, 1.0, 0.0), fov_deg: float = 45.0,
                         res: int = 1024) -> np.ndarray:
    """n eye rays through uniformly random points of a res x res image, the
    jittered form of RayTracer::CalcEyeRaySamples (RayTracer.cpp:501-502)."""
    rng = np.random.default_rng(seed)
    eye = np.asarray(eye, dtype=F32)
    look = np.asarray(look, dtype=F32)
    up = np.asarray(up, dtype=F32)
    nv = (eye - look).astype(F32)
    u = normalize_ref(cross_ref(up, nv))
    nv = normalize_ref(nv)
    v = cross_ref(nv, u)
    H = F32(np.tan(F32(fov_deg) * (float(PI_F) / 360.0)))
    x = rng.random(n).astype(F32) * F32(res)
    y = rng.random(n).astype(F32) * F32(res)
    Uc = (-H + (H * (F32(2) * x) / F32(res))).astype(F32)
    Vr = (-H + (H * (F32(2) * y) / F32(res))).astype(F32)
    d = (-nv[None, :] + u[None, :] * Uc[:, None] + v[None, :] * Vr[:, None]).astype(F32)
    d = normalize_ref(d)
    rays = np.zeros((n, 8), dtype=F32)
    rays[:, 0:3] = eye
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def multi_scene_workload(nscenes: int = 64, seed: int = 0, scale: float = 1.0,
                         tri_range=(1_000, 500_000), ray_range=(4_096, 1_048_576)):
    """Scenes of random triangles with log-uniform triangle counts, each with a
    log-uniform-sized ray batch, half camera rays and half uniform-sphere rays.
    Returns (list of (N_i, 9) triangle arrays, list of (M_i, 8) ray arrays)."""
    rng = np.random.default_rng(seed)
    lt = np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]), nscenes)).astype(int)
    lr = np.exp(rng.uniform(np.log(ray_range[0]), np.log(ray_range[1]), nscenes)).astype(int)
    tris, rays = [], []
    for i in range(nscenes):
        t = random_triangles(int(lt[i]), seed=seed * 1000 + 2 * i, scale=scale)
        m = int(lr[i])
        cam = camera_rays_jittered(m // 2, seed=seed * 1000 + 2 * i + 1,
                                   eye=np.array([0.5, 0.5, -1.5]) * scale,
                                   look=np.array([0.5, 0.5, 0.5]) * scale)
        sph = random_sphere_rays(m - m // 2, seed=seed * 1000 + 2 * i + 2,
                                 hi=(scale, scale, scale))
        r = np.concatenate([cam, sph])
        rays.append(np.ascontiguousarray(r[rng.permutation(m)]))
        tris.append(t)
    return tris, rays


def surface_rays(tris: np.ndarray, n: int, seed: int, kind: str = "diffuse", light_center=None,
                 light_size: float = 0.1, offset: float = 1e-4, up_facing: bool = False) -> np.ndarray:
    """Rays leaving random points on random triangles of a scene: `diffuse`
    (cosine-weighted about the triangle normal, on a random side, or the +y
    side with up_facing) or `shadow` (toward a random point of a square light
    facing -y, tmax = distance, origin pushed `offset` along the ray)."""
    rng = np.random.default_rng(seed)
    t = tris.reshape(-1, 3, 3).astype(np.float64)
    ids = rng.integers(0, len(t), size=n)
    r1 = np.sqrt(rng.random(n))
    r2 = rng.random(n)
    p = ((1 - r1)[:, None] * t[ids, 0] + (r1 * (1 - r2))[:, None] * t[ids, 1]
         + (r1 * r2)[:, None] * t[ids, 2])
    if kind == "shadow":
        return shadow_rays(p.astype(F32), seed + 1, light_center, light_size, offset)
    nrm = np.cross(t[ids, 1] - t[ids, 0], t[ids, 2] - t[ids, 0])
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-300)
    if up_facing:
        nrm *= np.where(nrm[:, 1:2] < 0, -1.0, 1.0)
    else:
        nrm *= np.where(rng.random((n, 1)) < 0.5, -1.0, 1.0)
    d = cosine_directions(nrm, rng)
    rays = np.zeros((n, 8), dtype=F32)
    rays[:, 0:3] = p + offset * nrm
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays
