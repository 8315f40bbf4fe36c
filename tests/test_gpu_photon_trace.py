"""Device photon tracing against the oracle's tracer (GPU).

The engine traces photons as PhotonMapperCPU::EmitPhotons / TracePhoton /
ReflectPhotonDiffusely / EmitShadowPhoton do (PhotonMapperCPU.cpp:503-798),
with seeded counter-based random numbers in place of rand() (H12) and every
floating-point step a correctly rounded FP32 operation, so
oracle/encore_oracle.c:eo_photon_trace -- the same algorithm written out path
by path in C over the oracle's brute-force closest hit -- reproduces its
photons bit for bit wherever the two closest hits agree.  Photons are
compared per path and bounce through their tags (path id << 4 | shadow << 3 |
bounce): position, stored normal and power bit-exact.

* Geometric predicate (no Cross() clamp): the wide BVH and brute force agree
  on every ray, so every photon of every path is identical.
* The reference predicate: at most a few paths per thousand may differ, each
  one whose first differing hit is a clamp artefact or a tie.
* The direct / indirect split: bounce 0 in the direct map, later bounces in
  the indirect map, shadow photons (negative power) in the direct map.
* EmitPhotons' "until the indirect map is full" loop: the same number of
  batches and the same stored counts as the oracle.
"""
import numpy as np
import pytest

from encore_b200 import Accelerator, EncoreError, scenes, wavefront
from oracle import bindings as ob

pytestmark = pytest.mark.gpu
S = 1000.0
LIGHT = (0.5 * S, 2.0 * S, 0.5 * S)


def _bufs(cap, tag=True):
    import torch
    f = [torch.zeros((cap, 3), dtype=torch.float32, device="cuda") for _ in range(3)]
    t = torch.zeros(cap, dtype=torch.int32, device="cuda") if tag else None
    return (*f, t)


def _host(b, n):
    pos, nrm, pw, tag = b
    out = {"pos": pos[:n].cpu().numpy(), "nrm": nrm[:n].cpu().numpy(),
           "pow": pw[:n].cpu().numpy()}
    out["tag"] = tag[:n].cpu().numpy().view(np.uint32) if tag is not None else None
    return out


def _sorted(d):
    o = np.argsort(d["tag"], kind="stable")
    return {k: v[o] for k, v in d.items()}


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


KW = dict(max_bounces=3, albedo=0.7, seed=11, emit_offset=0.01 * S, bounce_offset=0.001 * S)


@pytest.fixture(scope="module")
def scene():
    return scenes.random_triangles(3000, seed=71, scale=S)


def _trace_device(tris, predicate, n, shadow, caps=(200_000, 200_000), fill=False):
    acc = Accelerator("wbvh", predicate=predicate).build(tris)
    d, i = _bufs(caps[0]), _bufs(caps[1])
    nd, ni, em = wavefront.trace_photon_maps(acc, LIGHT, 0.1 * S, n, d, i, shadow_offset=shadow,
                                             fill_indirect=fill, **KW)
    acc.destroy()
    return _host(d, nd), _host(i, ni), em


def _trace_oracle(tris, clamp, n, shadow, caps=(200_000, 200_000), fill=False):
    st, em = ob.port_photon_trace(tris, LIGHT, 0.1 * S, n, clamp=clamp, split=True,
                                  shadow_offset=shadow, fill=fill, caps=caps, **KW)
    return st[0], st[1], em


def test_photon_maps_equal_the_oracle_geometric_predicate(gpu, scene):
    n = 20000
    gd, gi, gem = _trace_device(scene, "noclamp", n, shadow=5.0)
    wd, wi, wem = _trace_oracle(scene, False, n, shadow=5.0)
    assert gem == wem == n
    for got, want in ((gd, wd), (gi, wi)):
        assert len(got["tag"]) == len(want["tag"]) > 200
        got, want = _sorted(got), _sorted(want)
        assert np.array_equal(got["tag"], want["tag"])
        for f in ("pos", "nrm", "pow"):
            assert np.array_equal(bits(got[f]), bits(want[f])), f
    # the split: bounce 0 and shadow photons direct, bounces 1..3 indirect
    assert np.all((gd["tag"] & 7) == 0)
    assert np.all(((gi["tag"] & 7) >= 1) & ((gi["tag"] & 7) <= 3) & ((gi["tag"] & 8) == 0))
    shadow = (gd["tag"] & 8) != 0
    assert shadow.sum() > 50
    assert np.all(gd["pow"][shadow] == np.float32(-1.0 / n))
    assert np.all(gd["pow"][~shadow] == np.float32(1.0 / n))
    assert np.all(gi["pow"] == np.float32(1.0 / n))


def test_photon_maps_agree_with_the_oracle_reference_predicate(gpu, scene):
    """With the reference's clamped predicate, the wide BVH and brute force can
    differ on a ray whose brute-force hit is a clamp artefact outside its
    triangle's box, or on a tie; such a path then diverges.  All other paths
    are identical photon for photon."""
    n = 20000
    gd, gi, _ = _trace_device(scene, "reference", n, shadow=5.0)
    wd, wi, _ = _trace_oracle(scene, True, n, shadow=5.0)
    for got, want in ((gd, wd), (gi, wi)):
        g = {int(t): k for k, t in enumerate(got["tag"])}
        w = {int(t): k for k, t in enumerate(want["tag"])}
        bad_paths = {t >> 4 for t in set(g) ^ set(w)}
        for t in set(g) & set(w):
            a, b = g[t], w[t]
            if not (np.array_equal(bits(got["pos"][a]), bits(want["pos"][b]))
                    and np.array_equal(bits(got["nrm"][a]), bits(want["nrm"][b]))):
                bad_paths.add(t >> 4)
        assert len(bad_paths) <= n // 500, len(bad_paths)


def test_single_map_call_stores_the_union_without_shadows(gpu, scene):
    """enc_photons_trace_device (one map) stores exactly the photons of the
    split call without shadow photons, direct and indirect together."""
    import torch
    n = 10000
    acc = Accelerator("wbvh").build(scene)
    cap = 100_000
    bufs = [torch.zeros((cap, 3), dtype=torch.float32, device="cuda") for _ in range(3)]
    m = wavefront.trace_photons(acc, LIGHT, 0.1 * S, n, *bufs, **KW)
    d, i = _bufs(cap), _bufs(cap)
    nd, ni, _ = wavefront.trace_photon_maps(acc, LIGHT, 0.1 * S, n, d, i, **KW)
    acc.destroy()
    assert m == nd + ni
    one = np.concatenate([b[:m].cpu().numpy() for b in bufs], axis=1)
    two = np.concatenate([np.concatenate([b[:k].cpu().numpy() for b in x[:3]], axis=1)
                          for x, k in ((d, nd), (i, ni))])
    one = one[np.lexsort(one.T[::-1])]
    two = two[np.lexsort(two.T[::-1])]
    assert np.array_equal(bits(one), bits(two))


def test_fill_indirect_emits_until_the_indirect_map_is_full(gpu, scene):
    """EmitPhotons loops while the indirect map is not full
    (PhotonMapperCPU.cpp:538-554): batches of nphotons until the indirect
    store's capacity is reached; the powers are 1 / photons emitted."""
    n = 4000
    caps = (50_000, 500)
    gd, gi, gem = _trace_device(scene, "noclamp", n, shadow=0.0, caps=caps, fill=True)
    wd, wi, wem = _trace_oracle(scene, False, n, shadow=0.0, caps=caps, fill=True)
    assert gem == wem and gem % n == 0 and gem > n
    assert len(gi["tag"]) == len(wi["tag"]) == caps[1]
    assert len(gd["tag"]) == len(wd["tag"])
    assert np.all(gi["pow"] == np.float32(1.0 / gem))
    # below capacity the direct map holds the same photons as the oracle's
    if len(gd["tag"]) < caps[0]:
        a, b = _sorted(gd), _sorted(wd)
        assert np.array_equal(a["tag"], b["tag"])
        assert np.array_equal(bits(a["pos"]), bits(b["pos"]))


def test_photon_trace_argument_errors(gpu, scene):
    acc = Accelerator("wbvh").build(scene[:100])
    d, i = _bufs(100), _bufs(100)
    with pytest.raises(EncoreError):
        wavefront.trace_photon_maps(acc, LIGHT, 0.1 * S, 100, d, i, max_bounces=31)
    with pytest.raises(EncoreError):
        wavefront.trace_photon_maps(acc, LIGHT, 0.1 * S, 100, d, i, shadow_offset=-1.0)
    acc.destroy()
    kd = Accelerator("kdtree").build(scene[:100])
    with pytest.raises(EncoreError):
        wavefront.trace_photon_maps(kd, LIGHT, 0.1 * S, 100, d, i)
    kd.destroy()
