"""Generates tests/golden/fullsize_mismatches.npz: every ray of the bench's
full-size batch whose closest hit differs between the wide BVH and the
reference Kdtree walk, with its class.

Runs on a GPU box (the engine traces the 4,179,838-ray batch; the kd-tree
mode, bit-exact with the reference's Kdtree::intersect at every scale, gives
the reference's answers).  The classes come from the oracle
(oracle/bindings.py:classify with the reference kd walk restated in C):

    python tests/golden/make_fullsize_mismatches.py [out.npz]

Two scales of the same workload (2,097,152-triangle heightfield, 1M
top-down primaries + 3 cosine bounces each, shuffled):
  x1000  the bench's scale;
  x1e5   a scale at which the Cross() clamp (|c| < 0.001) no longer acts on
         ordinary geometry: cells are 98 units across, so only rays crossing
         a shared edge differ.
Per scale the file holds `<tag>_idx` (ray index in the batch), `<tag>_got`
and `<tag>_want` (engine and reference hit records: tri, t, u, v),
`<tag>_cls` (index into `classes`).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

SCALES = {"x1000": 1000.0, "x100000": 100000.0}


def workload(scale: float):
    import bench
    from encore_b200 import Accelerator
    tris = bench.make_scene(seed=1, scale=scale)
    prim = bench.primary_rays(bench.RES, scale=scale)
    acc = Accelerator("wbvh").build(tris)
    ph = acc.intersect(prim)
    rays = bench.mixed_batch(tris, prim, ph, seed=101, scale=scale)
    return tris, rays, acc


def mismatches(tris, rays, acc):
    """(idx, got, want, classes) against the kd-tree mode."""
    from encore_b200 import Accelerator
    from oracle import bindings as ob
    got = acc.intersect(rays)
    kd = Accelerator("kdtree").build(tris)
    want = kd.intersect(rays)
    kd.destroy()
    mism, classes = ob.classify(tris, rays, got, want, kd=ob.PortKd(tris))
    return mism, got[mism], want[mism], classes


def main(out: str) -> None:
    from oracle import bindings as ob
    res = {"classes": np.array(ob.CLASS_NAMES)}
    for tag, scale in SCALES.items():
        tris, rays, acc = workload(scale)
        idx, got, want, classes = mismatches(tris, rays, acc)
        acc.destroy()
        res[f"{tag}_idx"] = idx.astype(np.int64)
        res[f"{tag}_got"] = got
        res[f"{tag}_want"] = want
        res[f"{tag}_cls"] = np.array([ob.CLASS_NAMES.index(c) for c in classes], np.int8)
        counts = {c: classes.count(c) for c in ob.CLASS_NAMES if classes.count(c)}
        print(f"{tag}: {len(rays)} rays, {len(idx)} differ: {counts}", flush=True)
    np.savez_compressed(out, **res)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).with_name("fullsize_mismatches.npz")))
