"""Autotuner for the traversal launch: sweeps BVH width, queue chunk size,
resident blocks per SM, block size and stack depth on a sample workload with
the batched multi-scene launch, and returns the fastest configuration.  Every
configuration must return the same hits as the first one (the launch shape
does not change results), which the tuner checks as it goes.
"""
from __future__ import annotations

import itertools
import json
import time
from pathlib import Path
from typing import Sequence

import numpy as np

from ._lib import EncoreError
from .accel import Accelerator, LaunchConfig
from .batch import BatchLaunch


def autotune(scene_tris: Sequence[np.ndarray], ray_batches: Sequence[np.ndarray],
             widths=(2, 4, 8), chunks=(16, 32, 64, 128), blocks_per_sm=(6, 8, 10),
             block_threads=(64, 128), stack_depths=(0,), reps: int = 5, device: int = 0,
             out: str | Path | None = None) -> dict:
    import torch
    dev = torch.device("cuda", device)
    d_rays = [torch.from_numpy(np.ascontiguousarray(r)).to(dev) for r in ray_batches]
    d_hits = [torch.empty((r.shape[0], 4), dtype=torch.int32, device=dev) for r in ray_batches]
    total = sum(r.shape[0] for r in ray_batches)
    results = []
    reference_tri = None
    for w in widths:
        accs = [Accelerator("wbvh", width=w, device=device).build(t) for t in scene_tris]
        for ch, bps, bt, sd in itertools.product(chunks, blocks_per_sm, block_threads, stack_depths):
            lc = LaunchConfig(block_threads=bt, blocks_per_sm=bps, chunk=ch, stack_depth=sd)
            b = BatchLaunch(list(zip(accs, d_rays, d_hits)), launch=lc)
            b.launch_graph()
            try:
                b.check()
            except EncoreError as e:
                # a stack shallower than the deepest tree stops rays at its
                # bound: the configuration is reported and never chosen
                b.destroy()
                results.append({"width": w, "chunk": ch, "blocks_per_sm": bps,
                                "block_threads": bt, "stack_depth": sd, "ms": None,
                                "mrays_s": None, "same_hits": False, "error": str(e)})
                continue
            tri = torch.cat([h[:, 0] for h in d_hits]).cpu().numpy()
            if reference_tri is None:
                reference_tri = tri
            same = bool(np.array_equal(tri, reference_tri))
            ts = []
            for _ in range(reps):
                a = torch.cuda.Event(enable_timing=True)
                e = torch.cuda.Event(enable_timing=True)
                a.record()
                b.launch_graph()
                e.record()
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(e))
            b.check()
            b.destroy()
            ms = float(np.median(ts))
            results.append({"width": w, "chunk": ch, "blocks_per_sm": bps, "block_threads": bt,
                            "stack_depth": sd, "ms": ms, "mrays_s": total / ms / 1e3,
                            "same_hits": same})
        for a in accs:
            a.destroy()
    ok = [r for r in results if r["same_hits"]]
    best = max(ok, key=lambda r: r["mrays_s"]) if ok else None
    failed = [r for r in results if "error" in r]
    report = {"best": best, "rays": total, "scenes": len(scene_tris),
              "all_same_hits": all(r["same_hits"] for r in results if "error" not in r),
              "configs": len(results), "configs_stopped_at_stack_bound": len(failed),
              "results": results,
              "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    if out:
        Path(out).write_text(json.dumps(report, indent=1))
    return report


def launch_config(best: dict) -> tuple[int, LaunchConfig]:
    """(BVH width, LaunchConfig) of a tuner result."""
    return best["width"], LaunchConfig(block_threads=best["block_threads"],
                                       blocks_per_sm=best["blocks_per_sm"], chunk=best["chunk"],
                                       stack_depth=best["stack_depth"])
