"""Multi-scene batched launch (GPU): the same hits as tracing every batch on
its own, bit for bit, whatever the batch sizes, launch shape or graph replay."""
import numpy as np
import pytest

from encore_b200 import Accelerator, EncoreError, LaunchConfig, scenes
from encore_b200.autotune import autotune
from encore_b200.batch import BatchLaunch

pytestmark = pytest.mark.gpu


def _mix(nscenes=9, seed=3):
    tris, rays = scenes.multi_scene_workload(nscenes, seed=seed, scale=1000.0,
                                             tri_range=(200, 20000), ray_range=(1, 30000))
    rays[0] = rays[0][:1]     # a one-ray batch
    rays[1] = rays[1][:0]     # an empty batch
    rays[2] = rays[2][:33]    # just past one chunk
    return tris, rays


def _device(rays):
    import torch
    d_rays = [torch.from_numpy(np.ascontiguousarray(r)).cuda() for r in rays]
    d_hits = [torch.full((r.shape[0], 4), -7, dtype=torch.int32, device="cuda") for r in rays]
    return d_rays, d_hits


def test_batched_equals_per_batch(gpu):
    tris, rays = _mix()
    accs = [Accelerator("wbvh").build(t) for t in tris]
    want = [a.intersect(r) for a, r in zip(accs, rays)]
    d_rays, d_hits = _device(rays)
    b = BatchLaunch(list(zip(accs, d_rays, d_hits)))
    b.launch()
    b.check()
    for w, h in zip(want, d_hits):
        got = h.cpu().numpy()
        assert np.array_equal(got[:, 0], w["tri"])
        assert np.array_equal(got[:, 1], np.where(w["tri"] >= 0, w["t"].view(np.int32), 0))
    # replay from a CUDA graph, twice, after clearing the outputs
    for _ in range(2):
        for h in d_hits:
            h.fill_(-7)
        b.launch_graph()
        b.check()
        for w, h in zip(want, d_hits):
            assert np.array_equal(h.cpu().numpy()[:, 0], w["tri"])


def test_batched_same_scene_many_batches_and_launch_shapes(gpu):
    tris, rays = _mix(nscenes=5, seed=4)
    acc = Accelerator("wbvh").build(tris[3])
    want = [acc.intersect(r) for r in rays]
    d_rays, d_hits = _device(rays)
    for lc in (LaunchConfig(chunk=1), LaunchConfig(chunk=16, blocks_per_sm=2, block_threads=64),
               LaunchConfig(chunk=128)):
        for h in d_hits:
            h.fill_(-7)
        b = BatchLaunch([(acc, r, h) for r, h in zip(d_rays, d_hits)], launch=lc)
        b.launch_graph()
        b.check()
        for w, h in zip(want, d_hits):
            assert np.array_equal(h.cpu().numpy()[:, 0], w["tri"])
        b.destroy()


def test_batched_rejects_mixed_widths(gpu):
    tris, rays = _mix(nscenes=3)
    a8 = Accelerator("wbvh", width=8).build(tris[0])
    a4 = Accelerator("wbvh", width=4).build(tris[1])
    d_rays, d_hits = _device(rays[:2])
    with pytest.raises(EncoreError):
        BatchLaunch([(a8, d_rays[0], d_hits[0]), (a4, d_rays[1], d_hits[1])])


def test_autotuner_picks_a_config_with_identical_hits(gpu):
    tris, rays = scenes.multi_scene_workload(6, seed=5, scale=1000.0, tri_range=(500, 5000),
                                             ray_range=(1000, 20000))
    rep = autotune(tris, rays, widths=(4, 8), chunks=(16, 64), blocks_per_sm=(8,),
                   block_threads=(128,), reps=2)
    assert rep["all_same_hits"]
    assert rep["best"] is not None and rep["best"]["mrays_s"] > 0
    assert len(rep["results"]) == 4
