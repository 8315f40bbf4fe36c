"""Benchmark: incoherent closest-hit Mrays/s on a 2,097,152-triangle heightfield.

Workload (one step = one pass of the closest-hit kernel over one batch):
  scene  heightfield 1024 x 1024 quads (2,097,152 triangles), y = 0.2 fBm
         (6 octaves, seeded), coordinates x1000 (the scale at which the
         reference's Cross() clamp does not act on ordinary geometry and its
         results are pinned bit-exact), FP32.
  rays   4,179,838 per step: 1,048,576 primary rays (1024 x 1024 top-down
         pinhole camera) + three cosine-weighted diffuse secondaries from
         each primary hit (3,131,262), shuffled into one incoherent batch.
  also   as many any-hit shadow rays toward a 0.1 x 0.1 light at height 2.0
         (reported as anyhit_mrays_s).

value: Mrays/s with rays and hits resident in HBM; timed with CUDA events on
the launch stream, L2 flushed (256 MiB write) between timed steps; max over
ranks; whole-job aggregate.  e2e: the same through the host-buffer C-ABI call
(enc_intersect_closest) from pinned host memory, copies inside the timed
region.  --gpus N runs N independent replicas (one process per GPU, each with
its own seeded batch, no collective on the data path).

--impl reference times the reference's own CPU Kdtree::intersect
(oracle/_ref/libencore_ref.so, compiled from the reference sources; the C
restatement in oracle/ when that library is absent) on the host cores, on a
bounded sample of the same ray mix.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE = 1000.0
RES = 1024
LIGHT = np.array([0.5, 2.0, 0.5]) * SCALE
METRIC = "Mrays/s incoherent closest-hit, 2M tris"
WORKLOAD = "heightfield1024_x1000_4M_incoherent"
CPU_SAMPLE = 65536  # rays per CPU step: 16384 primaries + 3 secondaries each


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# inputs

def make_scene(seed: int, scale: float = SCALE) -> np.ndarray:
    from encore_b200 import scenes
    return scenes.heightfield(res=RES, seed=seed, scale=scale)


def primary_rays(res: int, scale: float = SCALE) -> np.ndarray:
    from encore_b200 import scenes
    return scenes.camera_rays(res, res, eye=np.array([0.5, 1.3, 0.5]) * scale,
                              look=np.array([0.5, 0.0, 0.5]) * scale, up=(0.0, 0.0, 1.0),
                              fov_deg=40.0)


def mixed_batch(tris, prim, hits, seed: int, scale: float = SCALE) -> np.ndarray:
    """Primaries + 3 diffuse secondaries per primary hit, shuffled."""
    from encore_b200 import scenes
    sec = scenes.diffuse_rays(tris, prim, hits["tri"], hits["u"], hits["v"], per_hit=3,
                              seed=seed, offset=1e-4 * scale)
    rays = np.concatenate([prim, sec])
    perm = np.random.default_rng(seed + 1).permutation(len(rays))
    return np.ascontiguousarray(rays[perm])


def shadow_batch(tris, rays, hits, n: int, seed: int) -> np.ndarray:
    from encore_b200 import scenes
    h = hits["tri"] >= 0
    pts = scenes.hit_points(tris, rays[h], hits["tri"][h], hits["u"][h], hits["v"][h])
    reps = int(np.ceil(n / max(1, len(pts))))
    pts = np.tile(pts, (reps, 1))[:n]
    return scenes.shadow_rays(pts, seed=seed, light_center=LIGHT, light_size=0.1 * SCALE,
                              offset=0.01 * SCALE)


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    """Polls the GPU's SM clock, power and clock-event reasons through NVML
    every 2 ms from a background thread (the timed regions here last tens of
    milliseconds, below nvidia-smi's sampling period)."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[tuple] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self.err = None

    def start(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: report that instead of a number
            self.err = f"nvml unavailable: {e}"
            return
        reasons = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                   "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                   "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                   "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}

        def run():
            while not self._stop.is_set():
                try:
                    sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                    pw = N.nvmlDeviceGetPowerUsage(h) / 1000.0
                    r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, pw, [k for k, v in reasons.items() if r & v]))
                except Exception as e:
                    self.err = str(e)
                    return
                time.sleep(0.002)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self) -> dict:
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "samples": 0,
                    "reasons": [self.err or "no samples"]}
        sm = [s[0] for s in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)),
                "sm_max_mhz": self.max_mhz, "power_w_max": max(s[1] for s in self.samples),
                "samples": len(sm),
                "reasons": sorted({r for s in self.samples for r in s[2]})}


# ---------------------------------------------------------------------------
# CPU arm

def cpu_reference_rate(tris, rays_sample, steps: int = 1, warmup: int = 0):
    """Times the reference's CPU Kdtree::intersect on all host threads.
    Returns (Mrays/s over `steps` timed passes, kind, cores, build seconds)."""
    from oracle import bindings as ob
    lib = ob.reference()
    nthreads = os.cpu_count() or 1
    r6 = np.ascontiguousarray(np.concatenate([rays_sample[:, 0:3], rays_sample[:, 4:7]], axis=1))
    n = len(r6)
    tid = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    if lib is not None:
        import ctypes as C
        bs = C.c_double()
        h = lib.encref_scene_create(tris.ctypes.data, len(tris), 0, C.byref(bs))
        build_s = bs.value

        def run():
            lib.encref_closest(h, r6.ctypes.data, n, tid.ctypes.data, t.ctypes.data, None, None,
                               nthreads)
        kind = "reference"
    else:
        t0 = time.perf_counter()
        kd = ob.PortKd(tris)
        build_s = time.perf_counter() - t0

        def run():
            kd.closest(rays_sample, clamp=True, nthreads=nthreads)
        kind = "port"
    for _ in range(warmup):
        run()
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    rate = n * len(times) / sum(times) / 1e6
    return rate, kind, nthreads, build_s, times


def cpu_sample(tris, prim_res: int = 128, seed: int = 7) -> np.ndarray:
    """CPU_SAMPLE rays of the same mix: primaries of a prim_res^2 camera over
    the same view, their hits from the CPU reference path, 3 secondaries each."""
    from oracle import bindings as ob
    from encore_b200 import scenes
    prim = scenes.camera_rays(prim_res, prim_res, eye=np.array([0.5, 1.3, 0.5]) * SCALE,
                              look=np.array([0.5, 0.0, 0.5]) * SCALE, up=(0.0, 0.0, 1.0),
                              fov_deg=40.0)
    if ob.reference() is not None:
        hits, _ = ob.ref_closest(tris, prim, kind=0)
    else:
        hits = ob.PortKd(tris).closest(prim, clamp=True)
    return mixed_batch(tris, prim, hits, seed)[:CPU_SAMPLE]


def run_reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    tris = make_scene(seed=1)
    sample = cpu_sample(tris)
    rate, kind, cores, build_s, times = cpu_reference_rate(tris, sample, steps=args.steps,
                                                           warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(rate, 6), "unit": "Mrays/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_rays_per_step": int(len(sample)),
                   "accelerator": "reference Kdtree (spatial median)"},
        "cpu_baseline": {"value": round(rate, 6), "unit": "Mrays/s", "cores": cores, "kind": kind,
                         "sample": f"{len(sample)} rays of the 1:3 primary/diffuse mix per step, "
                                   f"Kdtree::intersect on {cores} host threads; build "
                                   f"{build_s:.1f} s not timed"},
        "e2e": {"value": round(rate, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm

def read_profile_traffic() -> float | None:
    p = ROOT / "profiles" / "wbvh_closest_heightfield_traffic.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("dram_bytes_per_ray:"):
            return float(ln.split(":", 1)[1])
    return None


def c0_section(dev: int, args, flush) -> dict:
    """The CPU-runnable plain case: 10,000 random triangles in the unit cube
    and one 1024 x 1024 pinhole camera ray per pixel, at unit scale as the
    workload states.  Device-resident rays, CUDA events, L2 flushed between
    steps; the reference Kdtree timed beside it on all host cores."""
    import torch
    from encore_b200 import Accelerator, scenes
    tris = scenes.random_triangles(10000, seed=0, scale=1.0)
    rays = scenes.camera_rays(1024, 1024, eye=np.array([0.5, 0.5, -1.5]),
                              look=np.array([0.5, 0.5, 0.5]))
    n = len(rays)
    acc = Accelerator("wbvh", device=dev).build(tris)
    stream = torch.cuda.current_stream()
    d_rays = torch.from_numpy(rays).to(dev)
    d_hits = torch.empty((n, 4), dtype=torch.int32, device=dev)
    for _ in range(3):
        acc.intersect_device(d_rays, n, d_hits, stream=stream)
    ms = []
    for _ in range(max(3, args.steps)):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        acc.intersect_device(d_rays, n, d_hits, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    acc.check(stream)
    rate = n * len(ms) / (sum(ms) * 1e-3) / 1e6
    # algorithmic bytes per ray from the kernel's own counts, as for the main line
    info = acc.info()
    d_vis = torch.empty((n, 2), dtype=torch.int32, device=dev)
    acc.count_visits(d_rays, n, d_vis, stream=stream)
    vis = d_vis.cpu().numpy().astype(np.int64)
    bpr = 32 + 16 + vis[:, 0].mean() * info["node_bytes"] / max(1, info["nnodes"]) + vis[:, 1].mean() * 48
    pk = ROOT / "MEASURED_PEAKS.json"
    hbm = json.loads(pk.read_text()).get("hbm_gbs", 6650.0) if pk.exists() else 6650.0
    achieved = bpr * rate * 1e6 / 1e9
    out = {"workload": "10k random triangles (unit cube), 1024x1024 primary rays, unit scale",
           "mrays_s": round(rate, 1), "ms_per_step": round(sum(ms) / len(ms), 4),
           "roofline": {"bytes_per_ray": round(float(bpr), 1), "achieved_gbs": round(achieved, 1),
                        "frac": round(achieved / hbm, 4)}}
    if not args.no_cpu:
        sub = rays[np.random.default_rng(3).choice(n, 65536, replace=False)]
        crate, kind, cores, build_s, _ = cpu_reference_rate(tris, sub, steps=1, warmup=0)
        out["cpu_baseline"] = {"value": round(crate, 4), "unit": "Mrays/s", "cores": cores,
                               "kind": kind, "sample": "65,536 of the camera rays, "
                               f"Kdtree::intersect; build {build_s:.2f} s not timed"}
    acc.destroy()
    return out


def batched_section(dev: int, args, flush) -> dict:
    """64 scenes of random triangles (log-uniform 1k-500k), one ray batch
    each (log-uniform 4k-1M, half camera, half uniform-sphere rays): every
    batch launched on its own back to back (plain) vs one persistent launch
    over all batches replayed from a CUDA graph (batched), with the launch
    shape and BVH width from the autotuner."""
    import torch
    from encore_b200 import Accelerator, scenes
    from encore_b200.autotune import autotune, launch_config
    from encore_b200.batch import BatchLaunch
    t0 = time.perf_counter()
    tris, rays = scenes.multi_scene_workload(64, seed=33, scale=SCALE)
    total = sum(len(r) for r in rays)
    tune_idx = list(range(0, 64, 4))
    rep = autotune([tris[i] for i in tune_idx], [rays[i] for i in tune_idx], widths=(4, 8),
                   chunks=(16, 32, 64), blocks_per_sm=(8, 10), block_threads=(128,), reps=3,
                   device=dev)
    width, lc = launch_config(rep["best"])
    accs8 = [Accelerator("wbvh", width=8, device=dev).build(t) for t in tris]
    accs = accs8 if width == 8 else [Accelerator("wbvh", width=width, device=dev).build(t)
                                     for t in tris]
    stream = torch.cuda.current_stream()
    d_rays = [torch.from_numpy(r).to(dev) for r in rays]
    d_plain = [torch.empty((len(r), 4), dtype=torch.int32, device=dev) for r in rays]
    d_bat = [torch.empty((len(r), 4), dtype=torch.int32, device=dev) for r in rays]
    b = BatchLaunch(list(zip(accs, d_rays, d_bat)), launch=lc)
    log(f"batched section inputs in {time.perf_counter() - t0:.1f}s: {total} rays, "
        f"{sum(len(t) for t in tris)} tris; tuned width {width} chunk {lc.chunk}")

    def plain():
        for a, r, h in zip(accs8, d_rays, d_plain):
            a.intersect_device(r, r.shape[0], h, stream=stream)

    def batched():
        b.launch_graph(stream=stream)

    out = {}
    for name, fn in (("plain", plain), ("batched", batched)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        out[name] = total * len(ts) / (sum(ts) * 1e-3) / 1e6
    b.check(stream)
    for a in accs8:
        a.check(stream)
    same = all(torch.equal(p[:, 0], q[:, 0]) for p, q in zip(d_plain, d_bat))
    b.destroy()
    for a in set(accs8) | set(accs):
        a.destroy()
    return {"workload": "64 random-triangle scenes (1k-500k tris), 4k-1M rays each, x1000",
            "rays": total, "plain_mrays_s": round(out["plain"], 1),
            "batched_mrays_s": round(out["batched"], 1),
            "batched_over_plain": round(out["batched"] / out["plain"], 3),
            "same_hits": bool(same), "tuned": rep["best"], "launches_plain": 64,
            "launches_batched": 1}


def served_section(dev: int, args) -> dict:
    """32 resident scenes (16 random-triangle scenes of 1k-2M triangles, 16
    1024x1024 heightfields with different seeds), requests of log-uniform
    16k-4M rays on a uniform-random scene, 60 % camera / 30 % diffuse
    closest-hit and 10 % shadow any-hit.  Saturation throughput of the server
    (all requests submitted at once) vs the plain per-request call run back to
    back; latency under Poisson arrivals at 60 % of the served throughput."""
    import torch
    from encore_b200 import Accelerator, scenes
    from encore_b200.serving import ANY, CLOSEST, Server
    t0 = time.perf_counter()
    rng = np.random.default_rng(44)
    tris = [scenes.random_triangles(int(np.exp(rng.uniform(np.log(1e3), np.log(2e6)))),
                                    seed=4400 + i, scale=SCALE) for i in range(16)]
    tris += [scenes.heightfield(res=RES, seed=4500 + i, scale=SCALE) for i in range(16)]
    accs = [Accelerator("wbvh", device=dev).build(t) for t in tris]
    npool = 24
    pool = []
    for j in range(npool):
        s = int(rng.integers(0, 32))
        n = int(np.exp(rng.uniform(np.log(16384), np.log(4 << 20))))
        u = rng.random()
        if u < 0.6:
            if s >= 16:  # heightfield: the top-down camera of the main workload
                cam = dict(eye=np.array([0.5, 1.3, 0.5]) * SCALE,
                           look=np.array([0.5, 0.0, 0.5]) * SCALE, up=(0.0, 0.0, 1.0),
                           fov_deg=40.0)
            else:
                cam = dict(eye=np.array([0.5, 0.5, -1.5]) * SCALE,
                           look=np.array([0.5, 0.5, 0.5]) * SCALE)
            r, k = scenes.camera_rays_jittered(n, 4600 + j, **cam), CLOSEST
        elif u < 0.9:
            r, k = scenes.surface_rays(tris[s], n, 4600 + j, "diffuse", offset=0.1,
                                       up_facing=s >= 16), CLOSEST
        else:
            r, k = scenes.surface_rays(tris[s], n, 4600 + j, "shadow", light_center=LIGHT,
                                       light_size=0.1 * SCALE, offset=0.01 * SCALE), ANY
        hr = torch.from_numpy(np.ascontiguousarray(r)).pin_memory()
        ho = torch.empty((n, 4) if k == CLOSEST else (n,), dtype=torch.int32 if k == CLOSEST
                         else torch.uint8).pin_memory()
        pool.append((s, k, n, hr, ho))
    total = sum(p[2] for p in pool)
    log(f"served section inputs in {time.perf_counter() - t0:.1f}s: {total} rays in {npool} requests")

    def out_view(p):
        from encore_b200.accel import HIT_DTYPE
        return p[4].numpy().view(HIT_DTYPE).reshape(p[2]) if p[1] == CLOSEST else p[4].numpy()

    # plain: the per-request host-buffer call, back to back; best of 3 passes
    # over the pool (host scheduling jitter only ever adds time), as for the
    # server below
    svc = None
    for rep in range(3):
        cur = []
        for p in pool:
            t1 = time.perf_counter()
            if p[1] == CLOSEST:
                accs[p[0]].intersect(p[3].numpy(), out=out_view(p))
            else:
                accs[p[0]].occluded(p[3].numpy(), out=out_view(p))
            cur.append(time.perf_counter() - t1)
        if svc is None or sum(cur) < sum(svc):
            svc = cur
    plain_rate = total / sum(svc) / 1e6
    plain_ref = [out_view(p).copy() for p in pool]

    srv = Server(device=dev, slots=args.server_slots, slot_rays=args.server_slot_rays)
    ids = [srv.add_scene(a) for a in accs]
    sat = []
    for rep in range(3):
        t1 = time.perf_counter()
        rids = [srv.submit(ids[p[0]], p[3].numpy(), p[1], out=out_view(p)) for p in pool]
        for rid in rids:
            srv.wait(rid)
        sat.append(time.perf_counter() - t1)
    served_rate = total / min(sat) / 1e6
    same = all(np.array_equal(out_view(p).view(np.uint8), ref.view(np.uint8))
               for p, ref in zip(pool, plain_ref))

    # latency under Poisson arrivals (ring of pooled requests, 3 passes)
    nreq = 3 * npool
    mean_rays = total / npool
    lam = 0.6 * served_rate * 1e6 / mean_rays  # requests per second
    gaps = rng.exponential(1.0 / lam, nreq)
    arrivals = np.cumsum(gaps)
    lat, sizes = [], []
    start = srv.now() + 0.01
    rids = [None] * nreq
    done = threading.Event()

    def submitter():
        for j in range(nreq):
            if j >= npool:  # reuse pooled buffers only after their last request finished
                while not waited[j - npool]:
                    time.sleep(0.0001)
            dt = start + arrivals[j] - srv.now()
            if dt > 0.001:
                time.sleep(dt - 0.0005)
            while srv.now() < start + arrivals[j]:
                pass
            p = pool[j % npool]
            rids[j] = srv.submit(ids[p[0]], p[3].numpy(), p[1], out=out_view(p))
        done.set()

    waited = [False] * nreq
    th = threading.Thread(target=submitter)
    th.start()
    for j in range(nreq):
        while rids[j] is None:
            time.sleep(0.00005)
        _, info = srv.wait(rids[j])
        lat.append(info["done_s"] - info["submit_s"])
        sizes.append(info["nrays"])
        waited[j] = True
    th.join()
    srv.destroy()
    # the plain per-request server under the same arrivals (FIFO, one call at a time)
    plain_lat, finish = [], 0.0
    for j in range(nreq):
        a = arrivals[j]
        finish = max(finish, a) + svc[j % npool]
        plain_lat.append(finish - a)
    lat = np.array(lat) * 1e3
    plain_lat = np.array(plain_lat) * 1e3
    sizes = np.array(sizes)
    m1 = (sizes >= (512 << 10)) & (sizes <= (2 << 20))
    for a in accs:
        a.destroy()
    return {"workload": "32 resident scenes (16 random 1k-2M tris, 16 heightfields 2.1M tris), "
                        "requests 16k-4M rays, 60/30/10 camera/diffuse/shadow, x1000",
            "requests": npool, "rays": int(total),
            "plain_mrays_s": round(plain_rate, 1), "served_mrays_s": round(served_rate, 1),
            "served_over_plain": round(served_rate / plain_rate, 3), "same_hits": bool(same),
            "poisson_offered_load": 0.6, "poisson_requests": nreq,
            "p50_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "p99_ms_1M_requests": (round(float(np.percentile(lat[m1], 99)), 3) if m1.any() else None),
            "plain_p50_ms": round(float(np.percentile(plain_lat, 50)), 3),
            "plain_p99_ms": round(float(np.percentile(plain_lat, 99)), 3),
            "copies": "host pinned buffers, copies inside every request"}


def gather_section(dev: int, args, flush) -> dict:
    """Photon mapping on the 10,000-random-triangle scene: 2M photons emitted
    from a 0.1 x 0.1 light at height 2.0 (cosine lobe, power 1/N, up to 3
    diffuse bounces, Russian roulette at albedo 0.7) traced on the GPU, one
    photon map, then a k = 50, r = 0.02 radiance gather at 1M primary-hit
    points (x1000 scale: r = 20)."""
    import torch
    from encore_b200 import Accelerator, scenes, wavefront
    from oracle import bindings as ob
    t0 = time.perf_counter()
    tris = scenes.random_triangles(10000, seed=0, scale=SCALE)
    acc = Accelerator("wbvh", device=dev).build(tris)
    nph, cap = 2_000_000, 8_000_000
    bufs = [torch.empty((cap, 3), dtype=torch.float32, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    # one untimed pass first: the call's wave buffers are allocated per call,
    # and the first allocation after the earlier sections maps fresh memory
    for rep in range(2):
        t1 = time.perf_counter()
        m = wavefront.trace_photons(acc, LIGHT, 0.1 * SCALE, nph, *bufs, max_bounces=3,
                                    albedo=0.7, seed=7, emit_offset=0.01 * SCALE,
                                    bounce_offset=0.001 * SCALE)
        trace_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    pm = wavefront.photon_map_from_device(bufs[0], bufs[1], bufs[2], m, device=dev)
    build_s = time.perf_counter() - t1
    side = 1536
    d_rays = torch.empty((side * side, 8), dtype=torch.float32, device=dev)
    wavefront.camera_rays(np.array([0.5, 0.5, -1.5]) * SCALE, np.array([0.5, 0.5, 0.5]) * SCALE,
                          (0.0, 1.0, 0.0), 45.0, side, side, d_rays)
    d_hits = torch.empty((side * side, 4), dtype=torch.int32, device=dev)
    acc.intersect_device(d_rays, side * side, d_hits)
    d_p = torch.empty((side * side, 3), dtype=torch.float32, device=dev)
    d_n = torch.empty((side * side, 3), dtype=torch.float32, device=dev)
    wavefront.hit_surface(acc, d_hits, side * side, d_p, d_n)
    ok = d_hits[:, 0] >= 0
    q = d_p[ok][: 1 << 20].contiguous()
    qn = d_n[ok][: 1 << 20].contiguous()
    nq = q.shape[0]
    d_rgb = torch.empty((nq, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    k, r = 50, 0.02 * SCALE
    for _ in range(3):
        pm.get_radiance_estimate_device(k, r, q, qn, nq, d_rgb, stream=stream.cuda_stream)
    ts = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pm.get_radiance_estimate_device(k, r, q, qn, nq, d_rgb, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    rate = nq * len(ts) / (sum(ts) * 1e-3) / 1e6
    # parity sample against the FP64 oracle on the same photons
    pos, nrm, pw = (b[:m].cpu().numpy() for b in bufs)
    sel = np.linspace(0, nq - 1, 2000).astype(int)
    qs, qns = q.cpu().numpy()[sel], qn.cpu().numpy()[sel]
    want, cnt = ob.port_gather(pos, nrm, pw, qs, qns, k, r)
    got = d_rgb.cpu().numpy()[sel]
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-30)
    cpu = None
    if not args.no_cpu and ob.reference() is not None:
        import ctypes as C
        lib = ob.reference()
        bs = C.c_double()
        h = lib.encref_pmap_create(pos.ctypes.data, nrm.ctypes.data, pw.ctypes.data, m, 0,
                                   C.byref(bs))
        out = np.empty((len(qs), 3), np.float32)
        nt = os.cpu_count() or 1
        t1 = time.perf_counter()
        lib.encref_pmap_radiance(h, np.ascontiguousarray(qs).ctypes.data,
                                 np.ascontiguousarray(qns).ctypes.data, len(qs), k, r,
                                 out.ctypes.data, nt)
        cpu_s = time.perf_counter() - t1
        lib.encref_pmap_destroy(h)
        cpu = {"value": round(len(qs) / cpu_s / 1e6, 6), "unit": "Mqueries/s", "cores": nt,
               "kind": "reference", "build_seconds": round(bs.value, 2),
               "sample": f"{len(qs)} of the same queries, PhotonMap::GetRadianceEstimate"}
        ref_rel = np.abs(got - out) / np.maximum(np.abs(out), 1e-30)
        cpu["max_rel_err_vs_reference"] = float(ref_rel.max())
    pm._destroy()
    acc.destroy()
    log(f"gather section in {time.perf_counter() - t0:.1f}s: {m} photons stored, {nq} queries")
    return {"workload": "10k random triangles x1000, 2M photons (<=3 bounces, RR 0.7), "
                        "k=50 r=0.02 (x1000) at primary hits",
            "photons_emitted": nph, "photons_stored": int(m),
            "photon_trace_ms": round(trace_s * 1e3, 2), "photon_map_build_s": round(build_s, 3),
            "queries": int(nq), "mqueries_s": round(rate, 2),
            "ms_per_gather": round(sum(ts) / len(ts), 3),
            "found_mean": float(cnt.mean()),
            "max_rel_err_vs_fp64": float(rel.max()), "cpu_baseline": cpu}


def run_engine_arm(args, rank: int, world: int) -> None:
    import torch
    import torch.distributed as dist
    from encore_b200 import Accelerator, HIT_DTYPE, LaunchConfig, replicas

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", dev),
                                timeout=__import__("datetime").timedelta(seconds=600))

    seed = 1 + rank
    t0 = time.perf_counter()
    tris = make_scene(seed=1)  # every replica serves the same scene
    prim = primary_rays(RES)
    acc = Accelerator("wbvh", width=args.width, max_leaf_tris=args.leaf, device=dev).build(tris)
    info = acc.info()
    launch = LaunchConfig(block_threads=args.block, blocks_per_sm=args.bps, chunk=args.chunk,
                          stack_depth=args.stack)
    ph = acc.intersect(prim)
    rays = mixed_batch(tris, prim, ph, seed=100 + seed)
    n = len(rays)
    hits_ref = acc.intersect(rays)
    shadow = shadow_batch(tris, rays, hits_ref, n, seed=200 + seed)
    log(f"[rank {rank}] inputs ready in {time.perf_counter() - t0:.1f}s: {n} rays, "
        f"{info['ntris']} tris, {info['nnodes']} nodes, build {info['build_seconds']:.2f}s")

    stream = torch.cuda.current_stream()
    d_rays = torch.from_numpy(rays).to(dev)
    d_hits = torch.empty((n, 4), dtype=torch.int32, device=dev)
    d_shadow = torch.from_numpy(shadow).to(dev)
    d_occ = torch.empty(n, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def closest():
        acc.intersect_device(d_rays, n, d_hits, launch=launch, stream=stream)

    def anyhit():
        acc.occluded_device(d_shadow, n, d_occ, launch=launch, stream=stream)

    def timed(fn, steps):
        evs = []
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    for _ in range(args.warmup):
        closest()
        anyhit()
    acc.check(stream)
    clocks = ClockSampler(dev)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms = timed(closest, args.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    acc.check(stream)
    ms_any = timed(anyhit, args.steps)
    acc.check(stream)

    # whole-job rate: every replica's rays over the slowest replica's device time
    rate, total_ms = replicas.aggregate_rate(n, args.steps, sum(ms))
    any_rate, _ = replicas.aggregate_rate(n, args.steps, sum(ms_any))
    ms_step = total_ms / args.steps
    value = rate / 1e6
    any_value = any_rate / 1e6

    # parity spot check of the timed output against the untimed host-form call
    got = d_hits.cpu().numpy()
    assert np.array_equal(got[:, 0], hits_ref["tri"]), "timed kernel output differs"

    # the kd-tree parity mode (the reference Kdtree's own cells and order,
    # bit-exact with it) on the same batch, for scale against the wide BVH
    kd_value = None
    if not args.no_extras:
        t_kd = time.perf_counter()
        kd = Accelerator("kdtree", device=dev).build(tris)
        kd_build_s = time.perf_counter() - t_kd

        def kd_closest():
            kd.intersect_device(d_rays, n, d_hits, launch=None, stream=stream)

        for _ in range(2):
            kd_closest()
        ms_kd = timed(kd_closest, max(1, args.steps // 4))
        kd.check(stream)
        kd_rate, _ = replicas.aggregate_rate(n, len(ms_kd), sum(ms_kd))
        kd_value = {"mrays_s": round(kd_rate / 1e6, 3), "build_seconds": round(kd_build_s, 2)}
        kd.destroy()

    # algorithmic bytes per ray from the engine's own traversal counts
    d_vis = torch.empty((n, 2), dtype=torch.int32, device=dev)
    acc.count_visits(d_rays, n, d_vis, stream=stream)
    vis = d_vis.cpu().numpy().astype(np.int64)
    node_b = info["node_bytes"] / max(1, info["nnodes"])
    nodes_per_ray = vis[:, 0].mean()
    tris_per_ray = vis[:, 1].mean()
    bytes_per_ray = 32 + 16 + nodes_per_ray * node_b + tris_per_ray * 48
    launch_s = ms_step * 1e-3
    achieved = bytes_per_ray * n / launch_s / 1e9
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dram_per_ray = read_profile_traffic()

    # e2e: host-buffer C-ABI call, pinned buffers, copies inside the timed region
    h_rays = torch.from_numpy(rays).pin_memory()
    h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory()
    h_rays_np = h_rays.numpy()
    h_hits_np = h_hits.numpy().view(HIT_DTYPE).reshape(n)
    for _ in range(min(2, args.warmup)):
        acc.intersect(h_rays_np, launch=launch, stream=stream, out=h_hits_np)
    if world > 1:
        dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        acc.intersect(h_rays_np, launch=launch, stream=stream, out=h_hits_np)
        e2e_ms.append((time.perf_counter() - t1) * 1e3)
    e2e_rate, _ = replicas.aggregate_rate(n, args.steps, sum(e2e_ms))
    e2e_value = e2e_rate / 1e6
    assert np.array_equal(h_hits_np["tri"], hits_ref["tri"])

    cpu = None
    if rank == 0 and not args.no_cpu:
        sample = cpu_sample(tris)
        rate, kind, cores, build_s, _ = cpu_reference_rate(tris, sample, steps=1, warmup=0)
        cpu = {"value": round(rate, 6), "unit": "Mrays/s", "cores": cores, "kind": kind,
               "sample": f"{len(sample)} rays of the same 1:3 primary/diffuse mix (16384 "
                         f"primaries of a 128x128 camera + 3 secondaries each), reference "
                         f"Kdtree::intersect on {cores} host threads; Kdtree build "
                         f"{build_s:.1f} s not timed"}

    acc.destroy()
    del d_rays, d_hits, d_shadow, d_occ, h_rays, h_hits
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        torch.cuda.empty_cache()
        extras["plain_c0"] = c0_section(dev, args, flush)
        torch.cuda.empty_cache()
        extras["batched"] = batched_section(dev, args, flush)
        torch.cuda.empty_cache()
        extras["served"] = served_section(dev, args)
        torch.cuda.empty_cache()
        extras["photon_gather"] = gather_section(dev, args, flush)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded fBm heightfield, pinhole + cosine-diffuse rays)",
            "config": {"workload": WORKLOAD, "triangles": int(info["ntris"]),
                       "rays_per_step": n, "scale": SCALE, "accelerator":
                       f"wbvh{info['width']} quantised 8-bit, leaf<={args.leaf}",
                       "l2": "flushed (256 MiB write) between timed steps",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "peak_source": peak_src,
                         "traffic": (round(dram_per_ray * n) if dram_per_ray else None),
                         "bytes_per_ray": round(bytes_per_ray, 1),
                         "nodes_per_ray": round(float(nodes_per_ray), 2),
                         "tris_per_ray": round(float(tris_per_ray), 2)},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(rays.nbytes), "d2h_bytes_per_step": int(n * 16)},
            "anyhit_mrays_s": round(any_value, 3),
            "kdtree_mode": kd_value,
            "build_seconds": round(info["build_seconds"], 3),
            "clocks": clk,
            "cpu_baseline": cpu,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--width", type=int, default=8)
    ap.add_argument("--leaf", type=int, default=3)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--bps", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--stack", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched multi-scene, served and photon-gather sections")
    ap.add_argument("--server-slots", type=int, default=6,
                    help="served section: request slots (rounds in flight)")
    ap.add_argument("--server-slot-rays", type=int, default=4 << 20,
                    help="served section: ray capacity of a slot (>= the largest request, 4M)")
    ap.add_argument("--served-only", action="store_true",
                    help="run only the served section (prints its JSON object)")
    ap.add_argument("--gather-only", action="store_true",
                    help="run only the photon-gather section (prints its JSON object)")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warm-up below 3 steps is not a valid measurement; using 3")
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.served_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(served_section(0, args)), flush=True)
    elif args.gather_only:
        import torch
        torch.cuda.set_device(0)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=0)
        print(json.dumps(gather_section(0, args, flush)), flush=True)
    elif args.impl == "reference":
        run_reference_arm(args, rank, world)
    else:
        run_engine_arm(args, rank, world)


if __name__ == "__main__":
    main()
