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

value: Mrays/s with rays and hits resident in HBM; one step = one
closest-hit launch over the batch (enc_intersect_closest_device); timed
with CUDA events on the launch stream, L2 flushed (256 MiB write) between
timed steps; max over ranks; whole-job aggregate.  --bin adds the binning
pass (enc_bin_rays, a counting sort of the batch by origin and direction
cell) to every step and traces the binned order
(enc_intersect_closest_device_ordered).  e2e: the same metric through the host-buffer
C-ABI call on the reference's Ray payload (enc_intersect_closest_od: origin and
direction, 24 bytes per ray) from pinned host memory, copies inside the timed
region; the 8-float call (enc_intersect_closest) is reported beside it.  --gpus N runs N independent replicas (one process per
GPU, each with its own seeded batch, no collective on the data path).

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
CPU_SAMPLE = 65536  # rays per CPU step, drawn from the bench batch


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


def cpu_sample(tris, batch: np.ndarray | None = None, seed: int = 7) -> np.ndarray:
    """CPU_SAMPLE rays drawn (seeded, without replacement) from the bench's
    own 4,179,838-ray batch.  Without `batch` (the reference arm, which runs
    no engine code) the batch is rebuilt the same way with the primaries'
    hits from the reference's Kdtree instead of the engine's."""
    from oracle import bindings as ob
    if batch is None:
        prim = primary_rays(RES)
        if ob.reference() is not None:
            hits, _ = ob.ref_closest(tris, prim, kind=0)
        else:
            hits = ob.PortKd(tris).closest(prim, clamp=True)
        batch = mixed_batch(tris, prim, hits, seed=101)
    sel = np.sort(np.random.default_rng(seed).choice(len(batch), CPU_SAMPLE, replace=False))
    return np.ascontiguousarray(batch[sel])


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
                         "sample": f"{len(sample)} rays per step drawn at random from the "
                                   f"4,179,838-ray batch (primaries' hits from the reference's "
                                   f"own Kdtree), Kdtree::intersect on {cores} host threads; "
                                   f"build {build_s:.1f} s not timed"},
        "e2e": {"value": round(rate, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm

TRAFFIC_PROFILE = "profiles/wbvh_closest_heightfield_traffic.txt"


def read_profile_traffic() -> dict:
    """Per-ray DRAM and L2 figures of the closest-hit launch from the
    committed ncu summary (keys: dram_bytes_per_ray, l2_bytes_per_ray,
    l2_pct_of_peak, binned)."""
    p = ROOT / TRAFFIC_PROFILE
    out = {}
    if not p.exists():
        return out
    for ln in p.read_text().splitlines():
        if ":" in ln and not ln.startswith("#"):
            k, v = ln.split(":", 1)
            try:
                out[k.strip()] = float(v)
            except ValueError:
                pass
    return out


MISMATCH_FIXTURE = "tests/golden/fullsize_mismatches.npz"


def parity_vs_kd(got: np.ndarray, kd: np.ndarray) -> dict:
    """Rays of the bench batch whose closest-hit triangle differs between the
    engine and the kd-tree parity mode (the reference Kdtree's own walk,
    bit-exact with Kdtree::intersect), checked against the committed,
    classified list of those rays (tests/golden/make_fullsize_mismatches.py
    made it and classified each ray with the oracle).  got, kd: (n, 4) int32
    hit records."""
    mism = np.nonzero(got[:, 0] != kd[:, 0])[0]
    same = got[:, 0] == kd[:, 0]
    out = {"vs": "reference Kdtree walk (kd-tree parity mode, bit-exact with Kdtree::intersect)",
           "rays": int(len(got)), "mismatches": int(len(mism)),
           "t_bits_equal_where_ids_agree": bool(np.array_equal(got[same, 1], kd[same, 1]))}
    fx = ROOT / MISMATCH_FIXTURE
    if not fx.exists():
        out["mismatch_by_class"] = None
        return out
    g = np.load(fx)
    idx, cls, names = g["x1000_idx"], g["x1000_cls"], g["classes"]
    listed = (np.array_equal(mism, idx) and np.array_equal(got[mism, 0], g["x1000_got"]["tri"])
              and np.array_equal(kd[mism, 0], g["x1000_want"]["tri"]))
    known = np.isin(mism, idx)
    pos = np.searchsorted(idx, mism[known])
    counts = {}
    for k in cls[pos]:
        counts[str(names[k])] = counts.get(str(names[k]), 0) + 1
    out.update({"matches_committed_list": bool(listed), "mismatch_by_class": counts,
                "unlisted": int((~known).sum()), "list": MISMATCH_FIXTURE})
    return out


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
    rep = autotune([tris[i] for i in tune_idx], [rays[i] for i in tune_idx], widths=(2, 4, 8),
                   chunks=(16, 32, 64), blocks_per_sm=(8, 10), block_threads=(64, 128),
                   stack_depths=(0, 16, 24), reps=3, device=dev, out=args.tune_table)
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
            "same_hits": bool(same), "tuned": rep["best"],
            "tuner": {"configs": rep["configs"], "stopped_at_stack_bound":
                      rep["configs_stopped_at_stack_bound"], "all_same_hits": rep["all_same_hits"],
                      "space": "width 2/4/8 x chunk 16/32/64 x blocks/SM 8/10 x block 64/128 x "
                               "stack 0 (tree depth)/16/24"},
            "launches_plain": 64, "launches_batched": 1}


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

    # latency under Poisson arrivals (the pooled requests reused as a ring)
    nreq = max(args.served_requests, npool)
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
    m1 = (sizes >= (512 << 10)) & (sizes <= (2 << 20))  # "1M-ray requests": 0.5M-2M rays
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
            "n_1M_requests": int(m1.sum()),
            "1M_requests": "requests of 524,288 to 2,097,152 rays",
            "max_ms": round(float(lat.max()), 3),
            "plain_p50_ms": round(float(np.percentile(plain_lat, 50)), 3),
            "plain_p99_ms": round(float(np.percentile(plain_lat, 99)), 3),
            "copies": "host pinned buffers, copies inside every request"}


def _gather_variant(dev: int, args, flush, pm, pos, nrm, pw, q, qn, k, r, label) -> dict:
    """Times one radiance gather over `pm` (a built photon map) at queries
    q/qn (device), counts the per-query work for the roofline, checks a
    sample against the FP64 oracle and times the reference's
    GetRadianceEstimate on the same sample."""
    import torch
    from oracle import bindings as ob
    nq = q.shape[0]
    stream = torch.cuda.current_stream()
    d_rgb = torch.empty((nq, 3), dtype=torch.float32, device=dev)
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
    pm.check(stream.cuda_stream)
    ms = sum(ts) / len(ts)
    rate = nq / (ms * 1e-3) / 1e6
    # algorithmic bytes per query from the kernel's own counts: query position
    # and normal in (24), rgb out (12), 24 per child box tested, 16 per
    # photon position tested, 16 per normal read, 16 per found photon's power
    d_vis = torch.empty((nq, 4), dtype=torch.int32, device=dev)
    d_rgb2 = torch.empty((nq, 3), dtype=torch.float32, device=dev)
    pm.count_visits(k, r, q, qn, nq, d_rgb2, d_vis, stream=stream.cuda_stream)
    vis = d_vis.cpu().numpy().astype(np.float64).mean(axis=0)
    same = bool(torch.equal(d_rgb, d_rgb2))
    bpq = 24 + 12 + 24 * vis[0] + 16 * vis[1] + 16 * vis[2] + 16 * vis[3]
    achieved = bpq * nq / (ms * 1e-3) / 1e9
    pk = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(pk.read_text()) if pk.exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
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
        m = len(pos)
        h = lib.encref_pmap_create(pos.ctypes.data, nrm.ctypes.data, pw.ctypes.data, m, 0,
                                   C.byref(bs))
        out = np.empty((len(qs), 3), np.float32)
        nt = os.cpu_count() or 1
        cpu_ts = []
        for _ in range(3):
            t1 = time.perf_counter()
            lib.encref_pmap_radiance(h, np.ascontiguousarray(qs).ctypes.data,
                                     np.ascontiguousarray(qns).ctypes.data, len(qs), k, r,
                                     out.ctypes.data, nt)
            cpu_ts.append(time.perf_counter() - t1)
        lib.encref_pmap_destroy(h)
        cpu = {"value": round(len(qs) / (sum(cpu_ts) / 3) / 1e6, 6), "unit": "Mqueries/s",
               "cores": nt, "kind": "reference", "build_seconds": round(bs.value, 2),
               "sample": f"{len(qs)} of the same queries, PhotonMap::GetRadianceEstimate, "
                         "mean of 3 passes"}
        ref_rel = np.abs(got - out) / np.maximum(np.abs(out), 1e-30)
        cpu["max_rel_err_vs_reference"] = float(ref_rel.max())
    return {"map": label, "photons": int(len(pos)),
            "map_bytes": int(len(pos)) * 48, "queries": int(nq), "mqueries_s": round(rate, 2),
            "ms_per_gather": round(ms, 3), "found_mean": float(cnt.mean()),
            "max_rel_err_vs_fp64": float(rel.max()),
            "roofline": {"bound": "hbm", "kernel": "gather_kernel", "achieved": round(achieved, 1),
                         "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "bytes_per_query": round(float(bpq), 1),
                         "per_query": {"boxes_tested": round(float(vis[0]), 2),
                                       "photons_tested": round(float(vis[1]), 2),
                                       "normals_read": round(float(vis[2]), 2),
                                       "found": round(float(vis[3]), 2)},
                         "counting_launch_same_rgb": same},
            "cpu_baseline": cpu}


def gather_section(dev: int, args, flush) -> dict:
    """Photon mapping on the 10,000-random-triangle scene (x1000): photons
    emitted from a 0.1 x 0.1 light at height 2.0 (cosine lobe, up to 3
    diffuse bounces, Russian roulette at albedo 0.7) and traced on the GPU,
    then a k = 50, r = 0.02 (x1000: 20) radiance gather at 1M primary-hit
    points, on two maps:
      l2_resident  one map of every stored photon of 2M emitted (about 0.5M
                   photons, 25 MB: it stays in the 126 MB L2);
      large        the reference's indirect map, filled as EmitPhotons fills
                   it (batches of 2M emitted until 4M indirect photons are
                   stored; 192 MB, above L2), beside its direct map."""
    import torch
    from encore_b200 import Accelerator, scenes, wavefront
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
    k, r = 50, 0.02 * SCALE
    pos, nrm, pw = (b[:m].cpu().numpy() for b in bufs)
    small = _gather_variant(dev, args, flush, pm, pos, nrm, pw, q, qn, k, r,
                            "every stored photon of 2M emitted (one map)")
    small.update({"photons_emitted": nph, "photon_trace_ms": round(trace_s * 1e3, 2),
                  "photon_map_build_s": round(build_s, 3)})
    pm._destroy()
    del bufs
    torch.cuda.empty_cache()
    # the large map: EmitPhotons' loop until the indirect map is full
    cap_i, cap_d = 4_000_000, 16_000_000
    ind = tuple(torch.empty((cap_i, 3), dtype=torch.float32, device=dev) for _ in range(3)) + (None,)
    dirm = tuple(torch.empty((cap_d, 3), dtype=torch.float32, device=dev) for _ in range(3)) + (None,)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    nd, ni, emitted = wavefront.trace_photon_maps(
        acc, LIGHT, 0.1 * SCALE, nph, dirm, ind, max_bounces=3, albedo=0.7, seed=8,
        emit_offset=0.01 * SCALE, bounce_offset=0.001 * SCALE, shadow_offset=2.0 * SCALE,
        fill_indirect=True)
    fill_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    pmi = wavefront.photon_map_from_device(ind[0], ind[1], ind[2], ni, device=dev)
    build_i = time.perf_counter() - t1
    posi, nrmi, pwi = (b[:ni].cpu().numpy() for b in ind[:3])
    large = _gather_variant(dev, args, flush, pmi, posi, nrmi, pwi, q, qn, k, r,
                            "indirect map filled to 4M photons (EmitPhotons' loop)")
    large.update({"photons_emitted": int(emitted), "direct_map_photons": int(nd),
                  "indirect_map_photons": int(ni), "photon_trace_ms": round(fill_s * 1e3, 1),
                  "photon_map_build_s": round(build_i, 3)})
    pmi._destroy()
    acc.destroy()
    log(f"gather section in {time.perf_counter() - t0:.1f}s: {m} / {ni} photons, {q.shape[0]} queries")
    return {"workload": "10k random triangles x1000, photons traced on the GPU (<=3 bounces, "
                        "RR 0.7), k=50 r=0.02 (x1000) at 1M primary hits",
            "mqueries_s": small["mqueries_s"], "l2_resident": small, "large": large}


def run_engine_arm(args, rank: int, world: int) -> None:
    import torch
    import torch.distributed as dist
    from encore_b200 import Accelerator, BinConfig, HIT_DTYPE, LaunchConfig, replicas

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
    binning = BinConfig(args.bin_origin, args.bin_dir, args.bin_probe) if args.bin else None
    scratch = (torch.empty(acc.bin_scratch_bytes(n, binning), dtype=torch.uint8, device=dev)
               if binning else None)

    def closest(mid=None):
        """One step: bin the batch, then trace it in the binned order (mid:
        an event recorded between the two, so the traversal launch alone is
        timed too)."""
        if binning is None:
            if mid is not None:
                mid.record(stream)
            acc.intersect_device(d_rays, n, d_hits, launch=launch, stream=stream)
            return
        order = acc.bin_rays(d_rays, n, scratch, binning, stream=stream)
        if mid is not None:
            mid.record(stream)
        acc.intersect_device_ordered(d_rays, n, order, d_hits, launch=launch, stream=stream)

    def anyhit(mid=None):
        if mid is not None:
            mid.record(stream)
        acc.occluded_device(d_shadow, n, d_occ, launch=launch, stream=stream)

    def timed(fn, steps):
        """Per step (whole step ms, traversal launch ms), CUDA events on the
        launch stream, L2 flushed before each step."""
        evs = []
        for _ in range(steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            m = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn(m)
            b.record(stream)
            evs.append((a, m, b))
        torch.cuda.synchronize()
        return ([a.elapsed_time(b) for a, m, b in evs], [m.elapsed_time(b) for a, m, b in evs])

    for _ in range(args.warmup):
        closest()
        anyhit()
    acc.check(stream)
    clocks = ClockSampler(dev)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms, ms_trace = timed(closest, args.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    acc.check(stream)
    ms_any, _ = timed(anyhit, args.steps)
    acc.check(stream)

    # whole-job rate: every replica's rays over the slowest replica's device time
    rate, total_ms = replicas.aggregate_rate(n, args.steps, sum(ms))
    any_rate, _ = replicas.aggregate_rate(n, args.steps, sum(ms_any))
    _, trace_total_ms = replicas.aggregate_rate(n, args.steps, sum(ms_trace))
    ms_step = total_ms / args.steps
    ms_trace_step = trace_total_ms / args.steps
    value = rate / 1e6
    any_value = any_rate / 1e6

    # parity spot check of the timed output against the untimed host-form call
    got = d_hits.cpu().numpy()
    assert np.array_equal(got[:, 0], hits_ref["tri"]), "timed kernel output differs"

    # the kd-tree parity mode (the reference Kdtree's own cells and order,
    # bit-exact with it) on the same batch, for scale against the wide BVH,
    # and the list of rays whose triangle differs between the two
    kd_value = None
    parity = None
    if not args.no_extras:
        t_kd = time.perf_counter()
        kd = Accelerator("kdtree", device=dev).build(tris)
        kd_build_s = time.perf_counter() - t_kd

        def kd_closest(mid=None):
            if mid is not None:
                mid.record(stream)
            kd.intersect_device(d_rays, n, d_hits, launch=None, stream=stream)

        for _ in range(2):
            kd_closest()
        ms_kd, _ = timed(kd_closest, max(1, args.steps // 4))
        kd.check(stream)
        kd_rate, _ = replicas.aggregate_rate(n, len(ms_kd), sum(ms_kd))
        kd_hits = d_hits.cpu().numpy().view(np.int32)
        # the same walk over the binned order (coherent warps), same hits
        kd_scratch = torch.empty(kd.bin_scratch_bytes(n), dtype=torch.uint8, device=dev)

        def kd_binned(mid=None):
            if mid is not None:
                mid.record(stream)
            kd.intersect_device_binned(d_rays, n, d_hits, kd_scratch, stream=stream)

        kd_binned()
        ms_kdb, _ = timed(kd_binned, max(1, args.steps // 4))
        kd.check(stream)
        kdb_rate, _ = replicas.aggregate_rate(n, len(ms_kdb), sum(ms_kdb))
        kd_same = bool(np.array_equal(d_hits.cpu().numpy().view(np.int32), kd_hits))
        kd_value = {"mrays_s": round(kd_rate / 1e6, 3), "mrays_s_binned": round(kdb_rate / 1e6, 3),
                    "binned_same_hits": kd_same, "build_seconds": round(kd_build_s, 2)}
        del kd_scratch
        kd.destroy()
        if rank == 0:
            parity = parity_vs_kd(got, kd_hits)

    # algorithmic bytes per ray from the engine's own traversal counts
    d_vis = torch.empty((n, 2), dtype=torch.int32, device=dev)
    acc.count_visits(d_rays, n, d_vis, stream=stream)
    vis = d_vis.cpu().numpy().astype(np.int64)
    node_b = info["node_bytes"] / max(1, info["nnodes"])
    nodes_per_ray = vis[:, 0].mean()
    tris_per_ray = vis[:, 1].mean()
    bytes_per_ray = 32 + 16 + nodes_per_ray * node_b + tris_per_ray * 48
    launch_s = ms_trace_step * 1e-3  # the traversal launch alone
    achieved = bytes_per_ray * n / launch_s / 1e9
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    prof = read_profile_traffic()
    dram_per_ray = prof.get("dram_bytes_per_ray")
    bin_ms = ms_step - ms_trace_step
    # binning: ray read (32) + key write (4) + key read (4) + order write (4)
    bin_bytes = 44 * n

    # e2e: host-buffer C-ABI calls, pinned buffers, copies inside the timed
    # region.  The headline takes the reference's Ray payload (origin and
    # direction, 24 bytes per ray: enc_intersect_closest_od; every ray of the
    # batch has tmin = 0 and tmax = +inf, the reference's own bounds); the
    # 8-float form (enc_intersect_closest, 32 bytes per ray) is reported beside it.
    h_rays = torch.from_numpy(rays).pin_memory()
    rays_od = np.ascontiguousarray(np.concatenate([rays[:, 0:3], rays[:, 4:7]], axis=1))
    assert (rays[:, 3] == 0).all() and np.isinf(rays[:, 7]).all()
    h_od = torch.from_numpy(rays_od).pin_memory()
    h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory()
    h_rays_np = h_rays.numpy()
    h_od_np = h_od.numpy()
    h_hits_np = h_hits.numpy().view(HIT_DTYPE).reshape(n)

    def e2e_run(call, src) -> float:
        for _ in range(min(2, args.warmup)):
            call(src, launch=launch, stream=stream, out=h_hits_np)
        if world > 1:
            dist.barrier()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            call(src, launch=launch, stream=stream, out=h_hits_np)
            ms.append((time.perf_counter() - t1) * 1e3)
        assert np.array_equal(h_hits_np.view(np.uint8), hits_ref.view(np.uint8))
        rate, _ = replicas.aggregate_rate(n, args.steps, sum(ms))
        return rate / 1e6

    e2e8_value = e2e_run(acc.intersect, h_rays_np)
    e2e_value = e2e_run(acc.intersect_od, h_od_np)

    cpu = None
    if rank == 0 and not args.no_cpu:
        sample = cpu_sample(tris, rays)
        rate, kind, cores, build_s, _ = cpu_reference_rate(tris, sample, steps=3, warmup=1)
        cpu = {"value": round(rate, 6), "unit": "Mrays/s", "cores": cores, "kind": kind,
               "sample": f"{len(sample)} rays drawn at random from the timed {n}-ray batch, "
                         f"reference Kdtree::intersect on {cores} host threads, mean of 3 passes "
                         f"after 1 untimed; Kdtree build {build_s:.1f} s not timed"}

    acc.destroy()
    del d_rays, d_hits, d_shadow, d_occ, h_rays, h_od, h_hits
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
            "gpu_launches": args.steps * (1 if binning is None else 4),
            "roofline": {"bound": "hbm", "kernel": "wbvh_trace (closest hit)",
                         "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "peak_source": peak_src,
                         "launch_ms": round(ms_trace_step, 4),
                         "traffic": (round(dram_per_ray * n) if dram_per_ray else None),
                         "traffic_source": (f"{TRAFFIC_PROFILE} (ncu capture, per ray x rays)"
                                            if dram_per_ray else None),
                         "l2": ({"bytes": round(prof["l2_bytes_per_ray"] * n),
                                 "achieved_gbs": round(prof["l2_bytes_per_ray"] * n / launch_s / 1e9, 1),
                                 "pct_of_peak": prof.get("l2_pct_of_peak"),
                                 "source": f"{TRAFFIC_PROFILE} (ncu capture)"}
                                if "l2_bytes_per_ray" in prof else None),
                         "bytes_per_ray": round(bytes_per_ray, 1),
                         "nodes_per_ray": round(float(nodes_per_ray), 2),
                         "tris_per_ray": round(float(tris_per_ray), 2)},
            "binning": ({"ms": round(bin_ms, 4), "bytes_per_ray": 44,
                         "achieved_gbs": round(bin_bytes / (bin_ms * 1e-3) / 1e9, 1)
                         if bin_ms > 0 else None,
                         "key_bits": {"origin": args.bin_origin, "dir": args.bin_dir},
                         "probe_frac": args.bin_probe}
                        if binning is not None else None),
            "parity": parity,
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(rays_od.nbytes), "d2h_bytes_per_step": int(n * 16),
                    "call": "enc_intersect_closest_od (origin + direction, 24 B per ray)",
                    "timing": "host wall clock around each synchronous call",
                    "eight_float_form": {"value": round(e2e8_value, 3),
                                         "call": "enc_intersect_closest (32 B per ray)",
                                         "h2d_bytes_per_step": int(rays.nbytes)}},
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
    ap.add_argument("--bin", action="store_true",
                    help="bin the batch (enc_bin_rays) inside every step and trace it in that "
                         "order (measured slower than the plain launch on this workload)")
    ap.add_argument("--bin-origin", type=int, default=0, help="binning key: origin bits (0 = default)")
    ap.add_argument("--bin-dir", type=int, default=0, help="binning key: direction bits")
    ap.add_argument("--bin-probe", type=float, default=0.0,
                    help="binning key: probe distance as a fraction of the scene diagonal")
    ap.add_argument("--tune-table", default=None,
                    help="batched section: write the autotuner's sweep table (JSON) here")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched multi-scene, served and photon-gather sections")
    ap.add_argument("--server-slots", type=int, default=6,
                    help="served section: request slots (rounds in flight)")
    ap.add_argument("--server-slot-rays", type=int, default=4 << 20,
                    help="served section: ray capacity of a slot (>= the largest request, 4M)")
    ap.add_argument("--served-requests", type=int, default=1200,
                    help="served section: Poisson arrivals behind the latency percentiles")
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
