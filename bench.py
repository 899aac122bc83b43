"""Benchmark: BVH trace throughput (Mrays/s) on the trace micro-benchmark workload.

Workload (one step): the 4,120-triangle small room (24-triangle box + 64x32
UV sphere), four batches of rays traced through the public ff_trace entry
point: 16,777,216 coherent pinhole camera rays (4096 x 4096 pixel centres)
and 16,777,216 incoherent rays (origins uniform in the scene box, directions
uniform on the sphere), each once closest-hit and once any-hit with tmax ~
U[0.1, 10] x scene diagonal.  67,108,864 ray queries per step per GPU.

`value` is whole-job ray queries per second with rays resident in HBM
(weak scaling: every rank traces its own full ray set).  `e2e` is the same
metric through ff_trace with pinned host buffers: the host-to-device copy of
the rays and the device-to-host copy of the hits are inside the timed region.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun every rank runs one GPU; rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s (BVH trace)"
WORKLOAD = "trace micro: small room 4120 tris, 16M coherent + 16M incoherent rays, closest + any-hit"
RAYS_PER_SET = 4096 * 4096
RAY_BYTES, HIT_BYTES = 32, 16


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def build_workload(n_per_set: int, seed_offset: int):
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0)
    side = int(round(math.sqrt(n_per_set)))
    coh = scenes.camera_rays(scn, side, side)
    inc = scenes.incoherent_rays(scn, side * side, seed=1 + seed_offset)
    coh_any = scenes.with_random_tmax(coh, scn, seed=2 + seed_offset)
    inc_any = scenes.with_random_tmax(inc, scn, seed=3 + seed_offset)
    batches = [("coherent_closest", coh, False), ("incoherent_closest", inc, False),
               ("coherent_any", coh_any, True), ("incoherent_any", inc_any, True)]
    return scn, batches


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("FF_CLOCK_LOG", f"/tmp/ff_clocks_{os.getpid()}.csv"))

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- CPU baselines
def cpu_trace_rate(batches, target_s: float, threads: int):
    """Time the reference's own BVH + intersect()/intersect_shadows(), compiled
    for the host (oracle/_ref), over a strided sample of every batch.  Falls
    back to the oracle's brute-force restatement when the reference build is
    absent.  Returns (Mrays/s, kind, sample description)."""
    import ctypes as C
    from oracle import ffo
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0)
    tris = scn.triangle_soup()
    ref_path = ffo.REF_LIB
    if ref_path.exists():
        lib = C.CDLL(str(ref_path))
        P = C.c_void_p
        lib.ffref_bvh_build.restype = P
        lib.ffref_bvh_build.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
        lib.ffref_bvh_trace.argtypes = [P, P, C.c_long, P, C.c_int, C.c_int]
        ms = C.c_double()
        h = lib.ffref_bvh_build(tris.ctypes.data, len(tris), C.byref(ms))

        def run(rays, any_hit):
            out = np.empty((len(rays), 2), np.float32)
            lib.ffref_bvh_trace(h, rays.ctypes.data, len(rays), out.ctypes.data, int(any_hit), threads)
        kind = "reference"
    else:
        def run(rays, any_hit):
            ffo.trace_brute(tris, rays, any_hit=any_hit, threads=threads)
        kind = "port"
    # calibrate on a small sample, then size the timed sample to target_s
    def sample(n):
        return [(np.ascontiguousarray(r[:: max(1, len(r) // n)][:n]), a) for _, r, a in batches]
    probe = sample(4096)
    t0 = time.perf_counter()
    for r, a in probe:
        run(r, a)
    dt = max(time.perf_counter() - t0, 1e-4)
    n = int(min(RAYS_PER_SET, max(4096, 4096 * target_s / dt)))
    timed = sample(n)
    t0 = time.perf_counter()
    for r, a in timed:
        run(r, a)
    dt = time.perf_counter() - t0
    total = sum(len(r) for r, _ in timed)
    desc = f"{total} rays: {n} strided from each of the 4 batches; {kind} BVH trace on {threads} threads"
    return total / dt / 1e6, kind, desc, dt


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    _, batches = build_workload(RAYS_PER_SET, 0)
    rates = []
    kind = desc = None
    for i in range(args.warmup + args.steps):
        rate, kind, desc, _ = cpu_trace_rate(batches, target_s=args.ref_step_s, threads=threads)
        if i >= args.warmup:
            rates.append(rate)
    value = statistics.median(rates)
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "rays_per_step": 4 * RAYS_PER_SET},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import firefly_b200 as ff

    # a dedicated stream shared by the library and the timing events
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ff.Context(local, stream=stream.cuda_stream)
    assert ctx.stream == stream.cuda_stream
    scn, batches = build_workload(args.rays, seed_offset=17 * rank)
    ds = ff.dScene(ctx, scn)
    n = batches[0][1].shape[0]

    d_rays = [torch.from_numpy(r).to(dev) for _, r, _ in batches]
    d_hits = [torch.empty((len(r), 4), dtype=torch.int32, device=dev) for _, r, _ in batches]
    torch.cuda.synchronize(dev)

    def step(evs=None):
        for k, (_, r, any_hit) in enumerate(batches):
            if evs is not None:
                evs[k][0].record(stream)
            ds.trace_device(d_rays[k].data_ptr(), len(r), d_hits[k].data_ptr(), any_hit=any_hit)
            if evs is not None:
                evs[k][1].record(stream)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launch_evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in batches] for _ in range(args.steps)]
    t0.record(stream)
    for s in range(args.steps):
        step(launch_evs[s])
    t1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    per_batch_ms = [statistics.mean(launch_evs[s][k][0].elapsed_time(launch_evs[s][k][1]) for s in range(args.steps))
                    for k in range(len(batches))]
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    rays_per_step = n * len(batches)
    value = ws * rays_per_step * args.steps / (ms_max / 1e3) / 1e6

    # end-to-end through the public entry point with pinned host buffers
    h_rays = [torch.from_numpy(r).pin_memory() for _, r, _ in batches]
    h_hits = [torch.empty((len(r), 4), dtype=torch.int32).pin_memory() for _, r, _ in batches]
    h_views = [(hr.numpy(), hh.numpy().view(np.uint8).view(ff.HIT_DTYPE).reshape(-1)) for hr, hh in zip(h_rays, h_hits)]

    def e2e_step():
        for k, (_, r, any_hit) in enumerate(batches):
            ds.trace(h_views[k][0], any_hit=any_hit, out=h_views[k][1])

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    barrier()
    e2e_steps = max(1, min(args.steps, 5))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e_ms = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(e_ms, op=dist.ReduceOp.MAX)
    e2e_value = ws * rays_per_step * e2e_steps / (float(e_ms.item()) / 1e3) / 1e6

    # correctness spot check of the timed outputs against the host path
    check = batches[1][1][:50_000]
    ok = np.array_equal(ds.trace(check)["prim"], h_views[1][1][:50_000]["prim"])

    if rank == 0:
        peak, peak_kind = measured_peaks()
        # roofline of the dominant kernel (closest-hit trace of incoherent rays):
        # algorithmic bytes = 32 B ray in + 16 B hit out per ray
        k_dom = int(np.argmax(per_batch_ms))
        achieved = n * (RAY_BYTES + HIT_BYTES) / (per_batch_ms[k_dom] / 1e3) / 1e9
        cpu = None
        if not args.no_cpu:
            rate, kind, desc, _ = cpu_trace_rate(batches, target_s=args.cpu_s, threads=os.cpu_count() or 1)
            cpu = {"value": round(rate, 3), "unit": "Mrays/s", "cores": os.cpu_count() or 1, "kind": kind,
                   "sample": desc}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rays_per_step": rays_per_step, "triangles": scn.num_triangles,
                       "bvh_nodes": ds.stats()["num_nodes"], "bvh_depth": ds.stats()["bvh_depth"],
                       "l2": "inputs larger than L2 (512 MiB of rays per batch)", "parallelism": f"replicas{ws}",
                       "per_batch_mrays": {b[0]: round(n / (t / 1e3) / 1e6, 1) for b, t in zip(batches, per_batch_ms)},
                       "hits_match_host_path": bool(ok)},
            "roofline": {"bound": "hbm", "kernel": f"k_trace ({batches[k_dom][0]})", "achieved": round(achieved, 2),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": None,
                         "peak_source": peak_kind, "bytes_per_ray": RAY_BYTES + HIT_BYTES},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(rays_per_step * RAY_BYTES),
                    "d2h_bytes_per_step": int(rays_per_step * HIT_BYTES)},
            "gpu_launches": len(batches) * args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ds.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rays", type=int, default=RAYS_PER_SET, help="rays per batch (4 batches per step)")
    ap.add_argument("--cpu-s", type=float, default=12.0, help="target seconds of CPU baseline work")
    ap.add_argument("--ref-step-s", type=float, default=4.0, help="reference arm: seconds of CPU work per step")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args(argv)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
