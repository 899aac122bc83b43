"""Benchmark of the wavefront path tracer: Mrays/s (BVH trace).

Default workload (`--workload render`), one step = one full render:
  an icosphere subdivided 8 times (1,310,720 triangles) displaced by 4-octave
  value noise inside a 12-triangle room, 33 materials of 5 kinds (the
  reference's mix material on the room; diffuse, GGX conductor, thin GGX
  dielectric and coated diffuse on the sphere, grouped by 3D noise), a
  2048 x 1024 sky with a 0.5 degree sun of radiance 5e4 as the light;
  1920 x 1080 at 64 samples per pixel, maximum depth 8, Russian roulette after
  depth 3, corrected mode.  Rays = extension (closest-hit) + shadow (any-hit)
  queries the wavefront traced.  Every step renders 64 new samples per pixel.
`value` is whole-job rays per second with the scene resident in HBM (weak
scaling: every rank renders its own frame).  `e2e` times the same render
through the public entry points with the camera uploaded from and the image
read back to pinned host memory every step.

At 1 GPU the render line also carries, under "metrics", the lines of the
other workloads, measured after the render's timed region (each in the same
format as its own --workload line):
  trace_micro     the trace micro-benchmark (4,120-triangle room, 16M coherent
                  + 16M incoherent rays, closest-hit and any-hit through
                  ff_trace), with the reference's own GPU traversal on the same
                  rays and every ray checked against the oracle;
  small_room      the plain tracer on the small room, 256 x 256 x 16 spp;
  adjoint         path-replay adjoint samples per second (inverse rendering);
  radiance_cache  time to relMSE 0.01 with the learned radiance cache against
                  the plain tracer.
--render-only skips them.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload render|trace|inverse|cache] [--render-only]
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
RENDER_WORKLOAD = ("wavefront path tracer at scale: displaced icosphere 1,310,720 tris in a 12-tri room, 5 material "
                   "kinds, 2048x1024 sky + sun, 1920x1080, 64 spp, depth 8")
TRACE_WORKLOAD = "trace micro: small room 4120 tris, 16M coherent + 16M incoherent rays, closest + any-hit"
RAYS_PER_SET = 4096 * 4096
RAY_BYTES, HIT_BYTES = 32, 16
# The traversal's records: an 8-wide quantized node (80 B), a triangle (48 B).
NODE_BYTES, TRI_BYTES = 80, 48
# The wavefront's traces read a tagged queue (32 B ray + 4 B tag): the
# closest-hit trace writes a 16 B hit, the any-hit trace a 1 B answer.
WF_CLOSEST_BYTES, WF_ANY_BYTES = 32 + 4 + 16, 32 + 4 + 1
# k_logic in the adjoint, per slot in flight and frame (continuing path):
# reads phase, key, ext_q, length, pass (20 B), the extension hit (16), ray
# origin and direction (32), throughput (16), radiance sum (16), shadow-queue
# indices (16) and ~1.5 shadow hits (24), the three light terms (48), ext_f /
# pdf / cos (20), the triangle's shading record (64); writes the sum (16) and
# the next vertex (uv, length, throughput, position, normal, light sample,
# queue entry: 112).  The replay pass adds dL/dI (12), L_s (16) and the
# vertex record (albedo + flags, uv, env coefficient, light direction: 56).
# Primal ~398 B, replay ~478 B: 438 B on average.
ADJ_LOGIC_BYTES_PER_HIT = 438
# k_logic in ff_render, per consumed extension hit of a continuing path:
# reads the slot words (12 B), the hit (16), the ray record (32), throughput,
# sum and compensation (48), the shading record (32), the pending light-term
# record of two frames back and its answer word (68) and the triangle's
# shading attributes (64); writes sum, compensation, length and throughput
# (52) and the vertex record (64): 388 B.
RENDER_LOGIC_BYTES_PER_HIT = 388
# k_shade, per shaded vertex: reads the vertex record (64 B), its queue
# entry (4) and the throughput (16), writes the shading record (32), the ray
# record (32), the extension-queue entry (36) and the pending light-term
# record (64): 248 B; plus 36 B per shadow-queue entry (32 B ray, 4 B tag).
# Environment and material lookups are L2 gathers and not counted.
RENDER_SHADE_BYTES_PER_VERTEX = 248
SHADOW_QUEUE_BYTES = 36
# Measured DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per unit
# of each render stage: ncu over every launch of one timed 16-spp C2 step on
# a 2,097,152-slot pool (104 frames), divided by the step's units (consumed
# hits, shaded vertices, extension rays, shadow rays).
RENDER_DRAM_BYTES_PER_UNIT = {"k_logic": 456.8, "k_shade (all kinds)": 418.7,
                              "k_trace<closest> (extension queue)": 109.4, "k_trace<any> (shadow queue)": 48.5}
# Issue slots busy (smsp__issue_active) of the closest-hit traversal on C2:
# ncu --set full of one steady-state launch of the same 16-spp, 2M-slot step
# (a figure from that capture, not measured by this run).
RENDER_ISSUE_SLOTS = {"k_trace<closest> (extension queue)": 0.696}
# Issue slots busy of the trace micro-benchmark's four launches (ncu --set full
# of one launch per batch kind, 4,194,304 rays each; figures from that
# capture, not measured by this run): the traversal is issue-bound.
TRACE_ISSUE_SLOTS = {"coherent_closest": 0.835, "incoherent_closest": 0.775, "coherent_any": 0.804,
                     "incoherent_any": 0.749}
RENDER = dict(width=1920, height=1080, spp=64, max_depth=8, rr_depth=3)
# Measured DRAM bytes per unit of the adjoint's stages (ncu over the profiled
# 512x512, 16-spp adjoint call of --workload inverse, 12 frames): per
# consumed extension hit for k_logic and k_shade, per traced ray for the traces.
ADJ_DRAM_BYTES_PER_UNIT = {"k_logic (adjoint)": 334.1, "k_shade (adjoint)": 259.2,
                           "k_trace closest (extension)": 52.0, "k_trace any (shadow)": 39.9}
# k_cache_infer: measured DRAM bytes per query (ncu over 6 cached 1080p
# frames, 9,513,224 queries): the 64 B record in and the film update; the
# hash grid's FP16 copy stays in L2.
CACHE_INFER_DRAM_BYTES_PER_QUERY = 110.8
# k_cache_infer's encoder: 16 levels x 8 corners x one 4-B FP16 pair per query.
CACHE_GATHER_BYTES_PER_QUERY = 16 * 8 * 4


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks(key: str = "hbm_gbs"):
    """(peak, "measured" | "fallback"): HBM copy GB/s or dense bf16 TFLOP/s."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d[key]), "measured"
        except Exception:
            pass
    return (6650.0 if key == "hbm_gbs" else 1590.0), "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(f"/tmp/ff_clocks_{os.getpid()}.csv")

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


# ------------------------------------------------------------------ workloads
def render_scene():
    from firefly_b200 import scenes
    return scenes.displaced_icosphere(subdiv=8, width=RENDER["width"], height=RENDER["height"])


def trace_batches(n_per_set: int, seed_offset: int):
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0)
    side = int(round(math.sqrt(n_per_set)))
    coh = scenes.camera_rays(scn, side, side)
    inc = scenes.incoherent_rays(scn, side * side, seed=1 + seed_offset)
    coh_any = scenes.with_random_tmax(coh, scn, seed=2 + seed_offset)
    inc_any = scenes.with_random_tmax(inc, scn, seed=3 + seed_offset)
    return scn, [("coherent_closest", coh, False), ("incoherent_closest", inc, False),
                 ("coherent_any", coh_any, True), ("incoherent_any", inc_any, True)]


# ------------------------------------------------------------- CPU baselines
def cpu_render_rate(scn, target_s: float, threads: int):
    """The reference's own path tracer compiled for the host (oracle/_ref:
    its gen_ray, SAH BVH, intersect(), lights and BRDF_L/BRDF_f/BRDF_pdf with
    their inline visibility rays) on every k-th pixel of the frame at the
    workload's spp and depth.  Returns (Mrays/s, kind, sample text, seconds)."""
    from oracle import ffref
    if not ffref.available():
        return None
    W, H = RENDER["width"], RENDER["height"]
    # calibrate on a sparse sample, then size the timed sample to target_s
    stride = 4099
    _, st, ms = ffref.render(scn, W, H, RENDER["spp"], RENDER["max_depth"], RENDER["rr_depth"], light=-1,
                             threads=threads, pixel_stride=stride)
    per_pixel_s = ms[0] / 1e3 / max(1, st[2] // RENDER["spp"])
    n_pix = max(64, int(target_s / max(per_pixel_s, 1e-9)))
    stride = max(1, (W * H) // n_pix)
    _, st, ms = ffref.render(scn, W, H, RENDER["spp"], RENDER["max_depth"], RENDER["rr_depth"], light=-1,
                             threads=threads, pixel_stride=stride)
    rays = st[0] + st[1]
    desc = (f"every {stride}th pixel of the 1920x1080 frame ({st[2] // RENDER['spp']} pixels x {RENDER['spp']} spp, "
            f"{rays} rays, {ms[0] / 1e3:.1f} s) with the reference's host-compiled path tracer on {threads} threads; "
            f"its SAH BVH build took {ms[1] / 1e3:.1f} s (not timed)")
    return rays / (ms[0] / 1e3) / 1e6, "reference", desc, ms[0] / 1e3


def cpu_trace_rate(batches, target_s: float, threads: int):
    """The reference's BVH + intersect()/intersect_shadows() compiled for the
    host on a strided sample of every trace batch."""
    import ctypes as C
    from oracle import ffo, ffref
    from firefly_b200 import scenes
    scn = scenes.small_room(seed=0)
    tris = scn.triangle_soup()
    if ffref.available():
        lib = ffref.load()
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
    rates, secs = [], []
    kind = desc = None
    if args.workload == "render":
        scn = render_scene()
        for i in range(args.warmup + args.steps):
            r = cpu_render_rate(scn, target_s=args.ref_step_s, threads=threads)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libffref.so was not built"}))
                return 0
            rate, kind, desc, sec = r
            if i >= args.warmup:
                rates.append(rate)
                secs.append(sec)
        workload, cfg = RENDER_WORKLOAD, dict(RENDER)
    else:
        _, batches = trace_batches(RAYS_PER_SET, 0)
        for i in range(args.warmup + args.steps):
            rate, kind, desc, sec = cpu_trace_rate(batches, target_s=args.ref_step_s, threads=threads)
            if i >= args.warmup:
                rates.append(rate)
                secs.append(sec)
        workload, cfg = TRACE_WORKLOAD, {"rays_per_step": 4 * RAYS_PER_SET}
    value = statistics.median(rates)
    line = {"metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            # one step = one bounded sample of the workload (see cpu_baseline.sample)
            "ms_per_step": round(1e3 * statistics.median(secs), 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload, **cfg},
            "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def setup_dist():
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    return ws, rank, local, dist


def max_over_ranks(dist, dev, x: float) -> float:
    import torch
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def trace_micro(ctx, ds_dev, args, rank, dev, stream, barrier, steps):
    """Trace micro-benchmark on this rank; returns (rays per step, per-batch ms, total ms, batches, scene)."""
    import torch
    import firefly_b200 as ff
    scn, batches = trace_batches(args.rays, seed_offset=17 * rank)
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
    for _ in range(3):
        step()
    barrier()
    evs = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in batches] for _ in range(steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for s in range(steps):
        step(evs[s])
    t1.record(stream)
    barrier()
    per = [statistics.mean(evs[s][k][0].elapsed_time(evs[s][k][1]) for s in range(steps)) for k in range(len(batches))]
    total = t0.elapsed_time(t1)
    return n * len(batches), per, total, batches, scn, ds, d_rays, d_hits


L2_PROBE_SRC = b"""
extern "C" __global__ void l2_read(const float4* __restrict__ a, unsigned long long n4, int reps, float* out)
{
    float acc = 0.f;
    for (int r = 0; r < reps; ++r)
        for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n4;
             i += (unsigned long long)gridDim.x * blockDim.x) {
            const float4 v = __ldcg(a + i);
            acc += v.x + v.y + v.z + v.w;
        }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}
"""


def l2_read_gbs(dev, mib=32, reps=40):
    """Reference bandwidth for L2-resident reads: one kernel (compiled here
    with NVRTC for sm_100a) reads a 32 MiB buffer, far below the 126 MB L2,
    `reps` times with L1-bypassing 16-byte loads; bytes read per second, best
    of 5 launches timed with CUDA events on the current stream.  None when
    cuda-python is unavailable."""
    import ctypes
    import torch
    try:
        from cuda.bindings import driver as cu, nvrtc
    except ImportError:
        return None
    err, prog = nvrtc.nvrtcCreateProgram(L2_PROBE_SRC, b"l2_probe.cu", 0, [], [])
    opts = [b"--gpu-architecture=sm_100a"]
    if nvrtc.nvrtcCompileProgram(prog, len(opts), opts)[0] != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        return None
    _, size = nvrtc.nvrtcGetCUBINSize(prog)
    cubin = b" " * size
    nvrtc.nvrtcGetCUBIN(prog, cubin)
    a = torch.ones(mib * 2 ** 18, dtype=torch.float32, device=dev)
    threads, blocks = 256, torch.cuda.get_device_properties(dev).multi_processor_count * 8
    out = torch.empty(threads * blocks, dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)   # torch's context is current on this thread
    err, mod = cu.cuModuleLoadData(cubin)
    if err != cu.CUresult.CUDA_SUCCESS:
        return None
    _, fn = cu.cuModuleGetFunction(mod, b"l2_read")
    cur = torch.cuda.current_stream(dev)
    params = ((a.data_ptr(), a.numel() // 4, reps, out.data_ptr()),
              (ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_void_p))

    def launch():
        r = cu.cuLaunchKernel(fn, blocks, 1, 1, threads, 1, 1, 0, cu.CUstream(cur.cuda_stream), params, 0)
        assert r[0] == cu.CUresult.CUDA_SUCCESS, r
    for _ in range(3):
        launch()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        launch()
        e1.record(cur)
        e1.synchronize()
        best = max(best, a.numel() * 4 * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    cu.cuModuleUnload(mod)
    return best


# DRAM bytes per ray of k_trace launches, from an ncu capture at 4,194,304
# rays per launch (the trace micro-benchmark's profile); traffic scales with rays.
TRACE_DRAM_BYTES_PER_RAY = {"coherent_closest": (134.470144e6 + 42.339328e6) / 4194304,
                            "incoherent_closest": (135.088384e6 + 40.223232e6) / 4194304,
                            "coherent_any": (134.470144e6 + 42.339328e6) / 4194304,
                            "incoherent_any": (135.088384e6 + 40.223232e6) / 4194304}


def reference_cuda_trace(scn, batches, d_hits):
    """The reference's own GPU traversal (intersect / intersect_shadows of
    CUDA-RayTracer/dTriangle.cu, built unmodified for sm_100a) over its own
    SAH BVH, on the same rays: Mrays/s per batch and agreement of its hits
    with ours.  Outside the timed region; None when oracle/_ref lacks it."""
    try:
        from oracle import ffrefcuda
    except Exception:
        return None
    if not ffrefcuda.available():
        return {"unavailable": "oracle/_ref/libffrefcuda.so was not built (no reference checkout at build time)"}
    bvh = ffrefcuda.RefGpuBVH(scn.triangle_soup())
    out, agree = {}, {}
    total_rays, total_ms = 0, 0.0
    for k, (name, rays, any_hit) in enumerate(batches):
        t, prim, ms = bvh.trace(rays, any_hit=any_hit, reps=2)
        out[name] = round(len(rays) / (ms / 1e3) / 1e6, 1)
        total_rays += len(rays)
        total_ms += ms
        ours = d_hits[k].cpu().numpy()[:, 3]
        agree[name] = round(float(np.mean((ours >= 0) == (prim >= 0)) if any_hit else np.mean(ours == prim)), 6)
    bvh.close()
    return {"mrays": round(total_rays / (total_ms / 1e3) / 1e6, 1), "per_batch_mrays": out,
            "hit_agreement_with_ours": agree, "bvh_nodes": bvh.num_nodes,
            "build": "CUDA-RayTracer/dRay.cu + dTriangle.cu unmodified, nvcc 12.9 -O3 sm_100a (FMA contraction on, "
                     "nvcc's default), 64-thread blocks as wavefront_pathtrace launches them, BVH2 from the "
                     "reference's host SAH build, 200-byte dTriangle records, 80-byte Isect written per ray"}


def oracle_trace_check(scn, batches, d_hits):
    """Every ray of every batch against the oracle (its CPU hierarchy over
    the same triangles, deciding each triangle with the restated
    dTriangle::intersect / shadow_hit): closest hits must agree bit for bit
    (prim, t, u, v; ties to the lowest index), any-hit answers as occluded or
    not.  Outside the timed region, on all host threads."""
    from oracle import ffo
    t0 = time.perf_counter()
    bvh = ffo.BVH(scn.triangle_soup())
    out = {}
    for k, (name, rays, any_hit) in enumerate(batches):
        ours = d_hits[k].cpu().numpy().view(np.uint32)
        ref = bvh.trace(rays, any_hit=any_hit).view(np.uint32).reshape(-1, 4)
        if any_hit:
            bad = (ours[:, 3].view(np.int32) >= 0) != (ref[:, 3].view(np.int32) >= 0)
        else:
            hit = ref[:, 3].view(np.int32) != -1
            bad = (ours[:, 3] != ref[:, 3]) | (hit & np.any(ours[:, :3] != ref[:, :3], axis=1))
        out[name] = {"rays": int(len(rays)), "mismatches": int(bad.sum())}
    bvh.close()
    return {"per_batch": out, "rays": int(sum(v["rays"] for v in out.values())),
            "mismatches": int(sum(v["mismatches"] for v in out.values())),
            "seconds": round(time.perf_counter() - t0, 1), "threads": os.cpu_count() or 1,
            "compared": "closest: prim, t, u, v bit for bit; any-hit: occluded or not"}


def run_trace(args, ws, rank, local, dist):
    import torch
    import firefly_b200 as ff
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ff.Context(local, stream=stream.cuda_stream)
    line = trace_line(args, ws, rank, local, dist, ctx, dev, stream, args.steps)
    if line is not None:
        print(json.dumps(line), flush=True)
    ctx.close()


def trace_line(args, ws, rank, local, dist, ctx, dev, stream, steps):
    """The trace micro-benchmark (C3) on this rank; rank 0 gets its JSON line."""
    import torch
    import firefly_b200 as ff

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    rays_per_step, per, total_ms, batches, scn, ds, d_rays, d_hits = trace_micro(ctx, None, args, rank, dev, stream,
                                                                                barrier, steps)
    clk = clocks.stop()
    ms_max = max_over_ranks(dist, dev, total_ms)
    value = ws * rays_per_step * steps / (ms_max / 1e3) / 1e6
    n = batches[0][1].shape[0]
    # end to end through ff_trace with pinned host buffers
    h_rays = [torch.from_numpy(r).pin_memory() for _, r, _ in batches]
    h_hits = [torch.empty((len(r), 4), dtype=torch.int32).pin_memory() for _, r, _ in batches]
    views = [(hr.numpy(), hh.numpy().view(np.uint8).view(ff.HIT_DTYPE).reshape(-1)) for hr, hh in zip(h_rays, h_hits)]

    def e2e_step():
        for k, (_, r, any_hit) in enumerate(batches):
            ds.trace(views[k][0], any_hit=any_hit, out=views[k][1])
    e2e_step()
    barrier()
    e2e_steps = max(1, min(steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e_ms = max_over_ranks(dist, dev, e0.elapsed_time(e1))
    e2e_value = ws * rays_per_step * e2e_steps / (e_ms / 1e3) / 1e6
    if rank == 0:
        peak, peak_kind = measured_peaks()
        k_dom = int(np.argmax(per))
        achieved = n * (RAY_BYTES + HIT_BYTES) / (per[k_dom] / 1e3) / 1e9
        cpu = None
        if not args.no_cpu:
            rate, kind, desc, _ = cpu_trace_rate(batches, target_s=args.cpu_s, threads=os.cpu_count() or 1)
            cpu = {"value": round(rate, 3), "unit": "Mrays/s", "cores": os.cpu_count() or 1, "kind": kind, "sample": desc}
        ref_cuda = reference_cuda_trace(scn, batches, d_hits) if not args.no_ref_cuda else None
        check = None if args.no_oracle_check else oracle_trace_check(scn, batches, d_hits)
        # traversal fetch bytes: node records and triangles each ray's traversal
        # reads (counted by the same traversal on the device, outside the timed
        # region), against an L2-resident copy
        try:
            l2_ref = l2_read_gbs(dev)
        except Exception as e:   # the reference bandwidth is optional
            print(f"l2 read probe unavailable: {e}", file=sys.stderr)
            l2_ref = None
        fetch = {}
        for k, (name, _, any_hit) in enumerate(batches):
            wk = ds.trace_count(d_rays[k].data_ptr(), n, any_hit=any_hit)
            fetch[name] = {"nodes_per_ray": round(wk["nodes"] / n, 3), "tris_per_ray": round(wk["tris"] / n, 3),
                           "fetch_bytes_per_ray": round(wk["fetch_bytes_per_ray"], 1),
                           "achieved_fetch_gbs": round(wk["fetch_bytes_per_ray"] * n / (per[k] / 1e3) / 1e9, 1)}
        l2_fetch = {"per_batch": fetch, "l2_read_gbs": None if l2_ref is None else round(l2_ref, 1),
                    "frac_of_l2_read": (None if l2_ref is None else
                                        round(fetch[batches[k_dom][0]]["achieved_fetch_gbs"] / l2_ref, 4)),
                    "node_bytes": wk["node_bytes"], "tri_bytes": wk["tri_bytes"],
                    "note": ("fetched bytes = node records x node bytes + triangles tested x triangle bytes per ray "
                             "(the device traversal's counts, equal to the oracle's restatement of it: "
                             "tests/test_trace_gpu.py); "
                             "l2_read_gbs = a probe kernel reading a 32 MiB L2-resident buffer 40 times (L1 bypassed); "
                             "the traversal's fetches are partly served by L1, so the fraction is an upper bound "
                             "on its L2 load")}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": ws, "steps": steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": TRACE_WORKLOAD, "rays_per_step": rays_per_step, "triangles": scn.num_triangles,
                       "l2": "inputs larger than L2 (512 MiB of rays per batch)", "parallelism": f"replicas{ws}",
                       "per_batch_mrays": {b[0]: round(n / (t / 1e3) / 1e6, 1) for b, t in zip(batches, per)},
                       "reference_cuda": ref_cuda, "oracle_check": check},
            "roofline": {"bound": "hbm", "kernel": f"k_trace ({batches[k_dom][0]})", "achieved": round(achieved, 2),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5),
                         "traffic": int(TRACE_DRAM_BYTES_PER_RAY[batches[k_dom][0]] * n),
                         "traffic_source": "ncu dram__bytes_read+write of a 4,194,304-ray launch, scaled to the "
                                           "launch's rays",
                         "peak_source": peak_kind, "bytes_per_ray": RAY_BYTES + HIT_BYTES, "l2_fetch": l2_fetch,
                         "issue_slots_busy": {"per_batch": TRACE_ISSUE_SLOTS,
                                              "source": "ncu smsp__issue_active of one launch per batch kind "
                                                        "(4,194,304 rays), not measured by this run",
                                              "note": "the bound of this kernel: instruction issue under "
                                                      "divergence, not HBM (frac) or L2 (l2_fetch)"}},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": int(rays_per_step * RAY_BYTES),
                    "d2h_bytes_per_step": int(rays_per_step * HIT_BYTES)},
            "gpu_launches": len(batches) * steps,
            "clocks": clk,
        }
    ds.close()
    return line if rank == 0 else None


def run_render(args, ws, rank, local, dist):
    import torch
    import firefly_b200 as ff
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ff.Context(local, stream=stream.cuda_stream)
    assert ctx.stream == stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    scn = render_scene()
    ds = ff.dScene(ctx, scn)
    W, H = RENDER["width"], RENDER["height"]
    pt = ff.PathTracer(ctx, W, H)
    from firefly_b200 import multigpu
    kw = dict(spp=RENDER["spp"], max_depth=RENDER["max_depth"], rr_depth=RENDER["rr_depth"], light=-1,
              mode=ff.FF_MODE_CORRECTED, seed=0, max_paths=args.max_paths)
    step_no = [0]
    film_rgba = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    film_cnt = torch.empty((H, W), dtype=torch.int32, device=dev)

    def step(profile=False):
        # every rank renders its own sample range of the same frame; with N > 1 the
        # films are summed with one all-reduce (sample-parallel, weak scaling)
        pt.clear_buffer()
        off = multigpu.sample_offset(rank, ws, RENDER["spp"], step_no[0])
        st = pt.draw(ds, sample_offset=off, profile=profile, **kw)
        step_no[0] += 1
        if dist is not None:
            multigpu.read_film_device(pt, film_rgba, film_cnt)
            multigpu.allreduce_film(film_rgba, film_cnt)
        return st

    for _ in range(args.warmup):
        step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    # the NVTX range lets ncu capture exactly the timed steps (--nvtx --nvtx-include "timed/")
    torch.cuda.nvtx.range_push("timed")
    t0.record(stream)
    for _ in range(args.steps):
        stats.append(step())
    t1.record(stream)
    torch.cuda.nvtx.range_pop()
    barrier()
    clk = clocks.stop()
    ms_max = max_over_ranks(dist, dev, t0.elapsed_time(t1))
    rays = sum(s["extension_rays"] + s["shadow_rays"] for s in stats)
    rays_max = max_over_ranks(dist, dev, float(rays))
    value = ws * rays_max / (ms_max / 1e3) / 1e6
    samples = sum(s["samples"] for s in stats)
    # one profiled step (outside the timed region): per-stage device time
    prof = step(profile=True)
    # end to end through the public entry points: camera in, image out, pinned host memory
    img = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    cnt = torch.empty((H, W), dtype=torch.int32).pin_memory()
    cam = scn.camera
    import ctypes as C
    lib = ff.lib()

    def e2e_step():
        ds.update(cam)
        st = step()
        if dist is not None:
            img.copy_(film_rgba)
            cnt.copy_(film_cnt)
        else:
            rc = lib.ff_film_read(pt.film, C.c_void_p(img.data_ptr()), C.c_void_p(cnt.data_ptr()), 0)
            assert rc == 0
        return st
    e2e_step()
    barrier()
    e2e_steps = max(1, min(args.steps, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    est = []
    e0.record(stream)
    for _ in range(e2e_steps):
        est.append(e2e_step())
    e1.record(stream)
    barrier()
    e_ms = max_over_ranks(dist, dev, e0.elapsed_time(e1))
    e_rays = sum(s["extension_rays"] + s["shadow_rays"] for s in est)
    e2e_value = ws * e_rays / (e_ms / 1e3) / 1e6
    image = img.numpy()[..., :3] / np.maximum(cnt.numpy(), 1)[..., None]
    finite = bool(np.isfinite(image).all())
    conv = None
    if rank == 0 and not args.no_relmse:
        # relMSE of the step's image against a float64-accumulated 16k-spp render
        # of the centre tile (1/16 of the pixels) under its own seed
        from firefly_b200 import convergence
        tile = convergence.centre_tile(W, H)
        ref, info = convergence.reference_image(ctx, ds, cam, W, H, tile=tile, max_depth=kw["max_depth"],
                                                rr_depth=kw["rr_depth"], light=-1, mode=ff.FF_MODE_CORRECTED)
        x0, y0, tw, th = tile
        crop = image[y0:y0 + th, x0:x0 + tw]
        conv = {"relmse": round(convergence.relmse(crop, ref), 6),
                "relmse_trimmed_1e-4": round(convergence.relmse_trimmed(crop, ref), 6),
                "median_pixel_rel_sq_err": round(float(np.median(convergence.pixel_terms(crop, ref))), 6),
                "spp": int(cnt.numpy()[y0, x0]), "reference_spp": info["spp"], "tile": info["tile"],
                "reference_s": round(info["seconds"], 1), "accumulation": "float64"}

    metrics = None
    if ws == 1 and not args.render_only:
        # the other three metrics and the small-room workload, measured after
        # the render's timed region on the same GPU (one GPU only)
        metrics = {"trace_micro": trace_line(args, ws, rank, local, dist, ctx, dev, stream, 3),
                   "small_room": small_room_line(args, ws, rank, local, dist, ctx, dev, stream),
                   "adjoint": inverse_line(args, ws, rank, local, dist, ctx, dev, stream, known_lighting_run=False),
                   "radiance_cache": cache_line(args, ws, rank, local, dist, ctx, dev, stream)}
    elif ws > 1:
        metrics = {"note": "the trace micro-benchmark, small room, adjoint and cache lines are measured at 1 GPU"}
    if rank == 0:
        peak, peak_kind = measured_peaks()
        # dominant stage by device time (events of the profiled step), with the
        # algorithmic bytes of one launch sequence: the traced rays' queue I/O,
        # or the slot-state bytes above per consumed hit / shaded vertex
        vertices = max(0, prof["extension_rays"] - prof["samples"])
        stage = {"k_trace<any> (shadow queue)": (prof["ms_trace_shadow"], prof["shadow_rays"] * WF_ANY_BYTES,
                                                 f"{WF_ANY_BYTES} B per shadow ray (ray + tag in, 1 B answer out)"),
                 "k_trace<closest> (extension queue)": (prof["ms_trace_extension"],
                                                        prof["extension_rays"] * WF_CLOSEST_BYTES,
                                                        f"{WF_CLOSEST_BYTES} B per extension ray (ray + tag in, "
                                                        "hit out)"),
                 "k_logic": (prof["ms_logic"], prof["extension_rays"] * RENDER_LOGIC_BYTES_PER_HIT,
                             f"{RENDER_LOGIC_BYTES_PER_HIT} B of slot state per consumed extension hit"),
                 "k_shade (all kinds)": (prof["ms_shade"], vertices * RENDER_SHADE_BYTES_PER_VERTEX
                                         + prof["shadow_rays"] * SHADOW_QUEUE_BYTES,
                                         f"{RENDER_SHADE_BYTES_PER_VERTEX} B of slot records and queue entries per "
                                         f"shaded vertex + {SHADOW_QUEUE_BYTES} B per shadow-queue entry")}
        units = {"k_logic": prof["extension_rays"], "k_shade (all kinds)": vertices,
                 "k_trace<closest> (extension queue)": prof["extension_rays"],
                 "k_trace<any> (shadow queue)": prof["shadow_rays"]}
        # the HBM roofline's kernel: the stage that moves the most DRAM bytes
        # in the step (measured bytes per unit x the profiled step's units).  The three stages on
        # the frame's critical path take about the same device time each, and
        # the two traversals are bound by instruction issue, not by HBM
        dram_step = {k: RENDER_DRAM_BYTES_PER_UNIT[k] * units[k] for k in stage}
        dom = max(stage, key=lambda k: dram_step[k])
        dms, dbytes, dnote = stage[dom]
        achieved = dbytes / (dms / 1e3) / 1e9
        # DRAM traffic of one launch sequence (one frame) of the dominant
        # stage: the measured bytes per unit times the frame's average units
        frames = max(1, prof["frames"])
        traffic = int(RENDER_DRAM_BYTES_PER_UNIT[dom] * units[dom] / frames)
        alg_launch = int(dbytes / frames)
        cpu = None
        if not args.no_cpu:
            r = cpu_render_rate(scn, target_s=args.cpu_s, threads=os.cpu_count() or 1)
            if r is not None:
                cpu = {"value": round(r[0], 3), "unit": "Mrays/s", "cores": os.cpu_count() or 1, "kind": r[1],
                       "sample": r[2]}
        pstat = {k: round(prof[k], 2) for k in ("ms_total", "ms_logic", "ms_shade", "ms_trace_extension", "ms_trace_shadow")}
        # the traces' node and triangle fetches (counted by a second pass of the
        # same traversal over each frame's queues in the profiled step) against
        # an L2-resident read: the traversal reads a 0.27 GB scene mostly from
        # L2, so this and the issue rate bound it rather than DRAM
        try:
            l2_ref = l2_read_gbs(dev)
        except Exception as e:   # the reference bandwidth is optional
            print(f"l2 read probe unavailable: {e}", file=sys.stderr)
            l2_ref = None
        l2_fetch = {}
        for name, ms_k, rays_k, nodes_k, tris_k in (
                ("k_trace<closest> (extension queue)", prof["ms_trace_extension"], prof["extension_rays"],
                 prof["ext_nodes"], prof["ext_tris"]),
                ("k_trace<any> (shadow queue)", prof["ms_trace_shadow"], prof["shadow_rays"],
                 prof["shadow_nodes"], prof["shadow_tris"])):
            fb = nodes_k * NODE_BYTES + tris_k * TRI_BYTES
            gbs = fb / (ms_k / 1e3) / 1e9 if ms_k > 0 else None
            l2_fetch[name] = {"nodes_per_ray": round(nodes_k / max(1, rays_k), 3),
                              "tris_per_ray": round(tris_k / max(1, rays_k), 3),
                              "fetch_bytes_per_ray": round(fb / max(1, rays_k), 1),
                              "achieved_fetch_gbs": None if gbs is None else round(gbs, 1),
                              "frac_of_l2_read": None if (gbs is None or l2_ref is None) else round(gbs / l2_ref, 4)}
        l2_fetch = {"stages": l2_fetch, "l2_read_gbs": None if l2_ref is None else round(l2_ref, 1),
                    "node_bytes": NODE_BYTES, "tri_bytes": TRI_BYTES,
                    "note": ("fetched bytes = 8-wide node records x node bytes + triangles tested x triangle bytes, "
                             "counted over the profiled step's queues by the device traversal, whose counts equal "
                             "the oracle's restatement of it (tests/test_trace_gpu.py); l2_read_gbs = a probe kernel "
                             "reading a 32 MiB L2-resident buffer 40 times (L1 bypassed); part of the fetches hit "
                             "L1, so the fraction is an upper bound on the L2 load")}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": RENDER_WORKLOAD, **RENDER, "triangles": scn.num_triangles,
                       "bvh_nodes": ds.stats()["num_nodes"], "bvh_build_ms": round(ds.stats()["build_ms"], 2),
                       "mode": "corrected", "light": "environment (importance-sampled sky + sun)",
                       "rays_per_step": int(rays / args.steps),
                       "units_per_step": {k: int(sum(s[k] for s in stats) / args.steps)
                                          for k in ("extension_rays", "shadow_rays", "samples", "frames")},
                       "msamples_per_s": round(ws * samples / (ms_max / 1e3) / 1e6, 2),
                       "frames_per_step": stats[-1]["frames"], "stage_ms_profiled_step": pstat,
                       "l2": "each step traces ~1.3G rays over a 0.27 GB scene; per-step state and queues ~0.5 GB",
                       "parallelism": (f"sample-parallel x{ws}: disjoint sample ranges of one frame, one film "
                                       f"all-reduce (41 MB) per step" if ws > 1 else "1 GPU"),
                       "image_finite": finite, "relmse_vs_16k_spp": conv},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5), "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes": dnote, "algorithmic_bytes_per_launch": alg_launch,
                         "traffic_note": ("bytes per frame's launch sequence of the dominant stage: ncu DRAM bytes "
                                          "per unit of a 16-spp step on a 2M-slot pool x this step's units per frame"),
                         "selection": ("the stage with the most DRAM bytes in the step (dram_gb_per_step); the "
                                       "stages' device times (ms) are within a few percent of each other, and the "
                                       "traversals are bound by instruction issue (see issue_slots_busy and "
                                       "l2_fetch), where an HBM fraction does not apply"),
                         "stages": {k: {"ms": round(v[0], 2), "achieved_gbs": round(v[1] / (v[0] / 1e3) / 1e9, 1)
                                        if v[0] > 0 else None,
                                        "frac": round(v[1] / (v[0] / 1e3) / 1e9 / peak, 4) if v[0] > 0 else None,
                                        "algorithmic_bytes_per_unit": round(v[1] / max(1, units[k]), 1),
                                        "dram_bytes_per_unit": RENDER_DRAM_BYTES_PER_UNIT[k],
                                        "dram_gb_per_step": round(dram_step[k] / 1e9, 1),
                                        **({"issue_slots_busy": RENDER_ISSUE_SLOTS[k]} if k in RENDER_ISSUE_SLOTS
                                           else {})}
                                    for k, v in stage.items()},
                         "l2_fetch": l2_fetch},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 80,
                    "d2h_bytes_per_step": int(W * H * (16 + 4))},
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "clocks": clk,
            "metrics": metrics,
        }
        print(json.dumps(line), flush=True)
    pt.close()
    ds.close()
    ctx.close()


SMALL_ROOM_WORKLOAD = ("plain tracer, small room: 24-tri box + 64x32 UV sphere (4,120 tris) at a seeded position, "
                       "mix-material albedos U[0.2, 0.8], one area light of radiance 15; 256x256, 16 spp, depth 5, "
                       "RR from depth 3, parity mode (the reference's behaviours), seed 0")
SMALL_ROOM = dict(width=256, height=256, spp=16, max_depth=5, rr_depth=3)


def small_room_line(args, ws, rank, local, dist, ctx, dev, stream, steps=20, warmup=3):
    """The small-room workload (C1): extension + shadow rays per second of
    whole 256 x 256 x 16-spp frames (every step renders 16 new samples per
    pixel), with the reference's host-compiled path tracer on the same scene
    beside it; rank 0 gets its JSON line."""
    import ctypes as C
    import torch
    import firefly_b200 as ff
    from firefly_b200 import scenes
    W, H = SMALL_ROOM["width"], SMALL_ROOM["height"]
    scn = scenes.small_room(seed=0, width=W, height=H)
    ds = ff.dScene(ctx, scn)
    pt = ff.PathTracer(ctx, W, H)
    kw = dict(spp=SMALL_ROOM["spp"], max_depth=SMALL_ROOM["max_depth"], rr_depth=SMALL_ROOM["rr_depth"], light=0,
              mode=ff.FF_MODE_PARITY, seed=0)
    k = [0]

    def step(profile=False):
        pt.clear_buffer()
        st = pt.draw(ds, sample_offset=SMALL_ROOM["spp"] * k[0], profile=profile, **kw)
        k[0] += 1
        return st
    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    t0.record(stream)
    for _ in range(steps):
        stats.append(step())
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = max_over_ranks(dist, dev, t0.elapsed_time(t1))
    rays = sum(s["extension_rays"] + s["shadow_rays"] for s in stats)
    samples = sum(s["samples"] for s in stats)
    prof = step(profile=True)
    # end to end: camera in, image and counts out to pinned host memory
    img = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    cnt = torch.empty((H, W), dtype=torch.int32).pin_memory()
    lib = ff.lib()

    def e2e_step():
        ds.update(scn.camera)
        st = step()
        assert lib.ff_film_read(pt.film, C.c_void_p(img.data_ptr()), C.c_void_p(cnt.data_ptr()), 0) == 0
        return st
    e2e_step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    est = []
    e0.record(stream)
    for _ in range(5):
        est.append(e2e_step())
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e_ms = e0.elapsed_time(e1)
    e_rays = sum(s["extension_rays"] + s["shadow_rays"] for s in est)
    line = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        stages = {"k_trace<any> (shadow queue)": (prof["ms_trace_shadow"], prof["shadow_rays"] * WF_ANY_BYTES),
                  "k_trace<closest> (extension queue)": (prof["ms_trace_extension"],
                                                         prof["extension_rays"] * WF_CLOSEST_BYTES),
                  "k_logic": (prof["ms_logic"], prof["extension_rays"] * RENDER_LOGIC_BYTES_PER_HIT),
                  "k_shade (all kinds)": (prof["ms_shade"], max(0, prof["extension_rays"] - prof["samples"])
                                          * RENDER_SHADE_BYTES_PER_VERTEX + prof["shadow_rays"] * SHADOW_QUEUE_BYTES)}
        dom = max(stages, key=lambda n: stages[n][0])
        achieved = stages[dom][1] / (stages[dom][0] / 1e3) / 1e9
        cpu = None
        if not args.no_cpu:
            from oracle import ffref
            if ffref.available():
                threads = os.cpu_count() or 1
                # whole 256 x 256 x 16-spp frames, repeated for about cpu_s / 2 seconds
                target, frames, rays_cpu, secs = max(args.cpu_s / 2, 1.0), 0, 0, 0.0
                while secs < target:
                    _, st1, ms1 = ffref.render(scn, W, H, SMALL_ROOM["spp"], SMALL_ROOM["max_depth"],
                                               SMALL_ROOM["rr_depth"], light=0, threads=threads, pixel_stride=1)
                    frames += 1
                    rays_cpu += st1[0] + st1[1]
                    secs += ms1[0] / 1e3
                cpu = {"value": round(rays_cpu / secs / 1e6, 3), "unit": "Mrays/s", "cores": threads,
                       "kind": "reference",
                       "sample": (f"{frames} whole 256x256 x 16-spp frames ({rays_cpu} rays, {secs:.1f} s) with the "
                                  f"reference's host-compiled path tracer (area light, its SAH BVH build not timed) "
                                  f"on {threads} threads")}
        line = {"metric": METRIC, "value": round(ws * rays / (ms / 1e3) / 1e6, 2), "unit": "Mrays/s", "n_gpus": ws,
                "steps": steps, "warmup": warmup, "ms_per_step": round(ms / steps, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": SMALL_ROOM_WORKLOAD, **SMALL_ROOM, "triangles": scn.num_triangles,
                           "msamples_per_s": round(ws * samples / (ms / 1e3) / 1e6, 2),
                           "rays_per_step": int(rays / steps), "frames_per_step": stats[-1]["frames"],
                           "stage_ms_profiled_step": {n: round(prof[n], 3) for n in
                                                      ("ms_total", "ms_logic", "ms_shade", "ms_trace_extension",
                                                       "ms_trace_shadow")},
                           "l2": "scene (0.5 MB) and the 1M-slot path state (0.45 GB) stay resident; each step "
                                 "re-renders every pixel"},
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": peak,
                             "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": None,
                             "peak_source": peak_kind,
                             "note": "algorithmic bytes per unit as in the at-scale render line (slot state per hit "
                                     "or vertex, queue I/O per ray) over the stage's event-timed duration"},
                "cpu_baseline": cpu,
                "e2e": {"value": round(e_rays / (e_ms / 1e3) / 1e6, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 80,
                        "d2h_bytes_per_step": W * H * 20},
                "gpu_launches": int(sum(s["kernel_launches"] for s in stats)), "clocks": clk}
    pt.close()
    ds.close()
    return line


INVERSE_WORKLOAD = ("inverse rendering on the room opened to the sky at 512x512: hidden 512x512 Perlin albedo in "
                    "[0.1, 0.9] + 256x128 hazy sky (sun radiance 8, 20 deg); target at 256 spp; start 0.5 albedo + "
                    "flat env; 16-spp path-replay adjoint, Adam lr 1e-2 falling geometrically to 1e-3, 200 steps")


def inverse_experiment(ctx, steps=200, res=512, dev=None, known_lighting=False, rank=0, world=1):
    """C4 workload; returns a dict of results (timings, losses, parameter errors)."""
    import torch
    import firefly_b200 as ff
    from firefly_b200 import inverse, scenes
    # A hazy sky: under a small bright sun the 16-spp images are so noisy that
    # their variance, not the parameters' error, sets the image error.
    sky = scenes.sky_env(256, 128, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    hidden = scenes.textured_room(seed=0, width=res, height=res, tex_res=512, env=sky)
    flat_env = np.full_like(hidden.env_rgb, float(hidden.env_rgb.mean()))
    start = scenes.textured_room(seed=0, width=res, height=res, albedo=np.full((512, 512, 3), 0.5, np.float32),
                                 env=flat_env)
    ds = ff.dScene(ctx, hidden)
    pt = ff.PathTracer(ctx, res, res)
    t0 = time.perf_counter()
    pt.draw(ds, spp=256, max_depth=3, rr_depth=3, seed=12345, light=-1, mode=ff.FF_MODE_CORRECTED)
    target = torch.from_numpy(pt.image().astype(np.float32)).to(dev)
    t_target = time.perf_counter() - t0
    albedo = torch.from_numpy(start.textures[0].copy()).to(dev)
    env = torch.from_numpy((hidden.env_rgb if known_lighting else start.env_rgb).copy()).to(dev)
    tex_err0 = float(np.sqrt(((start.textures[0] - hidden.textures[0]) ** 2).mean()))
    t0 = time.perf_counter()
    res_opt = inverse.optimize(ds, pt, target, albedo, env, steps=steps, spp=16, lr=1e-2, max_depth=3, rr_depth=3,
                               lr_env=0.0 if known_lighting else None, lr_decay=0.1, rank=rank, world=world)
    wall = time.perf_counter() - t0
    tex_err1 = float(np.sqrt(((albedo.cpu().numpy() - hidden.textures[0]) ** 2).mean()))
    e_h = hidden.env_rgb
    env_err = lambda e: float(np.abs(e - e_h).mean() / np.abs(e_h).mean())
    # held-out image error (fresh seed, 64 spp) before and after, and with the
    # hidden parameters themselves: the floor that the two images' noise sets
    def heldout(tex, e):
        ds.set_texture(0, tex)
        ds.set_environment(e)
        pt.clear_buffer()
        pt.draw(ds, spp=64, max_depth=3, rr_depth=3, seed=777, light=-1, mode=ff.FF_MODE_CORRECTED)
        return float(((pt.image() - target.cpu().numpy()) ** 2).mean())
    h0 = heldout(start.textures[0], hidden.env_rgb if known_lighting else start.env_rgb)
    h1 = heldout(albedo.cpu().numpy(), env.cpu().numpy())
    hf = heldout(hidden.textures[0], hidden.env_rgb)
    out = {"workload": INVERSE_WORKLOAD + (" (known lighting: albedo only)" if known_lighting else ""),
           "steps": steps, "wall_s": round(wall, 2), "heldout_mse_start": h0, "heldout_mse_end": h1,
           "heldout_mse_hidden_params": hf,
           "adjoint_spp_per_s": round(res_opt["adjoint_spp_per_s"], 1),
           "adjoint_samples_per_step": int(res_opt["adjoint_samples"] / steps),
           "grad_atomics_per_step": int(res_opt["grad_atomics"] / steps),
           "kernel_launches_per_step": round(res_opt["kernel_launches"] / steps, 1),
           "adjoint_ms_per_step": round(res_opt["ms_adjoint"] / steps, 3),
           "primal_ms_per_step": round(res_opt["ms_primal"] / steps, 3), "target_render_s": round(t_target, 2),
           "loss_first": res_opt["losses"][0], "loss_last": res_opt["losses"][-1],
           "albedo_rmse_start": round(tex_err0, 4), "albedo_rmse_end": round(tex_err1, 4),
           "env_rel_err_start": round(env_err(flat_env), 4), "env_rel_err_end": round(env_err(env.cpu().numpy()), 4)}
    pt.close()
    ds.close()
    return out


def run_inverse(args, ws, rank, local, dist):
    import torch
    import firefly_b200 as ff
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ff.Context(local, stream=stream.cuda_stream)
    line = inverse_line(args, ws, rank, local, dist, ctx, dev, stream)
    if line is not None:
        print(json.dumps(line), flush=True)
    ctx.close()


def inverse_line(args, ws, rank, local, dist, ctx, dev, stream, known_lighting_run=True):
    """The inverse-rendering workload (C4): adjoint samples per second over
    200 Adam steps; rank 0 gets its JSON line."""
    clocks = ClockSampler(local)
    clocks.start()
    r = inverse_experiment(ctx, steps=args.steps if args.steps > 5 else 200, dev=dev, rank=rank, world=ws)
    if known_lighting_run:
        r["known_lighting_run"] = inverse_experiment(ctx, steps=args.steps if args.steps > 5 else 200, dev=dev,
                                                     known_lighting=True, rank=rank, world=ws)
    # every rank adjoints its own samples of each step (gradients averaged
    # across ranks): whole-job samples over the slowest rank's adjoint time
    adj_ms_max = max_over_ranks(dist, dev, r["adjoint_ms_per_step"])
    value = ws * r["adjoint_samples_per_step"] / (adj_ms_max / 1e3)
    r["parallelism"] = (f"{ws} GPUs: sample-parallel steps, films summed and gradients averaged by all-reduce"
                        if ws > 1 else "1 GPU")
    clk = clocks.stop()
    e2e, prof = inverse_e2e(ctx, dev, stream)
    if rank == 0:
        peak, peak_kind = measured_peaks()
        # dominant stage of the wavefront adjoint (per-stage events of one
        # profiled call at the same size)
        stages = {"k_logic (adjoint)": prof["ms_logic"], "k_shade (adjoint)": prof["ms_shade"],
                  "k_trace closest (extension)": prof["ms_trace_extension"],
                  "k_trace any (shadow)": prof["ms_trace_shadow"]}
        r["adjoint_stage_ms"] = {k: round(v, 3) for k, v in stages.items()}
        r["adjoint_rays"] = {"extension": prof["extension_rays"], "shadow": prof["shadow_rays"]}
        dom = max(stages, key=stages.get)
        if dom.startswith("k_logic"):
            # one consumed extension hit per slot and frame
            achieved = prof["extension_rays"] * ADJ_LOGIC_BYTES_PER_HIT / (stages[dom] / 1e3) / 1e9
            note = (f"algorithmic bytes = {ADJ_LOGIC_BYTES_PER_HIT} B of slot state read and written per consumed "
                    "extension hit (primal and replay passes averaged) over the stage's event-timed duration")
        elif "trace" in dom:
            rays = prof["extension_rays"] if "closest" in dom else prof["shadow_rays"]
            per = WF_CLOSEST_BYTES if "closest" in dom else WF_ANY_BYTES
            achieved = rays * per / (stages[dom] / 1e3) / 1e9
            note = (f"algorithmic bytes = {per} B per ray (32 B ray + 4 B tag in, the hit or answer out) x the "
                    "stage's rays over its event-timed duration; BVH and triangles are L2-resident")
        else:
            adj_ms = r["adjoint_ms_per_step"]
            achieved = r["grad_atomics_per_step"] * 12 / (adj_ms / 1e3) / 1e9
            note = ("algorithmic bytes = 12 B of float atomics per texel touch after the warp pre-reduction "
                    "(counted by the kernels) over the whole adjoint")
        # DRAM traffic of the dominant stage per frame: measured bytes per
        # unit (ncu over the profiled call) x this call's units per frame
        units = {"k_logic (adjoint)": prof["extension_rays"], "k_shade (adjoint)": prof["extension_rays"],
                 "k_trace closest (extension)": prof["extension_rays"], "k_trace any (shadow)": prof["shadow_rays"]}
        traffic = int(ADJ_DRAM_BYTES_PER_UNIT[dom] * units[dom] / max(1, prof["frames"]))
        cpu = None if args.no_cpu else inverse_cpu_baseline(target_s=args.cpu_s)
        line = {"metric": "adjoint spp/s", "value": round(value, 1), "unit": "samples/s", "n_gpus": ws,
                "steps": r["steps"], "warmup": 0, "ms_per_step": r["adjoint_ms_per_step"] + r["primal_ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": r,
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2),
                             "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": traffic,
                             "peak_source": peak_kind, "note": note,
                             "traffic_note": ("DRAM bytes per frame of the dominant stage: ncu dram bytes per unit of "
                                              "the profiled 512x512x16-spp adjoint call x its units per frame"),
                             "dram_bytes_per_unit": ADJ_DRAM_BYTES_PER_UNIT},
                "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(round(r["kernel_launches_per_step"] * r["steps"])), "clocks": clk}
    return line if rank == 0 else None


def inverse_e2e(ctx, dev, stream, iters=5, res=512):
    """The adjoint through the public API with host buffers: d_image in,
    texture and env gradients out, every call (ff_render_adjoint with host
    pointers into pinned host memory, as the other lines' e2e)."""
    import torch
    import firefly_b200 as ff
    from firefly_b200 import scenes
    sky = scenes.sky_env(256, 128, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    scn = scenes.textured_room(seed=0, width=res, height=res, tex_res=512, env=sky)
    ds = ff.dScene(ctx, scn)
    rng = np.random.default_rng(0)

    def pinned(shape):
        return torch.zeros(shape, dtype=torch.float32).pin_memory().numpy()
    d_image = pinned((res, res, 3))
    d_image[...] = (rng.normal(size=(res, res, 3)) / (res * res * 3)).astype(np.float32)
    g_tex = pinned((512, 512, 3))
    g_env = pinned(sky.shape)
    ds.render_adjoint(res, res, d_image, grad_texture=g_tex, grad_env=g_env, spp=16, seed=1)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    samples = 0
    e0.record(stream)
    for k in range(iters):
        st = ds.render_adjoint(res, res, d_image, grad_texture=g_tex, grad_env=g_env, spp=16, seed=2 + k)
        samples += st["samples"]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    # one more call with per-stage events: the split between the wavefront
    # stages of the adjoint (outside the timed region)
    # (the NVTX range lets ncu capture exactly this call: --nvtx --nvtx-include "profiled/")
    torch.cuda.nvtx.range_push("profiled")
    prof = ds.render_adjoint(res, res, d_image, grad_texture=g_tex, grad_env=g_env, spp=16, seed=99, profile=True)
    torch.cuda.nvtx.range_pop()
    ds.close()
    e2e = {"value": round(samples / (ms / 1e3), 1), "unit": "samples/s",
           "h2d_bytes_per_step": int(d_image.nbytes + g_tex.nbytes + g_env.nbytes),
           "d2h_bytes_per_step": int(g_tex.nbytes + g_env.nbytes)}
    return e2e, prof


def inverse_cpu_baseline(target_s=15.0):
    """The oracle's path tracer (C restatement, all host threads) on the same
    scene: primal samples per second over a pixel subset, the lower bound of a
    CPU adjoint sample's cost (the replay traces every path twice)."""
    try:
        from oracle import ffo
    except Exception:
        return None
    from firefly_b200 import scenes
    sky = scenes.sky_env(256, 128, seed=0, sun_radiance=8.0, sun_diameter_deg=20.0)
    res = 64
    scn = scenes.textured_room(seed=0, width=res, height=res, tex_res=512, env=sky)
    threads = os.cpu_count() or 1
    spp, ms = 16, 0.0
    t0 = time.perf_counter()
    ffo.render(scn, res, res, spp, max_depth=3, rr_depth=3, seed=1, mode=1, light=-1, threads=threads)
    dt = time.perf_counter() - t0
    spp2 = max(16, int(spp * target_s / max(dt, 1e-3)))
    t0 = time.perf_counter()
    ffo.render(scn, res, res, spp2, max_depth=3, rr_depth=3, seed=2, mode=1, light=-1, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": round(res * res * spp2 / dt, 1), "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"the oracle's path tracer on the same scene at {res}x{res} x {spp2} spp ({dt:.1f} s), "
                      "primal samples only"}


CACHE_WORKLOAD = ("small room (24-tri box + 64x32 UV sphere, area light radiance 15) at 1920x1080, depth 5, "
                  "RR from 3, corrected mode: time until the progressively accumulated image reaches relMSE 0.01 "
                  "on the centre tile (480x270) against a float64-accumulated 16k-spp render; learned radiance cache "
                  "(hash grid 16 levels x 2 x 2^19, MLP 4 x 64 ReLU bf16 on tcgen05, 65,536 training paths per "
                  "frame, Adam in steps of 16,384) against the plain wavefront tracer")
CACHE_TARGET = 0.01


def checkpoints(limit):
    """Frame counts at which the accumulated image's error is measured
    (about +6% each, so the time to the target overshoots by at most that)."""
    out, k = [], 1
    while k <= limit:
        out.append(k)
        k = max(k + 1, int(round(k * 1.06)))
    return out


def run_cache(args, ws, rank, local, dist):
    import torch
    import firefly_b200 as ff
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = ff.Context(local, stream=stream.cuda_stream)
    line = cache_line(args, ws, rank, local, dist, ctx, dev, stream)
    if line is not None:
        print(json.dumps(line), flush=True)
    ctx.close()


def cache_line(args, ws, rank, local, dist, ctx, dev, stream):
    """The radiance-cache workload (C5): time to relMSE 0.01 against the
    plain tracer; rank 0 gets its JSON line."""
    import ctypes as C
    import torch
    import firefly_b200 as ff
    from firefly_b200 import _abi as A
    from firefly_b200 import convergence, scenes
    from firefly_b200.cache import RadianceCache
    W, H = 1920, 1080
    scn = scenes.small_room(seed=0, width=W, height=H)
    ds = ff.dScene(ctx, scn)
    kw = dict(max_depth=5, rr_depth=3, light=0)
    if args.cache_frames_only:
        # a short run for profilers: cached frames only, no reference, no plain tracer
        cache = RadianceCache(ds)
        pt = ff.PathTracer(ctx, W, H)
        st = cache.render(ds, pt, frames=args.cache_frames_only, seed=12, **kw)
        cache.close()
        pt.close()
        ds.close()
        return ({"workload": "cached frames only (profiling)", "frames": args.cache_frames_only,
                 "ms_total": st["ms_total"], "queries": st["cache_queries"], "records": st["cache_records"]}
                if rank == 0 else None)
    tile = convergence.centre_tile(W, H)
    ref, info = convergence.reference_image(ctx, ds, scn.camera, W, H, tile=tile, mode=ff.FF_MODE_CORRECTED, **kw)
    x0, y0, tw, th = tile
    pt = ff.PathTracer(ctx, W, H)
    cps = checkpoints(args.cache_max_frames)

    def error_now():
        img = pt.image()
        return convergence.relmse(img[y0:y0 + th, x0:x0 + tw], ref)

    def progressive(render_more):
        """(ms to reach the target or None, trajectory [(frames, ms, relMSE)])"""
        pt.clear_buffer()
        ms, done, traj, hit = 0.0, 0, [], None
        for c in cps:
            ms += render_more(c - done, done)
            done = c
            e = error_now()
            traj.append((c, round(ms, 2), round(e, 5)))
            if e <= CACHE_TARGET:
                hit = ms
                break
        return hit, traj

    clocks = ClockSampler(local)
    clocks.start()
    # the plain tracer: one draw call per increment
    plain_ms, plain_traj = progressive(
        lambda k, done: pt.draw(ds, spp=k, seed=11, sample_offset=done, mode=ff.FF_MODE_CORRECTED, **kw)["ms_total"])
    # the cache from scratch: warm-up frames (trained, then discarded) count in the time
    cache = RadianceCache(ds)
    pt.clear_buffer()
    warm = cache.render(ds, pt, frames=args.cache_warmup, seed=12, **kw)
    warm_ms = warm["ms_total"]
    cache_ms, cache_traj = progressive(
        lambda k, done: cache.render(ds, pt, frames=k, seed=13, sample_offset=args.cache_warmup + done,
                                     **kw)["ms_total"])
    cache_total = None if cache_ms is None else warm_ms + cache_ms
    # one profiled frame: stage times, queries and records
    s = A.ff_render_settings(spp=4, max_depth=5, rr_depth=3, seed=14, mode=ff.FF_MODE_CORRECTED, light=0,
                             max_paths=0, sample_offset=200000, flags=A.FF_RENDER_PROFILE, shadow_offset=0.001)
    st = A.ff_render_stats()
    rc = ff.lib().ff_render_cached(ctx.handle, ds.handle, cache.handle, C.byref(s), pt.film, C.byref(st))
    assert rc == 0
    prof = {k: getattr(st, k) for k, _ in st._fields_}
    # end to end: camera in, warm-up, frames, image to pinned host memory
    img_h = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    cnt_h = torch.empty((H, W), dtype=torch.int32).pin_memory()
    frames_needed = cache_traj[-1][0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cache.reset()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    ds.update(scn.camera)
    pt.clear_buffer()
    cache.render(ds, pt, frames=args.cache_warmup, seed=12, **kw)
    pt.clear_buffer()
    cache.render(ds, pt, frames=frames_needed, seed=13, sample_offset=args.cache_warmup, **kw)
    rc = ff.lib().ff_film_read(pt.film, C.c_void_p(img_h.data_ptr()), C.c_void_p(cnt_h.data_ptr()), 0)
    assert rc == 0
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(dist, dev, cache_total if cache_total is not None else float("nan"))
    if rank == 0:
        peak, peak_kind = measured_peaks("bf16_tflops")
        q_flops = prof["cache_queries"] * 2.0 * (4 * 64 * 64 + 16 * 64)
        q_tflops = q_flops / (prof["ms_cache_query"] / 1e3) / 1e12 if prof["ms_cache_query"] > 0 else None
        # the encoder's hash-grid gathers (16 levels x 8 corners x 4 B per
        # query, from the L2-resident FP16 table) against an L2-resident read
        try:
            l2_ref = l2_read_gbs(dev)
        except Exception as e:   # the reference bandwidth is optional
            print(f"l2 read probe unavailable: {e}", file=sys.stderr)
            l2_ref = None
        g_gbs = (prof["cache_queries"] * CACHE_GATHER_BYTES_PER_QUERY / (prof["ms_cache_query"] / 1e3) / 1e9
                 if prof["ms_cache_query"] > 0 else None)
        l2_gather = {"gather_bytes_per_query": CACHE_GATHER_BYTES_PER_QUERY,
                     "achieved_gather_gbs": None if g_gbs is None else round(g_gbs, 1),
                     "l2_read_gbs": None if l2_ref is None else round(l2_ref, 1),
                     "frac_of_l2_read": None if (g_gbs is None or l2_ref is None) else round(g_gbs / l2_ref, 4),
                     "note": ("the kernel is bound by these gathers (L1 and L2 throughput), not by the tensor pipe; "
                              "l2_read_gbs = a probe kernel reading a 32 MiB L2-resident buffer 40 times (L1 "
                              "bypassed); each 4-B entry moves a 32-B sector, two corners per sector where they "
                              "share an aligned group of four")}
        line = {"metric": "time-to-relMSE 0.01 (learned radiance cache)", "value": None if ms != ms else round(ms, 2),
                "unit": "ms", "n_gpus": ws, "steps": len(cache_traj), "warmup": args.cache_warmup,
                "ms_per_step": None, "higher_is_better": False, "scaling": "replicas", "vs_baseline": None,
                "dtype": "bf16 MLP / f32 paths", "data": "synthetic",
                "config": {"workload": CACHE_WORKLOAD, "target_relmse": CACHE_TARGET,
                           "plain_tracer_ms": None if plain_ms is None else round(plain_ms, 2),
                           "speedup_vs_plain": (None if (plain_ms is None or cache_total is None)
                                                else round(plain_ms / cache_total, 3)),
                           "cache_warmup_frames": args.cache_warmup, "cache_warmup_ms": round(warm_ms, 2),
                           "trajectory_plain": plain_traj, "trajectory_cache": cache_traj,
                           "reference": info, "tile": list(tile),
                           "profiled_4_frames": {k: (round(v, 3) if isinstance(v, float) else v)
                                                 for k, v in prof.items()},
                           "parallelism": "1 GPU" if ws == 1 else f"{ws} independent replicas (time = max over ranks)"},
                "roofline": {"bound": "tensor", "kernel": "k_cache_infer (+ k_frame_to_film)",
                             "achieved": None if q_tflops is None else round(q_tflops, 3), "peak": peak,
                             "unit": "TFLOP/s", "frac": None if q_tflops is None else round(q_tflops / peak, 5),
                             "traffic": int(CACHE_INFER_DRAM_BYTES_PER_QUERY * prof["cache_queries"]
                                            / max(1, prof["frames"])),
                             "traffic_note": ("DRAM bytes of one k_cache_infer launch (one per frame): ncu dram bytes "
                                              "per query over 6 frames x this run's queries per frame"),
                             "peak_source": peak_kind,
                             "flops_per_query": 2 * (4 * 64 * 64 + 16 * 64), "l2_gather": l2_gather},
                "cpu_baseline": None,
                "cpu_baseline_note": "not timed for the cache: the plain tracer on the same GPU is the comparator",
                "e2e": {"value": round(e2e_ms, 2), "unit": "ms", "h2d_bytes_per_step": 80,
                        "d2h_bytes_per_step": W * H * 20},
                "gpu_launches": int(warm["kernel_launches"]) + sum(1 for _ in cache_traj),
                "clocks": clk}
    cache.close()
    pt.close()
    ds.close()
    return line if rank == 0 else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["render", "trace", "inverse", "cache"], default="render")
    ap.add_argument("--cache-warmup", type=int, default=2, help="cache workload: training frames before accumulating")
    ap.add_argument("--cache-max-frames", type=int, default=1024, help="cache workload: give up after this many")
    ap.add_argument("--cache-frames-only", type=int, default=0,
                    help="cache workload: only render this many cached frames (for profilers)")
    ap.add_argument("--rays", type=int, default=RAYS_PER_SET, help="trace workload: rays per batch")
    ap.add_argument("--cpu-s", type=float, default=15.0, help="target seconds of CPU-baseline work")
    ap.add_argument("--ref-step-s", type=float, default=6.0, help="reference arm: seconds of CPU work per step")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-relmse", action="store_true", help="skip the 16k-spp reference tile and its relMSE")
    ap.add_argument("--no-ref-cuda", action="store_true", help="trace workload: skip the reference's GPU traversal")
    ap.add_argument("--render-only", action="store_true",
                    help="render workload: skip the trace, small-room, adjoint and cache lines")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="trace workload: skip the check of every ray against the oracle")
    ap.add_argument("--spp", type=int, default=RENDER["spp"], help="render workload: samples per pixel per step")
    ap.add_argument("--max-paths", type=int, default=0,
                    help="render workload: path-pool slots (0: the library's default; smaller pools for profiling)")
    args = ap.parse_args(argv)
    RENDER["spp"] = args.spp
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    ws, rank, local, dist = setup_dist()
    if args.workload == "render":
        run_render(args, ws, rank, local, dist)
    elif args.workload == "inverse":
        run_inverse(args, ws, rank, local, dist)
    elif args.workload == "cache":
        run_cache(args, ws, rank, local, dist)
    else:
        run_trace(args, ws, rank, local, dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
