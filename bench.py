#!/usr/bin/env python3
"""Benchmark of the path-tracing hot path (one JSON line on stdout, rank 0).

A step is one full frame of the measured workload, rendered by the compat-mode kernel (the reference's
semantics: per-pixel thrust::minstd_rand stream, mixture-PDF lambertian, floor(sqrt(spp))^2 samples):

  spheres (default)  1280x720, 64 spp, depth 50, 488 spheres (ground r=1000, 22x22 grid of r=0.2, three
                     r=1 feature spheres; 80/15/5 % lambertian/metal/dielectric), defocus aperture 0.1 at
                     focus 10, sky-gradient background, one quad light; synthetic, seed 20261203.
  cornell            256x256, 16 spp, depth 8 (the small Cornell box, reference host-build size).
  meshes             1920x1080, 121 traced spp (128 requested), depth 16, 1,310,720 triangles, env map.

value  = Mpaths/s of the whole job (all ranks; weak scaling, one replica frame per rank), device time
         from CUDA events on the launching stream, L2 flushed (256 MiB write) between steps.
e2e    = the same metric through the public C ABI with host buffers: per step rtc_scene_create
         (flatten + BVH build + H2D upload) + rtc_render (kernel + D2H of the FP32 radiance) + destroy.
         The BVH is the host SAH build unless --builder device|lbvh (PLOC or linear BVH built on the GPU).
roofline: algorithmic bytes of the render kernel per launch (BVH node visits x 64 B + primitive tests x
         their record size + per-ray state), counted by an instrumented launch of the same frame, divided
         by the mean event time of the timed launches, against the measured HBM copy bandwidth.
cpu_baseline: the reference's own CPU code (oracle/_ref/libref_cpu.so: the reference's classes built
         with g++) on all host cores, on a deterministic pixel subsample of the same frame.

  batched            64 heterogeneous scenes (1K-500K triangles, 256^2..1024^2, spp 4/16/64, depth
                     8-32, seed 20261203) rendered as one batch per step through rtc_render_batch, against
                     the plain form: the same 64 images one rtc_render_device call each.
  served             Poisson request streams (rate --lambdas, --requests each) over the batched scenes
                     (Zipf s=1.1 popularity, orbiting cameras, each scene's resolution/spp/depth) through
                     the render server; p50/p95/p99 latency and Mpaths/s, against a plain server that
                     renders one request per launch in arrival order.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config spheres|cornell|meshes|batched|served]
                  [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from cortexraytracercuda_b200 import configs  # noqa: E402
from cortexraytracercuda_b200.scene import (DRAW_ORDER_DEVICE, DRAW_ORDER_HOST, ENGINE_MEGAKERNEL,  # noqa: E402
                                            ENGINE_WAVEFRONT, FLAG_KERNEL_TIMING, FLAG_SAMPLE_GROUPS,
                                            FLAG_WIDE_BVH, MODE_CLEAN, MODE_COMPAT, BVH_DEVICE, BVH_DEVICE_LBVH, BVH_SAH,
                                            RenderParams)

METRIC = "Mpaths/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0

# bytes fetched per visit (ignoring caches) for the roofline's algorithmic traffic
NODE_BYTES = 64          # BVH2 node: two child boxes + two child links (4 x float4)
NODE8_BYTES = 80         # 8-wide compressed node: origin, exponents, link bases, slot links, 8-bit child bounds (5 x float4)
PRIM_BYTES = {"spheres": 16, "cornell": 48, "meshes": 48}   # dominant primitive record of each workload
# algorithmic FP32 operations per visit (the fixed constants of the roofline's flop count): a binary node's
# two slab tests, and the dominant primitive test of each workload (sphere 20, triangle 30)
NODE_FLOPS = 24
PRIM_FLOPS = {"spheres": 20, "cornell": 30, "meshes": 30}
STATE_BYTES = 32 + 16 + 2 * 48   # ray read + hit write + path state read/write per traversal
EXTEND_STATE_BYTES = 4 + 32 + 8   # queue entry + the slot's ray sector (origin, direction, start, depth) read, hit write


# Path-state bytes the shade kernel moves per traced ray (its algorithmic traffic): the queue entry and
# the slot's three 32-byte sectors read (ray, shade with the hit, pixel: 4 + 3 x 32), the ray and shade
# sectors and the stream word written back (2 x 32 + 4), and the survivor's queue entry (4).
SHADE_STATE_BYTES = 4 + 3 * 32 + 2 * 32 + 4 + 4
NCU_SUMMARY = ROOT / "profiles" / "ncu_wavefront_{config}.json"


def kernel_bounds(config, peak, kstats, ext_rays, roof):
    """What binds each wavefront kernel: the live per-frame times of this run (CUDA events) beside the
    figures of one ncu --set full capture per kernel of the same frame (profiles/ncu_wavefront_<config>
    .json): DRAM and L2 bytes per launch, issue-active and lanes active per instruction.  DRAM traffic is
    far below the algorithmic bytes (the BVH, the scene and most of the path state stay in L1/L2), and
    no kernel is near the DRAM or FP32 peak: the kernels are bound by memory latency and divergence."""
    f = NCU_SUMMARY.with_name(NCU_SUMMARY.name.format(config=config))
    prof = {}
    if f.exists():
        try:
            prof = json.loads(f.read_text())
        except Exception:
            prof = {}
    live = {"wf_extend": (float(np.mean([s["extend_ms"] for s in kstats])), int(np.mean([s["extend_launches"] for s in kstats]))),
            "wf_shade": (float(np.mean([s["shade_ms"] for s in kstats])), int(np.mean([s["shade_launches"] for s in kstats]))),
            "wf_finish": (float(np.mean([s["drain_ms"] for s in kstats])), 1)}
    out = {}
    for k, (ms, n) in live.items():
        rec = {"ms_per_frame": round(ms, 3), "launches_per_frame": n, "avg_launch_us": round(1e3 * ms / max(n, 1), 2)}
        p = prof.get(k)
        if p:
            avg_s = ms / 1e3 / max(n, 1) if k != "wf_finish" else ms / 1e3
            rec.update({kk: p[kk] for kk in ("dram_bytes_per_launch", "l2_bytes_per_launch", "l1_hit_pct", "l2_hit_pct",
                                              "issue_active_pct", "lanes_active_per_inst", "warps_active_pct",
                                              "registers", "top_stalls") if kk in p})
            if "dram_bytes_per_launch" in p and k != "wf_finish":
                rec["dram_frac"] = round(p["dram_bytes_per_launch"] / avg_s / 1e9 / peak, 4)
            if "l2_bytes_per_launch" in p and k != "wf_finish":
                rec["l2_gbs"] = round(p["l2_bytes_per_launch"] / avg_s / 1e9, 1)
        out[k] = rec
    shade_ms = live["wf_shade"][0]
    out["wf_shade"]["alg_bytes_per_frame"] = int(ext_rays * SHADE_STATE_BYTES)
    out["wf_shade"]["alg_gbs"] = round(ext_rays * SHADE_STATE_BYTES / (shade_ms / 1e3) / 1e9, 1)
    ext = out["wf_extend"]
    res = {"bound": "latency",
           "bound_why": "DRAM traffic per launch is a few percent of the algorithmic bytes and of the DRAM peak; "
                        "FP32 issue is a few percent of peak; the kernels wait on dependent L1/L2 fetches "
                        "(long_scoreboard) with about a third of the lanes active (divergent walks)",
           "kernels": out}
    if "dram_bytes_per_launch" in ext:
        res["traffic"] = ext["dram_bytes_per_launch"]
        res["dram_frac"] = ext.get("dram_frac")
    if prof:
        res["profile_source"] = f"profiles/{f.name} (ncu --set full, one launch per kernel, command in " \
                                f"profiles/wavefront_kernels_{config}.md)"
    return res


def workload(name):
    mk, mp = configs.SCENES[name]
    scene = mk()
    params = mp()
    params.mode = MODE_COMPAT
    params.draw_order = DRAW_ORDER_DEVICE
    return scene, params


# what each measured scene adds to the workload as specified, named in the bench line
ADDED = {"spheres": " + hidden quad light of random_spheres.scene (the config names none)",
         "meshes": " + hidden 8x4 quad light (the config names none)", "cornell": ""}


def describe(name, params, scene):
    return {"workload": f"{name} {params.width}x{params.height} spp{params.spp} (traced {params.traced_spp}) "
                        f"depth{params.max_depth}{ADDED.get(name, '')}",
            "primitives": scene.num_primitives, "mode": "compat (reference RNG stream and quirks)",
            "l2": "flushed between steps (256 MiB write)", "seed": configs.DEFAULT_SEED}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_reference_rate(scene, params, target_s=10.0, max_pixels=None):
    """Times the reference's own CPU implementation on a deterministic pixel subsample.
    Returns (Mpaths/s, Mrays/s, info)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    ref = oracles.ref_cpu()
    kind = "reference"
    threads = os.cpu_count() or 1
    if ref is not None:
        p = params.__class__(**{**params.__dict__, "draw_order": DRAW_ORDER_HOST})
        rs = ref.scene(scene)
        run = lambda pix: rs.render_pixels(p, pix, threads)   # noqa: E731
    else:
        kind = "port"
        port = oracles.port()
        ps = port.scene(scene)
        p = params.__class__(**{**params.__dict__, "draw_order": DRAW_ORDER_HOST})
        run = lambda pix: ps.render_pixels(p, pix, threads, trig=0)   # noqa: E731
    npix = params.width * params.height
    # calibration on 1/4096 of the frame, then a sample sized for ~target_s
    stride = 4096
    pix = np.arange(0, npix, stride, dtype=np.int64)
    t = time.perf_counter()
    run(pix)
    dt = max(time.perf_counter() - t, 1e-6)
    per_px = dt / pix.size
    want = int(min(npix, max(pix.size, target_s / per_px)))
    if max_pixels:
        want = min(want, max_pixels)
    stride = max(1, npix // want)
    pix = np.arange(0, npix, stride, dtype=np.int64)
    t = time.perf_counter()
    _, rays = run(pix)
    dt = time.perf_counter() - t
    paths = pix.size * params.traced_spp
    info = {"kind": kind, "cores": threads,
            "sample": f"every {stride}th pixel of the frame ({pix.size} px x {params.traced_spp} paths), "
                      f"{dt:.1f} s"}
    return paths / dt / 1e6, rays / dt / 1e6, info


# The reference's own GPU build timed on the same B200 (a second reported baseline, not a target): its
# classes compiled by nvcc for sm_100a (oracle/_ref/libref_gpu.so), its render loop in its own launch
# shape (16x16 blocks, one thread per pixel, gpu.cu:2072-2080), the per-pixel printf left out.
REF_GPU_CASES = [
    # (label, scene builder, parameters)
    ("cornell 256x256 spp16 depth8", lambda: configs.cornell(), dict(width=256, height=256, spp=16, max_depth=8)),
    ("spheres 1280x720 spp64 depth50 (the timed frame)", lambda: configs.spheres(),
     dict(width=1280, height=720, spp=64, max_depth=50)),
    ("spheres 320x180 spp16 depth16, constant background", lambda: configs.spheres(sky=False),
     dict(width=320, height=180, spp=16, max_depth=16)),
    ("textured 160x120 spp16 depth10", lambda: configs.textured(), dict(width=160, height=120, spp=16, max_depth=10)),
    ("icosphere (1,280 triangles x3) 150x100 spp16 depth12", lambda: configs.icosphere_scene(),
     dict(width=150, height=100, spp=16, max_depth=12)),
]


def ref_gpu_baseline(ctx, stream, warmup=3, steps=3):
    """Per case: the reference's own nvcc build (kernel time from CUDA events, one launch after one
    untimed launch) against this library's default engine on the same scene and parameters (nvcc
    flavour, scene resident, mean of `steps` event-timed launches after `warmup`).  None when the
    reference's GPU build is not available."""
    import torch
    from cortexraytracercuda_b200.renderer import DeviceScene
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    ref = oracles.ref_gpu()
    if ref is None:
        return None
    out = []
    sp = stream.cuda_stream
    for label, mk, kw in REF_GPU_CASES:
        scene = mk()
        p = RenderParams(**kw)
        p.mode, p.draw_order, p.engine = MODE_COMPAT, DRAW_ORDER_DEVICE, ENGINE_WAVEFRONT
        ds = DeviceScene(ctx, scene)
        img = torch.empty((p.height, p.width, 4), dtype=torch.float32, device="cuda")
        for _ in range(warmup):
            ds.render_device(p, img.data_ptr(), stream=sp)
        evs = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ds.render_device(p, img.data_ptr(), stream=sp)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        ours_ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
        ds.close()
        rs = ref.scene(scene)
        if p.width * p.height <= 65536:
            rs.render_frame_timed(p)   # untimed first launch (module load, heap warm-up)
        ref_ms, _ = rs.render_frame_timed(p)
        del rs
        paths = p.width * p.height * p.traced_spp
        out.append({"case": label, "reference_gpu_ms": round(ref_ms, 2),
                    "reference_gpu_mpaths_per_s": round(paths / ref_ms / 1e3, 3),
                    "ours_ms": round(ours_ms, 3), "ours_mpaths_per_s": round(paths / ours_ms / 1e3, 3),
                    "speedup": round(ref_ms / ours_ms, 2)})
    return {"kind": "reference GPU build (oracle/_ref/libref_gpu.so: the reference's classes, nvcc -O3 sm_100a, "
                    "device-heap object graph and bvh_node as load_scene builds them; its render loop in 16x16 "
                    "blocks, per-pixel printf left out)", "cases": out}


def cpu_reference_batched(work, every=8, target_s=12.0):
    """The reference's own CPU code on a subsample of the batched workload: every `every`-th scene, a
    deterministic pixel subsample of each image sized to about target_s in total, compat mode (its g++
    build's draw order).  Returns the record (Mpaths/s over the rendered paths)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    ref = oracles.ref_cpu()
    if ref is None:
        return None
    threads = os.cpu_count() or 1
    picked = list(range(0, len(work), every))
    per_scene = target_s / max(len(picked), 1)
    paths = 0
    secs = 0.0
    px_total = 0
    for k in picked:
        sc, p0 = work[k]
        p = p0.__class__(**{**p0.__dict__, "mode": MODE_COMPAT, "draw_order": DRAW_ORDER_HOST})
        rs = ref.scene(sc)
        npix = p.width * p.height
        probe = np.arange(0, npix, max(1, npix // 512), dtype=np.int64)
        t = time.perf_counter()
        rs.render_pixels(p, probe, threads)
        per_px = max(time.perf_counter() - t, 1e-6) / probe.size
        stride = max(1, int(npix / max(1.0, per_scene / per_px)))
        pix = np.arange(0, npix, stride, dtype=np.int64)
        t = time.perf_counter()
        rs.render_pixels(p, pix, threads)
        secs += time.perf_counter() - t
        paths += pix.size * p.traced_spp
        px_total += pix.size
    return {"value": round(paths / secs / 1e6, 4), "unit": METRIC, "kind": "reference", "cores": threads,
            "sample": f"scenes 0, {every}, ... ({len(picked)} of {len(work)}), {px_total} pixels at each image's spp "
                      f"and depth, compat mode, {secs:.1f} s"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    name = args.config
    scene, params = workload(name)
    vals = []
    rays_rates = []
    info = None
    step_s = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        v, r, info = cpu_reference_rate(scene, params, target_s=args.ref_step_s)
        if it >= args.warmup:
            vals.append(v)
            rays_rates.append(r)
            step_s.append(time.perf_counter() - t0)
    value = float(np.mean(vals))
    # a step is a bounded pixel sample of the frame (the rate is the metric), timed on the host clock
    line = {"metric": METRIC, "value": round(value, 4), "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * float(np.mean(step_s)), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference", "config": describe(name, params, scene),
            "mrays_per_s": round(float(np.mean(rays_rates)), 4),
            "cpu_baseline": {"value": round(value, 4), "unit": METRIC, **info},
            "e2e": {"value": round(value, 4), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if name == "spheres" and not args.no_batched:
        line["batched"] = cpu_reference_batched(configs.batch_workload(args.scenes))
    print(json.dumps(line), flush=True)


def _mode_order(args):
    return (MODE_CLEAN, DRAW_ORDER_DEVICE) if args.mode == "clean" else (MODE_COMPAT, DRAW_ORDER_DEVICE)


def _init_dist(world, local):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return dist


def _max_over_ranks(x, world, device="cuda"):
    """The largest value of `x` over all ranks (the whole job's time is its slowest rank's)."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world, steps, total_ms):
    """Whole-job rate of `world` replicas, each processing `units_per_rank` per step for `steps` steps,
    timed by the slowest rank's total (ms): millions of units per second."""
    return units_per_rank * world * steps / (total_ms / 1e3) / 1e6


def fp64_references(work, px_per_scene=128, mult=16, seed_offset=7919):
    """Converged references for the RMSE of the batched workload: the double-precision clean-mode
    estimator (oracle/fp64_clean.c) on a deterministic subsample of `px_per_scene` pixels of every image,
    at `mult` x that image's spp, with a seed independent of the renders'.  Returns [(pixels, mean
    radiance (n, 3))] per image, or None when the oracle is not built."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracles
    from concurrent.futures import ThreadPoolExecutor
    f = oracles.fp64()
    if f is None:
        return None
    workers = min(8, os.cpu_count() or 1)
    threads = max(1, (os.cpu_count() or 1) // workers)

    def one(k):
        sc, p = work[k]
        npx = p.width * p.height
        pix = np.arange(0, npx, max(1, npx // px_per_scene), dtype=np.int64)[:px_per_scene]
        out = f.render(sc, p.width, p.height, p.spp * mult, p.max_depth, (p.seed + seed_offset) & 0xFFFFFFFF, pix,
                       threads=threads)
        return pix, out / float(p.spp * mult)

    with ThreadPoolExecutor(max_workers=workers) as ex:
        return list(ex.map(one, range(len(work))))


def relative_rmse(images, refs, params):
    """sqrt(mean squared error) / sqrt(mean square) of the per-pixel mean radiance over the sampled pixels of
    every image (linear RGB; a non-finite pixel counts as 0)."""
    num = den = 0.0
    for img, (pix, ref), p in zip(images, refs, params):
        x = img.reshape(-1, 4)[pix, :3].astype(np.float64) / float(p.spp)
        x = np.where(np.isfinite(x), x, 0.0)
        num += float(((x - ref) ** 2).sum())
        den += float((ref ** 2).sum())
    return float(np.sqrt(num / max(den, 1e-30)))


def batched_record(ctx, work, dss, mode, groups, warmup, steps, stream, flush, slots=0, drain=0, bvh="2",
                   autotune=False, refs=None, launchgpu=False):
    """One batch of all the workload's images per step (rtc_render_batch, CUDA-graph replay) against the
    plain one-image-per-launch forms with every scene resident: the wavefront engine and the megakernel
    (one thread per pixel, the reference's kernel shape), same mode and parameters.  Device time from CUDA
    events on `stream`, L2 flushed between steps.  With `refs` (fp64_references), the relative RMSE of
    each form's images against the converged references."""
    import torch
    from cortexraytracercuda_b200.renderer import Job
    params = []
    for _, p0 in work:
        p = p0.__class__(**p0.__dict__)
        p.mode, p.draw_order, p.engine = mode, DRAW_ORDER_DEVICE, ENGINE_WAVEFRONT
        if groups:
            p.flags |= FLAG_SAMPLE_GROUPS
        if bvh == "8":
            p.flags |= FLAG_WIDE_BVH
        params.append(p)
    outs = [torch.empty((p.height, p.width, 4), dtype=torch.float32, device="cuda") for p in params]
    plain_outs = [torch.empty_like(o) for o in outs]
    mk_outs = [torch.empty_like(o) for o in outs]
    jobs = [Job(ds, p, o.data_ptr()) for ds, p, o in zip(dss, params, outs)]
    paths = sum(p.width * p.height * p.traced_spp for p in params)
    pixels = sum(p.width * p.height for p in params)
    sp = stream.cuda_stream
    tuned = None
    if autotune:
        from cortexraytracercuda_b200 import autotune as at
        tuned = at.autotune_batch(ctx, jobs, repeats=1, stream=sp)
        jobs = at.with_layout(jobs, tuned.layout)
        slots, drain = tuned.slots, tuned.drain
        torch.cuda.synchronize()

    def batched():
        ctx.render_batch(jobs, slots=slots, drain=drain, stream=sp, batch=tuned.batch if tuned else 0,
                         block=tuned.block if tuned else 0)

    def plain():
        for ds, p, o in zip(dss, params, plain_outs):
            ds.render_device(p, o.data_ptr(), stream=sp)

    mk_params = [p.__class__(**{**p.__dict__, "engine": ENGINE_MEGAKERNEL}) for p in params]

    def plain_megakernel():
        for ds, p, o in zip(dss, mk_params, mk_outs):
            ds.render_device(p, o.data_ptr(), stream=sp)

    def timed(fn, n):
        evs = []
        for k in range(n):
            flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    for _ in range(warmup):
        batched()
    plain()
    plain_megakernel()
    torch.cuda.synchronize()
    stats = []
    b_ms = timed(lambda: (batched(), stats.append(ctx.last_stats())), steps)
    p_steps = max(1, min(steps, 2))
    p_ms = timed(plain, p_steps)
    m_ms = timed(plain_megakernel, 1)
    value = paths * steps / (float(np.sum(b_ms)) / 1e3) / 1e6
    plain_value = paths * p_steps / (float(np.sum(p_ms)) / 1e3) / 1e6
    mk_value = paths / (m_ms[0] / 1e3) / 1e6
    # the same images: bit-identical pixels and image-mean agreement of batched vs plain
    same, mean_dev = [], []
    for o, q in zip(outs, plain_outs):
        a, b = o[..., :3].double().nan_to_num(), q[..., :3].double().nan_to_num()
        same.append(float((a == b).all(-1).float().mean()))
        mean_dev.append(float((a.mean() - b.mean()).abs() / b.mean().clamp_min(1e-9)))
    # end to end: the batch with every image copied to pinned host memory
    host = [torch.empty(o.shape, dtype=torch.float32, pin_memory=True) for o in outs]
    e2e = []
    for k in range(warmup + steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        batched()
        for h, o in zip(host, outs):
            h.copy_(o, non_blocking=True)
        torch.cuda.synchronize()
        if k >= warmup:
            e2e.append(time.perf_counter() - t)
    import ctypes as C
    from cortexraytracercuda_b200.scene import rtc_job
    rec = {"value": round(value, 3), "unit": METRIC, "ms_per_step": round(float(np.mean(b_ms)), 3),
           "steps": steps, "warmup": warmup,
           "mode": ("clean, sample groups" if groups else "clean") if mode == MODE_CLEAN else "compat",
           "workload": f"{len(work)} scenes, {pixels} pixels, {paths} paths per step",
           "slots": slots or "default", "drain": drain or "default",
           "plain_wavefront": {"value": round(plain_value, 3), "ms_per_step": round(float(np.mean(p_ms)), 3),
                               "form": "one rtc_render_device per image, wavefront engine, scene resident"},
           "plain_megakernel": {"value": round(mk_value, 3), "ms_per_step": round(m_ms[0], 3),
                                "form": "one rtc_render_device per image, megakernel (one thread per pixel, the "
                                        "reference's kernel shape), scene resident"},
           "batched_over_plain_wavefront": round(value / plain_value, 3),
           "batched_over_plain_megakernel": round(value / mk_value, 3),
           "equal_to_plain_wavefront": {"bit_identical_pixels_min": round(min(same), 4),
                                        "image_mean_rel_dev_max": round(max(mean_dev), 6)},
           "gpu_launches": int(sum(st["launches"] for st in stats)),
           "iterations": int(np.mean([st["iterations"] for st in stats])),
           "e2e": {"value": round(paths * steps / float(np.sum(e2e)) / 1e6, 3), "unit": METRIC,
                   "h2d_bytes_per_step": len(jobs) * C.sizeof(rtc_job), "d2h_bytes_per_step": pixels * 16}}
    if refs is not None:
        imgs = lambda lst: [o.cpu().numpy() for o in lst]   # noqa: E731
        px = len(refs[0][0])
        rec["rmse_vs_fp64"] = {
            "batched": round(relative_rmse(imgs(outs), refs, params), 5),
            "plain_wavefront": round(relative_rmse(imgs(plain_outs), refs, params), 5),
            "plain_megakernel": round(relative_rmse(imgs(mk_outs), refs, params), 5),
            "definition": f"relative RMSE of per-pixel mean linear RGB over {px} pixels of each of the {len(work)} "
                          "images (every (W*H/px)-th pixel) against oracle/fp64_clean.c at 16x each image's spp, "
                          "independent seed"}
    if launchgpu:
        # the reference's per-call pattern (launchGPU builds and uploads its world for every image):
        # rtc_scene_create + rtc_render with a host buffer + destroy, per image, one pass
        from cortexraytracercuda_b200._lib import check
        from cortexraytracercuda_b200.renderer import DeviceScene
        t = time.perf_counter()
        for (sc, _), p in zip(work, params):
            host_img = np.empty((p.height, p.width, 4), np.float32)
            d2 = DeviceScene(ctx, sc)
            pc = p.to_c()
            check(ctx.lib.rtc_render(ctx.handle, d2.handle, C.byref(pc), host_img.ctypes.data, None))
            d2.close()
        l_s = time.perf_counter() - t
        rec["plain_launchgpu"] = {"value": round(paths / l_s / 1e6, 3), "ms_per_step": round(l_s * 1e3, 1),
                                  "form": "per image: rtc_scene_create (host BVH + upload) + rtc_render to a host "
                                          "buffer + destroy, as launchGPU rebuilds its world per call"}
        rec["batched_over_plain_launchgpu"] = round(value / (paths / l_s / 1e6), 3)
    if tuned:
        rec["autotune"] = {"chosen": {"slots": tuned.slots, "batch": tuned.batch, "drain": tuned.drain,
                                      "layout": tuned.layout, "block": tuned.block},
                           "search": "coordinate descent",
                           "candidates_ms": [[c, round(ms, 1)] for c, ms in tuned.table]}
    del outs, plain_outs, mk_outs
    return rec


def run_batched(args, rank, world, local):
    """64 heterogeneous images per step: one rtc_render_batch call vs one plain launch per image."""
    import torch
    from cortexraytracercuda_b200.renderer import Context, DeviceScene
    dist = _init_dist(world, local)
    mode, _ = _mode_order(args)
    ctx = Context(local)
    work = configs.batch_workload(args.scenes)
    t0 = time.perf_counter()
    dss = [DeviceScene(ctx, sc) for sc, _ in work]
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    refs = fp64_references(work) if args.rmse else None
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    rec = batched_record(ctx, work, dss, mode, args.groups, args.warmup, args.steps, stream, flush, args.slots,
                         args.drain, args.bvh, args.autotune, refs, launchgpu=True)
    clk = clocks.stop()
    b_tot = _max_over_ranks(rec["ms_per_step"] * args.steps, world)
    value = rec["value"] * world * (rec["ms_per_step"] * args.steps) / b_tot
    line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(b_tot / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched: {rec['workload']}",
                       "triangles": int(sum(sc.num_triangles for sc, _ in work)), "mode": rec["mode"],
                       "slots": rec["slots"], "drain": rec["drain"],
                       "l2": "flushed between steps (256 MiB write)", "seed": configs.DEFAULT_SEED,
                       "parallelism": f"replicas x{world}"},
            **{k: v for k, v in rec.items() if k not in ("value", "ms_per_step", "steps", "warmup", "workload", "mode",
                                                         "slots", "drain")},
            "setup_s": round(setup_s, 2), "clocks": clk, "roofline": None, "cpu_baseline": None}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for ds in dss:
        ds.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def _zipf_weights(n, s=1.1):
    w = 1.0 / np.arange(1, n + 1) ** s
    return w / w.sum()


def _percentiles(lat):
    lat = np.asarray(lat, np.float64)
    return {"p50_ms": round(float(np.percentile(lat, 50)), 2), "p95_ms": round(float(np.percentile(lat, 95)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2), "mean_ms": round(float(lat.mean()), 2)}


def served_record(local, work, mode, groups, lambdas, requests, plain_requests, slots=0, seed_offset=0):
    """Poisson request streams through the render server (continuous admission, resident scenes, LRU under
    the HBM budget) against a plain server that renders one request per launch in arrival order, for each
    rate in `lambdas` (1/s).  Latency = completion - submission; Mpaths/s over the stream's span."""
    import torch
    from cortexraytracercuda_b200.renderer import Context, DeviceScene, Job, RenderServer
    order = DRAW_ORDER_DEVICE
    gflags = FLAG_SAMPLE_GROUPS if groups else 0
    srv = RenderServer(local, mode=mode, draw_order=order, slots=slots, flags=gflags)
    t0 = time.perf_counter()
    ids = [srv.add_scene(sc) for sc, _ in work]
    setup_s = time.perf_counter() - t0
    ctx = Context(local)
    dss = [DeviceScene(ctx, sc) for sc, _ in work]   # the plain server's resident scenes
    weights = _zipf_weights(len(work))
    rng = np.random.default_rng(configs.DEFAULT_SEED + seed_offset)
    pools = {}

    def take(shape):
        lst = pools.setdefault(shape, [])
        return lst.pop() if lst else np.empty(shape, np.float32)   # the server stages through pinned memory

    def stream_of(lam, n):
        arr = np.cumsum(rng.exponential(1.0 / lam, n))
        sc = rng.choice(len(work), n, p=weights)
        ang = rng.uniform(0.0, 2.0 * np.pi, n)
        return arr, sc, ang

    def request(sc, ang):
        cam = configs.orbit_camera(work[sc][0].camera, float(ang))
        p = work[sc][1]
        rp = p.__class__(**{**p.__dict__, "mode": mode, "draw_order": order, "engine": ENGINE_WAVEFRONT,
                            "flags": gflags})
        return rp, cam

    # warm-up: every scene once (uploads), not timed
    for k in range(len(work)):
        rp, cam = request(k, 0.0)
        out = take((rp.height, rp.width, 4))
        srv.wait(srv.submit(ids[k], rp, cam, out)[0])
        pools[(rp.height, rp.width, 4)].append(out)
    per_rate = {}
    for lam in lambdas:
        arr, scs, angs = stream_of(lam, requests)
        tickets = []
        lock = threading.Lock()

        def submitter():
            start = time.perf_counter()
            for k in range(len(arr)):
                dt = arr[k] - (time.perf_counter() - start)
                if dt > 0:
                    time.sleep(dt)
                rp, cam = request(scs[k], angs[k])
                with lock:
                    out = take((rp.height, rp.width, 4))
                t, _ = srv.submit(ids[scs[k]], rp, cam, out)
                with lock:
                    tickets.append((t, out, rp.width * rp.height * rp.traced_spp))

        th = threading.Thread(target=submitter)
        th.start()
        lat, first, last, total, k = [], None, 0.0, 0, 0
        while k < len(arr):
            with lock:
                have = len(tickets)
            if k >= have:
                time.sleep(0.0005)
                continue
            t, out, npaths = tickets[k]
            _, info = srv.wait(t)
            with lock:
                pools[tuple(out.shape)].append(out)
            lat.append(info["done_ms"] - info["submit_ms"])
            first = info["submit_ms"] if first is None else min(first, info["submit_ms"])
            last = max(last, info["done_ms"])
            total += npaths
            k += 1
        th.join()
        served = {"requests": len(arr), **_percentiles(lat), "mpaths_per_s": round(total / ((last - first) / 1e3) / 1e6, 3),
                  "offered_mpaths_per_s": round(total / arr[-1] / 1e6, 3)}
        # plain comparison: one launch per request, in arrival order, same stream prefix
        n_plain = min(plain_requests, len(arr))
        plat, ptotal = [], 0
        start = time.perf_counter()
        busy_until = 0.0
        for q in range(n_plain):
            now = time.perf_counter() - start
            if arr[q] > now:
                time.sleep(arr[q] - now)
            rp, cam = request(scs[q], angs[q])
            out = torch.empty((rp.height, rp.width, 4), dtype=torch.float32, device="cuda")
            host = take((rp.height, rp.width, 4))
            ds = dss[int(scs[q])]
            ctx.render_batch([Job(ds, rp, out.data_ptr(), cam)], slots=1 << 20)   # one image per launch
            np.copyto(host, out.cpu().numpy())
            pools[tuple(host.shape)].append(host)
            done = time.perf_counter() - start
            plat.append((done - arr[q]) * 1e3)
            ptotal += rp.width * rp.height * rp.traced_spp
            busy_until = done
        plain = {"requests": n_plain, **_percentiles(plat),
                 "mpaths_per_s": round(ptotal / (busy_until - arr[0]) / 1e6, 3)}
        per_rate[str(int(lam))] = {"served": served, "plain": plain,
                                   "served_over_plain": round(served["mpaths_per_s"] / plain["mpaths_per_s"], 3)}
    st = srv.stats()
    rec = {"mode": ("clean, sample groups" if groups else "clean") if mode == MODE_CLEAN else "compat",
           "workload": f"Poisson streams over {len(work)} batched scenes, Zipf s=1.1, orbit cameras, "
                       f"{requests} requests per rate ({plain_requests} for the plain server)",
           "rates": per_rate, "server": {k: st[k] for k in ("completed", "failed", "scene_uploads", "scene_evictions",
                                                            "peak_resident_bytes", "iterations", "launches")},
           "gpu_launches": int(st["launches"]), "setup_s": round(setup_s, 2), "hbm_budget": "120 GB"}
    srv.close()
    for ds in dss:
        ds.close()
    ctx.close()
    return rec


def run_served(args, rank, world, local):
    """Poisson request streams through the render server vs a plain one-request-per-launch server."""
    dist = _init_dist(world, local)
    mode, _ = _mode_order(args)
    work = configs.batch_workload(args.scenes)
    clocks = ClockSampler(local)
    clocks.start()
    rec = served_record(local, work, mode, args.groups, [float(x) for x in args.lambdas.split(",")], args.requests,
                        args.plain_requests, args.slots, seed_offset=rank)
    clk = clocks.stop()
    top = rec["rates"][max(rec["rates"], key=lambda x: float(x))]
    line = {"metric": METRIC, "value": top["served"]["mpaths_per_s"], "unit": METRIC, "n_gpus": world,
            "steps": len(rec["rates"]), "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"served: {rec['workload']}", "mode": rec["mode"], "slots": args.slots or "default",
                       "hbm_budget": rec["hbm_budget"], "parallelism": f"replicas x{world}", "seed": configs.DEFAULT_SEED},
            "rates": rec["rates"], "server": rec["server"], "gpu_launches": rec["gpu_launches"],
            "e2e": {"value": top["served"]["mpaths_per_s"], "unit": METRIC, "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None, "note": "requests in, radiance in pinned host buffers out"},
            "setup_s": rec["setup_s"], "clocks": clk, "roofline": None, "cpu_baseline": None}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="spheres", choices=["spheres", "cornell", "meshes", "batched", "served"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="compat", choices=["compat", "clean"])
    ap.add_argument("--engine", default="wavefront", choices=["wavefront", "megakernel"])
    ap.add_argument("--bvh", default="2", choices=["2", "8"], help="BVH node layout (binary or 8-wide quantised)")
    ap.add_argument("--builder", default="sah", choices=["sah", "device", "lbvh"],
                    help="BVH builder: host binned SAH, device PLOC, or device linear BVH")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-baseline-s", type=float, default=12.0)
    ap.add_argument("--ref-step-s", type=float, default=8.0)
    ap.add_argument("--small", action="store_true", help="quarter-size frame, 16 spp (profiling captures)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling captures)")
    ap.add_argument("--scenes", type=int, default=64, help="batched/served: number of scenes")
    ap.add_argument("--slots", type=int, default=0, help="batched/served: path slots (0: library default)")
    ap.add_argument("--drain", type=int, default=0, help="batched: drain threshold (0: default, 1: no drain)")
    ap.add_argument("--autotune", action="store_true",
                    help="batched: pick slots / batch / drain / BVH layout with the autotuner before timing")
    ap.add_argument("--groups", action="store_true",
                    help="batched/served, clean mode: split pixels into sample groups (RTC_FLAG_SAMPLE_GROUPS)")
    ap.add_argument("--no-batched", action="store_true", help="default line: skip the batched record")
    ap.add_argument("--no-served", action="store_true", help="default line: skip the served record")
    ap.add_argument("--no-ref-gpu", action="store_true", help="default line: skip the reference GPU build's timings")
    ap.add_argument("--no-rmse", action="store_true", help="skip the RMSE against the fp64 oracle")
    ap.add_argument("--served-requests", type=int, default=100, help="default line: served requests at 200/s")
    ap.add_argument("--served-plain-requests", type=int, default=100,
                    help="default line: requests of the plain server (the same stream prefix as the served form)")
    ap.add_argument("--lambdas", default="20,50,200,800", help="served: request rates (1/s)")
    ap.add_argument("--requests", type=int, default=300, help="served: requests per rate")
    ap.add_argument("--plain-requests", type=int, default=120, help="served: requests of the plain comparison")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    args.rmse = not args.no_rmse

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world:
        # one process per GPU: --gpus N is launched by torchrun with N ranks; a mismatch would time and
        # report a different number of replicas than asked for
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; launch N>1 with "
                 f"python -m torch.distributed.run --nproc-per-node {args.gpus} bench.py --gpus {args.gpus}")

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.config == "batched":
        run_batched(args, rank, world, local)
        return
    if args.config == "served":
        run_served(args, rank, world, local)
        return

    import torch
    import torch.distributed as dist
    from cortexraytracercuda_b200.renderer import Context, DeviceScene

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    ctx = Context(local)
    scene, params = workload(args.config)
    if args.mode == "clean":
        params.mode = MODE_CLEAN
        if args.groups:
            params.flags |= FLAG_SAMPLE_GROUPS
    if args.small:
        params.width, params.height, params.spp = params.width // 4, params.height // 4, 16
    params.engine = ENGINE_WAVEFRONT if args.engine == "wavefront" else ENGINE_MEGAKERNEL
    if args.bvh == "8":
        params.flags |= FLAG_WIDE_BVH
    builder = {"sah": BVH_SAH, "device": BVH_DEVICE, "lbvh": BVH_DEVICE_LBVH}[args.builder]
    ds = DeviceScene(ctx, scene, builder)
    info = ds.info()
    W, H = params.width, params.height
    out = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    counters = torch.zeros(8, dtype=torch.int64, device="cuda")
    # a dedicated stream: the kernels and the CUDA events that time them are on the same stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    def launch(cnt=None):
        ds.render_device(params, out.data_ptr(), None, cnt.data_ptr() if cnt is not None else None, sp)

    # instrumented launch: algorithmic work counters (not timed)
    counters.zero_()
    launch(counters)
    torch.cuda.synchronize()
    rays, paths, nodes, prims, ext_rays, ext_nodes, ext_prims, _ = [int(x) for x in counters.tolist()]
    wavefront = params.engine == ENGINE_WAVEFRONT

    for _ in range(args.warmup):
        flush.fill_(1.0)
        launch()
    torch.cuda.synchronize()
    barrier()

    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(float(k))          # L2 flush between steps (outside the kernel's events)
        ev[k][0].record(stream)
        launch()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    t_wall = time.perf_counter() - t_wall
    step_ms = [a.elapsed_time(b) for a, b in ev]
    clk = clocks.stop()
    launches_per_step = int(ctx.last_stats()["launches"])
    # the per-kernel split, from two more frames with CUDA events around every extend and shade launch
    # (untimed: those events cost ~5 ms of a ~75 ms frame)
    kstats = []
    if wavefront:
        params.flags |= FLAG_KERNEL_TIMING
        for k in range(2):
            flush.fill_(float(k))
            launch()
            kstats.append(ctx.last_stats())
        params.flags &= ~FLAG_KERNEL_TIMING
    kernel_ms = float(np.mean(step_ms))
    total_ms = _max_over_ranks(float(np.sum(step_ms)), world)
    traced = W * H * params.traced_spp
    value = replica_rate(traced, world, args.steps, total_ms)
    mrays = replica_rate(rays, world, args.steps, total_ms)

    # ---- end to end through the C ABI with host buffers ----------------------------------------
    import ctypes as C
    host_out = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True).numpy()
    e2e_ms = []
    for k in range(0 if args.no_e2e else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ds2 = DeviceScene(ctx, scene, builder)
        p = params.to_c()
        from cortexraytracercuda_b200._lib import check
        check(ctx.lib.rtc_render(ctx.handle, ds2.handle, C.byref(p), host_out.ctypes.data, None))
        ds2.close()
        dt = (time.perf_counter() - t0) * 1e3
        if k >= args.warmup:
            e2e_ms.append(dt)
    e2e_total = _max_over_ranks(float(np.sum(e2e_ms)) if e2e_ms else float("nan"), world)
    e2e_value = replica_rate(traced, world, args.steps, e2e_total)

    # ---- roofline -------------------------------------------------------------------------------
    peak, peak_kind = hbm_peak()
    prim_b = PRIM_BYTES[args.config]
    node_b = NODE_BYTES if args.bvh == "2" else NODE8_BYTES
    if wavefront:
        # dominant kernel: wf_extend (closest-hit traversal of every queued ray).  Algorithmic bytes of
        # its launches in one frame, from its own counters, over its summed CUDA-event time.
        ext_ms = float(np.mean([st["extend_ms"] for st in kstats]))
        ext_launches = int(np.mean([st["extend_launches"] for st in kstats]))
        ext_bytes = ext_nodes * node_b + ext_prims * prim_b + ext_rays * EXTEND_STATE_BYTES
        achieved = ext_bytes / (ext_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": "rtc::wf_extend", "launches_per_frame": ext_launches,
                "alg_bytes_per_launch": int(ext_bytes / max(ext_launches, 1)),
                "avg_launch_ms": round(ext_ms / max(ext_launches, 1), 4), "kernel_ms_per_frame": round(ext_ms, 3),
                "share_of_frame": round(ext_ms / float(np.mean([st["bulk_ms"] + st["drain_ms"] for st in kstats])), 3),
                "per_frame": {"rays": ext_rays, "node_visits": ext_nodes, "prim_tests": ext_prims},
                "bytes_per_ray": round(ext_bytes / max(ext_rays, 1), 1),
                "frame": {"shade_ms": round(float(np.mean([st["shade_ms"] for st in kstats])), 3),
                          "drain_ms": round(float(np.mean([st["drain_ms"] for st in kstats])), 3),
                          "iterations": int(np.mean([st["iterations"] for st in kstats])),
                          "rays": rays, "paths": paths, "node_visits": nodes, "prim_tests": prims}}
    else:
        alg_bytes = nodes * node_b + prims * prim_b + rays * STATE_BYTES
        achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "kernel": "rtc::rtc_render_compat" if params.mode == MODE_COMPAT else "rtc::rtc_render_clean",
                "alg_bytes_per_launch": int(alg_bytes), "kernel_ms": round(kernel_ms, 3),
                "per_launch": {"rays": rays, "paths": paths, "node_visits": nodes, "prim_tests": prims},
                "bytes_per_ray": round(alg_bytes / max(rays, 1), 1)}
    # the issue side of the same kernel: algorithmic FP32 flops over the FP32 SIMT peak at the sampled clock
    # (SMs x 128 lanes x 2 flops x f_SM)
    import torch as _t
    sms = _t.cuda.get_device_properties(local).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    fp32_peak = sms * 128 * 2 * mhz * 1e6 / 1e12
    if wavefront:
        flops = ext_nodes * NODE_FLOPS + ext_prims * PRIM_FLOPS[args.config]
        t_s = ext_ms / 1e3
    else:
        flops = nodes * NODE_FLOPS + prims * PRIM_FLOPS[args.config]
        t_s = kernel_ms / 1e3
    roof["flops"] = {"achieved": round(flops / t_s / 1e12, 3), "peak": round(fp32_peak, 1), "unit": "TFLOP/s",
                     "frac": round(flops / t_s / 1e12 / fp32_peak, 4),
                     "peak_source": f"FP32 SIMT: {sms} SMs x 128 x 2 x {mhz:.0f} MHz",
                     "per_visit": {"node": NODE_FLOPS, "prim": PRIM_FLOPS[args.config]}}
    if wavefront:
        roof.update(kernel_bounds(args.config, peak, kstats, ext_rays, roof))

    line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**describe(args.config, params, scene), "parallelism": f"replicas x{world}",
                       "bvh_nodes": info["num_nodes"], "bvh_layout": "binary" if args.bvh == "2" else "8-wide quantised",
                       "bvh_builder": {BVH_SAH: "host SAH", BVH_DEVICE: "device PLOC",
                                       BVH_DEVICE_LBVH: "device LBVH"}[info["bvh_builder"]],
                       "scene_build_ms": round(info["build_ms"], 1)},
            "mrays_per_s": round(mrays, 3),
            "gpu_launches": launches_per_step * args.steps,
            "e2e": {"value": round(e2e_value, 3), "unit": METRIC, "h2d_bytes_per_step": int(info["device_bytes"]),
                    "d2h_bytes_per_step": int(W * H * 16), "ms_per_step": round(e2e_total / args.steps, 3)},
            "roofline": roof, "clocks": clk, "wall_s": round(t_wall, 3)}

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, r, inf = cpu_reference_rate(scene, params, target_s=args.cpu_baseline_s)
        line["cpu_baseline"] = {"value": round(v, 4), "unit": METRIC, **inf, "mrays_per_s": round(r, 4)}
    ds.close()
    # ---- the batched form (64 scenes), the served form (request streams) and the reference's GPU build, one GPU only ----
    if world == 1 and args.config == "spheres" and not args.small:
        extra_clk = ClockSampler(local)
        extra_clk.start()
        if not args.no_batched:
            work = configs.batch_workload(args.scenes)
            t0 = time.perf_counter()
            bdss = [DeviceScene(ctx, sc) for sc, _ in work]
            setup_s = time.perf_counter() - t0
            refs = None if args.no_rmse else fp64_references(work)
            bsteps = max(1, min(args.steps, 3))
            line["batched"] = {
                "config": "batched: 64 seeded scenes (1K-500K triangles, 256^2..1024^2, spp 4/16/64, depth 8-32)",
                "scene_setup_s": round(setup_s, 2),
                "compat": batched_record(ctx, work, bdss, MODE_COMPAT, False, args.warmup, bsteps, stream, flush,
                                         refs=refs),
                "clean_groups": batched_record(ctx, work, bdss, MODE_CLEAN, True, args.warmup, bsteps, stream, flush,
                                               refs=refs)}
            for d in bdss:
                d.close()
            del bdss
        if not args.no_served:
            work = configs.batch_workload(args.scenes)
            line["served"] = {
                "compat": served_record(local, work, MODE_COMPAT, False, [200.0], args.served_requests,
                                        args.served_plain_requests),
                "clean_groups": served_record(local, work, MODE_CLEAN, True, [200.0], args.served_requests,
                                              args.served_plain_requests)}
        if not args.no_ref_gpu:
            line["gpu_baseline"] = ref_gpu_baseline(ctx, stream)
        line["clocks_extra_legs"] = extra_clk.stop()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
