#!/usr/bin/env python
"""Throughput of the B200 render device on the large plain-render workload.

Workload (the configuration the headline metric is quoted on): the seeded terrain scene of
prt_scenes.terrain() -- a 1024x1024 fBm heightfield plus 400 icospheres, 2,605,058
triangles, four material kinds (Lambert, GGX gold-like conductor, rough glass, rough coat over
Lambert) under the reference's sun-sky model -- rendered at 1920x1080, 64 spp, max depth 8,
Russian roulette from depth 3. One step = one 64-spp frame of that workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: Mrays/s = (closest + shadow rays traced) / device time, the reference's `mray`
(render/path_renderer_stream.h:175). Timing: CUDA events on the device's stream, barrier and
synchronize on both sides, max over ranks. The BVH (149 MB) and the path state (GBs) exceed the
126 MB L2, so no flush is needed between steps. One process per GPU: each rank renders its own
replica of the frame (independent sampler seed); there is no collective on the data path.
"""
import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "oidn-protoray_b200"))

import numpy as np  # noqa: E402

import prt_scenes  # noqa: E402
import prt_types as T  # noqa: E402

METRIC = "Mrays/s (closest + shadow rays per second), terrain workload"
UNIT = "Mrays/s"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--inverse-steps", type=int, default=100,
                    help="Adam steps of the batched inverse-rendering measurement (the workload's 100)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the small-scene, batched and adjoint measurements")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched measurement (64-frame batch against 64 frame-form renders) and "
                         "print it as one JSON line, for profiling it")
    ap.add_argument("--traffic-csv", default=None,
                    help="ncu --csv --print-units base log (dram__bytes_read.sum, dram__bytes_write.sum) of the "
                         "kTrace launches of a 1-spp frame of this workload, to measure roofline.traffic instead "
                         "of using the recorded figure")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        rows = [r.split(",") for r in open(self.tmp.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for name, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(min_seconds=10.0):
    """The reference's own CPU path (oracle/_ref, compiled from the reference sources) on a
    bounded sample of the same workload: full-resolution 1-spp frames of the terrain scene,
    after one warm-up frame, until at least `min_seconds` of render time; all host threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref  # test infrastructure: the CPU-baseline leg only

    if not ref.ref_available():
        return None
    scene = prt_scenes.terrain()
    dev = ref.RefDevice(scene, seed=0)
    dev.render(1)  # warm-up frame
    rays, secs, frames = 0.0, 0.0, 0
    while secs < min_seconds:
        st = dev.render(1)
        rays += st["rays"]
        secs += st["seconds"]
        frames += 1
    dev.close()
    return {"value": rays / 1e6 / secs, "unit": UNIT, "cores": ref.hardware_threads(),
            "kind": "reference",
            "sample": f"{frames} frames of the terrain workload at 1920x1080 x 1 spp (samples 1..{frames} of the "
                      f"64-spp frame) after 1 warm-up frame ({rays / 1e6:.1f}M rays in {secs:.1f} s); reference "
                      f"pathStream renderer compiled from its sources, oracle CPU BVH in place of Embree (not installed)"}


class Ranks:
    """Process-group plumbing of the replica runs: barrier, max and sum over ranks (a no-op
    with one process). `device` is where the reduction tensor lives ("cuda:N" for NCCL, "cpu"
    for gloo)."""

    def __init__(self, pg, device):
        self.pg = pg
        self.device = device

    @classmethod
    def init(cls, backend, local_rank, timeout_s=120):
        import torch
        import torch.distributed as torch_dist
        from datetime import timedelta

        device = "cpu"
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
            device = f"cuda:{local_rank}"
        torch_dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
        return cls(torch_dist, device)

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()

    def _reduce(self, x, op):
        if self.pg is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return x if self.pg is None else self._reduce(x, self.pg.ReduceOp.MAX)

    def sum(self, x):
        return x if self.pg is None else self._reduce(x, self.pg.ReduceOp.SUM)


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import ref

    if not ref.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libprt_ref.so is not built"}))
        return
    scene = prt_scenes.terrain()
    dev = ref.RefDevice(scene, seed=0)
    for _ in range(args.warmup):
        dev.render(1)
    rays, secs = 0.0, 0.0
    for _ in range(args.steps):
        st = dev.render(1)
        rays += st["rays"]
        secs += st["seconds"]
    dev.close()
    value = rays / 1e6 / secs
    cores = ref.hardware_threads()
    sample = ("each step = one 1920x1080 x 1-spp frame of the terrain workload (a bounded sample of the "
              "64-spp frame); reference pathStream + sobolBurley compiled from its sources; oracle CPU BVH in "
              "place of Embree (not installed)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded terrain scene)",
        "config": {"workload": "terrain 2.6M tris, 1920x1080, 1 spp per step, depth 8, rr 3, sun-sky",
                   "flush": "inputs larger than L2 not applicable (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# The sun-sky products (sun radiance and angle, sky image) of the terrain's sun-sky light, made
# by the reference's SunSkyLight for (elevation 30 deg, turbidity 3, ground albedo 0.2); the
# application side of the device computes them once per light and passes them in.
SUNSKY_PRODUCTS = ROOT / "tests" / "golden" / "sunsky_t3_e30.npz"


def register_sunsky():
    z = np.load(SUNSKY_PRODUCTS)
    prt_scenes.register_sunsky_products(z["params"], z["sun_color"], float(z["sun_angle"]), z["sky"])


def run_ours(args):
    rank, world, local = dist_info()
    import prt_cuda

    register_sunsky()

    ranks = Ranks.init("nccl", local) if world > 1 else Ranks(None, None)
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum
    pg = ranks.pg

    scene = prt_scenes.terrain(spp=args.spp)
    dev = prt_cuda.DeviceCuda(local)
    dev.setup(scene, seed=rank)

    # Traversal counts per ray (counting variant of the kernels, one 1-spp frame, untimed).
    dev.set_profiling(T.PRT_PROFILE_COUNTS)
    c = dev.render(1)
    n_closest = c["closest_nodes"] / max(c["closest_rays"], 1)
    t_closest = c["closest_tris"] / max(c["closest_rays"], 1)
    n_shadow = c["shadow_nodes"] / max(c["shadow_rays"], 1)
    t_shadow = c["shadow_tris"] / max(c["shadow_rays"], 1)
    dev.set_profiling(T.PRT_PROFILE_KERNELS)

    for _ in range(args.warmup):
        dev.render(args.spp)
    barrier()
    dev.clear_frame()
    sampler = ClockSampler(local)
    sampler.start()
    ms = rays = closest = shadow = trace_ms = shadow_ms = shade_ms = launches = trace_launches = 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = dev.render(args.spp)
        ms += st["render_ms"]
        rays += st["rays"]
        closest += st["closest_rays"]
        shadow += st["shadow_rays"]
        trace_ms += st["trace_ms"]
        shadow_ms += st["shadow_ms"]
        shade_ms += st["shade_ms"]
        launches += st["kernel_launches"]
        trace_launches += st["trace_launches"]
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    barrier()
    ms_max = max_over_ranks(ms)
    total_rays = sum_over_ranks(rays)
    value = total_rays / 1e6 / (ms_max * 1e-3)
    samples_per_s = sum_over_ranks(scene.width * scene.height * args.spp * args.steps) / (ms_max * 1e-3)

    # End to end through the C ABI with host buffers, every step: camera in, 64-spp render,
    # HDR image out into pinned host memory.
    import torch

    dev.set_profiling(0)
    img = torch.empty((scene.height, scene.width, 3), dtype=torch.float32, pin_memory=True).numpy()
    dev._check(dev.lib.prt_cuda_blit(dev.h, T.PRT_BLIT_HDR, T.fptr(img)))  # staging buffer set up once
    e2e_steps = args.steps
    barrier()
    te = time.perf_counter()
    e2e_rays = 0
    for _ in range(e2e_steps):
        dev.init_camera(scene.camera)
        st = dev.render(args.spp)
        e2e_rays += st["rays"]
        dev._check(dev.lib.prt_cuda_blit(dev.h, T.PRT_BLIT_HDR, T.fptr(img)))
    e2e_wall = max_over_ranks(time.perf_counter() - te)
    e2e_value = sum_over_ranks(e2e_rays) / 1e6 / e2e_wall

    # Roofline of the dominant kernel, the closest-hit BVH8 traversal (kTrace, ~60% of the
    # frame): algorithmic bytes per ray B = ray in + hit out + 80 B per node visit + 48 B per
    # triangle test, with the node visits and triangle tests per ray frozen on the reference
    # tree (TERRAIN_PER_RAY), over the kernel's CUDA-event time. The counts of the tree in use
    # are reported beside them. Measured DRAM traffic: the ncu DRAM bytes of one 1-spp frame's
    # kTrace launches (--traffic-csv, or the recorded NCU_TRACE_DRAM_BYTES), per closest ray of
    # that frame, times the closest rays of an average launch here.
    fz = TERRAIN_PER_RAY
    b_closest = 32 + 16 + 80 * fz["closest_nodes"] + 48 * fz["closest_tris"]
    b_shadow = 32 + 4 + 80 * fz["shadow_nodes"] + 48 * fz["shadow_tris"]
    achieved = closest * b_closest / (trace_ms * 1e-3) / 1e9
    per_launch_rays = closest / max(trace_launches, 1)
    traffic_bytes, traffic_note = NCU_TRACE_DRAM_BYTES, "recorded ncu capture (NCU_TRACE_DRAM_BYTES)"
    if args.traffic_csv:
        traffic_bytes = ncu_dram_bytes(args.traffic_csv, "kTrace")
        traffic_note = f"ncu capture of this build ({args.traffic_csv})"
    traffic = traffic_bytes / max(c["closest_rays"], 1) * per_launch_rays
    peak, peak_kind = measured_peaks()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded terrain scene, reference sun-sky model output)",
        "config": {"workload": f"terrain 2.6M tris, 1920x1080, {args.spp} spp per step, depth 8, rr 3, sun-sky",
                   "triangles": scene.tri_count, "flush": "inputs larger than L2 (BVH 148 MB, path state GBs)",
                   "parallelism": f"replicas x{world}"},
        "samples_per_s": samples_per_s,
        "wall_ms_per_step": wall * 1e3 / args.steps,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(C_CAMERA_BYTES),
                "d2h_bytes_per_step": int(img.nbytes)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "kTrace (closest-hit BVH8 traversal + hit binning)",
                     "algorithmic_bytes_per_launch": per_launch_rays * b_closest,
                     "launch_ms": trace_ms / max(trace_launches, 1),
                     "launches_per_step": trace_launches / args.steps,
                     "bytes_per_ray": {"closest": b_closest, "shadow": b_shadow},
                     "per_ray_reference_tree": fz,
                     "per_ray_tree_in_use": {"closest_nodes": n_closest, "closest_tris": t_closest,
                                             "shadow_nodes": n_shadow, "shadow_tris": t_shadow},
                     "traffic_note": "DRAM bytes of a 1-spp frame's kTrace launches, scaled per closest ray: "
                                     + traffic_note},
        "kernel_ms_per_step": {"trace": trace_ms / args.steps, "shadow": shadow_ms / args.steps,
                               "shade": shade_ms / args.steps},
        "rays_per_step": {"closest": closest / args.steps, "shadow": shadow / args.steps},
    }
    if not args.headline_only:
        barrier()
        out["bvh_build"] = bvh_build_bench(dev, scene)
        out["small_scene"] = small_scene_bench(dev)
        out["batched"] = batched_bench(dev)
        out["adjoint"] = adjoint_bench(dev)
        out["inverse_batched"] = inverse_batched_bench(dev, steps=args.inverse_steps)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline()
        except Exception as exc:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    dev.close()
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


# DRAM bytes (read + write) of the 9 kTrace launches of one 1920x1080 x 1-spp terrain frame,
# from ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum.
NCU_TRACE_DRAM_BYTES = 699_916_032

# Node visits and triangle tests per ray on the reference tree of the terrain workload: the host
# binned-SAH BVH8 with the SAH-optimal 8-wide collapse (284,895 nodes, at most 3 triangles per
# leaf), counted by the counting traversal over every closest and shadow ray of one
# 1920x1080 x 1-spp frame. Frozen, so that a worse tree cannot raise the roofline's bytes.
TERRAIN_PER_RAY = {"closest_nodes": 13.004, "closest_tris": 4.300, "shadow_nodes": 12.963, "shadow_tris": 5.543}


def ncu_dram_bytes(path, kernel):
    """Sum of dram__bytes_read.sum + dram__bytes_write.sum over the launches of `kernel` in an
    ncu --csv log (units printed as base units, bytes)."""
    import csv

    with open(path) as f:
        rows = list(csv.reader(line for line in f if line.startswith('"')))
    head = rows[0]
    k_name, k_metric, k_value, k_unit = (head.index(c) for c in ("Kernel Name", "Metric Name", "Metric Value",
                                                                 "Metric Unit"))
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    total = 0.0
    for r in rows[1:]:
        if kernel in r[k_name] and r[k_metric] in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            total += float(r[k_value].replace(",", "")) * scale.get(r[k_unit], 1.0)
    return total

def bvh_build_bench(dev, scene, builds=3, spp=8):
    """BVH8 build of the terrain workload on the host (binned SAH) and on the device (PLOC), the
    reference's buildMs / buildMprim (accel/embree_intersector.cpp:88-90): best of `builds`
    uploads each, wall time of the build alone; then the render speed over each tree (one
    `spp`-sample frame, device-timed) -- the images are identical, the trees differ in quality."""
    out = {"triangles": scene.tri_count}
    for name, builder in (("host", T.PRT_BVH_HOST), ("device", T.PRT_BVH_DEVICE)):
        scene.bvh_build = builder
        best = None
        for _ in range(builds if builder == T.PRT_BVH_DEVICE else 1):
            dev.init_scene(scene)
            st = dev.scene_stats()
            best = st if best is None or st["build_ms"] < best["build_ms"] else best
        dev.setup(scene, seed=0)
        dev.render(1)
        r = dev.render(spp)
        out[name] = {"ms": best["build_ms"], "mprim_s": scene.tri_count / 1e3 / best["build_ms"],
                     "nodes": best["node_count"], "depth": best["depth"], "iterations": best["iterations"],
                     "render_mrays_s": r["mray"]}
    scene.bvh_build = T.PRT_BVH_HOST
    out["note"] = (f"build = wall time of the BVH build inside the scene upload; render = one 1920x1080 x {spp}-spp "
                   "frame over that tree")
    return out


def small_scene_bench(dev, repeats=5):
    """The small plain-render workload: the Cornell-style room with 32 icospheres (10.3k
    triangles), 256x256, 16 spp, max depth 5, seed 0. Best of `repeats` device-timed frames."""
    scene = prt_scenes.cornell(seed=0)
    dev.setup(scene, seed=0)
    dev.set_profiling(T.PRT_PROFILE_COUNTS)
    c = dev.render(1)
    dev.set_profiling(0)
    per_ray = {"closest_nodes": c["closest_nodes"] / max(c["closest_rays"], 1),
               "closest_tris": c["closest_tris"] / max(c["closest_rays"], 1),
               "shadow_nodes": c["shadow_nodes"] / max(c["shadow_rays"], 1),
               "shadow_tris": c["shadow_tris"] / max(c["shadow_rays"], 1)}
    dev.render(scene.spp)
    best = None
    for _ in range(repeats):
        dev.init_sampler(0)
        dev.clear_frame()
        st = dev.render(scene.spp)
        if best is None or st["render_ms"] < best["render_ms"]:
            best = st
    return {"workload": "room + 32 icospheres, 10,252 tris, 256x256, 16 spp, depth 5", "mrays_per_s": best["mray"],
            "samples_per_s": scene.width * scene.height * scene.spp / (best["render_ms"] * 1e-3),
            "ms_per_frame": best["render_ms"], "rays": best["rays"], "per_ray": per_ray,
            "bytes_per_ray": {"closest": 48 + 80 * per_ray["closest_nodes"] + 48 * per_ray["closest_tris"],
                              "shadow": 36 + 80 * per_ray["shadow_nodes"] + 48 * per_ray["shadow_tris"]}}


def batched_bench(dev, count=64, repeats=3):
    """64 independent terrain frames (triangles log-uniform in [1k, 500k], square sizes 64..512,
    spp in {4..64}, depth 3..10, beauty + albedo1 + normal1): one batch render (persistent
    wavefront, path regeneration, graph-captured bounce loop) against 64 frame-form renders of
    the same frames with the same seeds. Device time; scene upload outside both."""
    import prt_cuda

    frames = prt_scenes.batch_frames(count=count, seed=0)
    samples = sum(s.width * s.height * s.spp for s, _, _ in frames)
    batch = prt_cuda.Batch(dev, frames)
    batch.render()
    b_ms, b_rays, launches = None, 0, 0
    for _ in range(repeats):
        st = batch.render()
        if b_ms is None or st["render_ms"] < b_ms:
            b_ms, b_rays, launches = st["render_ms"], st["rays"], st["kernel_launches"]
    batch.close()
    p_ms, p_rays = 0.0, 0
    for scene, seed, aov in frames:
        dev.init_scene(scene)
        dev.init_frame(scene.width, scene.height, aov)
        dev.init_camera(scene.camera)
        dev.init_renderer(scene.max_depth, scene.rr_depth)
        dev.init_sampler(seed)
        dev.render(scene.spp)  # warm-up (path state allocation)
        dev.init_sampler(seed)
        dev.clear_frame()
        st = dev.render(scene.spp)
        p_ms += st["render_ms"]
        p_rays += st["rays"]
    return {"workload": f"{count} terrain frames, {sum(s.tri_count for s, _, _ in frames):,} tris in total, "
                        f"{samples:,} pixel-samples, 3 AOVs",
            "batched_ms": b_ms, "plain_ms": p_ms, "speedup": p_ms / b_ms,
            "batched_mrays_per_s": b_rays / 1e6 / (b_ms * 1e-3), "plain_mrays_per_s": p_rays / 1e6 / (p_ms * 1e-3),
            "batched_samples_per_s": samples / (b_ms * 1e-3), "rays_equal": b_rays == p_rays,
            "batched_kernel_launches": launches}


def adjoint_bench(dev, repeats=3):
    """Inverse-rendering workload: the room with textured floor and back wall (256^2 RGB
    albedo textures) and rough specular spheres, 256x256, 16 spp per gradient. Cost of one
    path-replay adjoint (all texel and roughness gradients) against one forward render."""
    scene, params = prt_scenes.cornell_inverse(seed=0)
    dev.setup(scene, seed=0)
    dl = np.full((scene.height, scene.width, 3), 1e-3, np.float32)
    dev.render(scene.spp)
    dev.adjoint(dl, scene.spp)
    f_ms = a_ms = None
    for _ in range(repeats):
        dev.init_sampler(0)
        dev.clear_frame()
        f = dev.render(scene.spp)["render_ms"]
        a = dev.adjoint(dl, scene.spp)[2]["render_ms"]
        f_ms = f if f_ms is None else min(f_ms, f)
        a_ms = a if a_ms is None else min(a_ms, a)
    n_params = sum(int(scene.textures[t].size) for t in params["textures"]) + len(params["roughness"])
    return {"workload": "room, 2 x 256^2 RGB albedo textures + 32 roughnesses, 256x256, 16 spp",
            "forward_ms": f_ms, "adjoint_ms": a_ms, "cost_ratio": a_ms / f_ms,
            "gradients_per_s": 1e3 / a_ms, "parameters": n_params}


def inverse_batched_bench(dev, count=16, steps=100, lr=1e-2):
    """Batched differentiable workload: 16 terrain inverse-rendering problems (100k-1M
    triangles, 512x512, 16 spp, depth 6), each optimising a 512^2 RGB albedo texture on its
    terrain and the roughness of every sphere against a target render (L2 loss). One step =
    push parameters, batched forward of all 16 (one persistent wavefront), images blitted into torch tensors,
    batched path-replay adjoint of all 16 (one persistent wavefront), Adam update (torch,
    lr 1e-2). Compared with the same step done as 16 sequential frame-form renders and
    adjoints. Wall time per step; scene upload outside both."""
    import torch
    import prt_cuda

    probs = prt_scenes.batch_inverse_frames(count=count, seed=0)
    targets = prt_scenes.batch_inverse_frames(count=count, seed=0, target=True)
    batch = prt_cuda.Batch(dev, [(s, seed, 0) for s, _, seed in probs])
    batch.enable_adjoint()

    def push(k, tex, rough, push_batch=True):
        s, params, _ = probs[k]
        mats = []
        for j, m in enumerate(params["roughness"]):
            mat = T.Material.from_buffer_copy(s.materials[m])
            mat.specular_roughness = float(rough[j])
            mats.append(mat)
        first = params["roughness"][0]
        if push_batch:
            batch.update_texture(k, params["textures"][0], tex)
            batch.update_materials(k, first, mats)
        else:
            dev.update_texture(params["textures"][0], tex)
            dev.update_materials(first, mats)

    # Target images: the target parameters pushed into the same batch, then the initial ones.
    for k in range(count):
        ts, tp, _ = targets[k]
        push(k, ts.textures[tp["textures"][0]],
             [ts.materials[m].specular_roughness for m in tp["roughness"]])
    batch.render()
    target_imgs = [torch.from_numpy(batch.blit(k)).cuda() for k in range(count)]
    tex = [torch.from_numpy(s.textures[p["textures"][0]].copy()).cuda().requires_grad_(True) for s, p, _ in probs]
    rough = [torch.tensor([s.materials[m].specular_roughness for m in p["roughness"]], device="cuda",
                          requires_grad=True) for s, p, _ in probs]
    opt = torch.optim.Adam(tex + rough, lr=lr)
    gts = [torch.zeros(t.numel(), device="cuda") for t in tex]
    grs = [torch.zeros(len(s.materials), device="cuda") for s, _, _ in probs]

    def step_batched():
        for k in range(count):
            push(k, tex[k].detach(), rough[k].detach().cpu().numpy())
        batch.render()
        imgs = [batch.blit(k, out=torch.empty_like(target_imgs[k])) for k in range(count)]
        dls = [2.0 * (imgs[k] - target_imgs[k]) for k in range(count)]
        batch.adjoint(dls, gts, grs)
        loss = sum(float(((imgs[k] - target_imgs[k]) ** 2).sum()) for k in range(count))
        opt.zero_grad()
        for k in range(count):
            s, p, _ = probs[k]
            tex[k].grad = gts[k].view_as(tex[k])
            rough[k].grad = grs[k][p["roughness"]].clone()
        opt.step()
        with torch.no_grad():
            for k in range(count):
                tex[k].clamp_(0.01, 1.0)
                rough[k].clamp_(0.01, 1.0)
        return loss

    losses = [step_batched()]  # warm-up (graph capture)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        losses.append(step_batched())
    torch.cuda.synchronize()
    batched_s = (time.perf_counter() - t0) / steps
    batch.close()

    # The same step as 16 sequential frame-form runs (upload of each scene outside the timing).
    seq_s = 0.0
    for k in range(count):
        s, p, seed = probs[k]
        dev.setup(s, seed=seed)
        push(k, tex[k].detach(), rough[k].detach().cpu().numpy(), push_batch=False)
        dev.render(s.spp)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        push(k, tex[k].detach(), rough[k].detach().cpu().numpy(), push_batch=False)
        dev.init_sampler(seed)
        dev.clear_frame()
        dev.render(s.spp)
        img = dev.blit_frame(out=torch.empty_like(target_imgs[k]))
        dl = 2.0 * (img - target_imgs[k])
        gt = torch.zeros(tex[k].numel(), device="cuda")
        gr = torch.zeros(len(s.materials), device="cuda")
        dev.adjoint(dl.contiguous(), s.spp, first_sample=0, grad_textures=gt, grad_roughness=gr)
        torch.cuda.synchronize()
        seq_s += time.perf_counter() - t0
    return {"workload": f"{count} terrain inverse problems, {sum(s.tri_count for s, _, _ in probs):,} tris, 512x512, "
                        f"16 spp, depth 6, 512^2 texture + sphere roughness each",
            "batched_step_s": batched_s, "sequential_step_s": seq_s, "speedup": seq_s / batched_s,
            "batched_gradients_per_s": count / batched_s, "sequential_gradients_per_s": count / seq_s,
            "adam_steps": steps, "loss_first": losses[0], "loss_last": losses[-1]}


C_CAMERA_BYTES = 4 * 14  # prt_camera_desc: 12 floats of basis and position + fov + near clip


def main():
    args = parse_args()
    if args.batched_only:
        import prt_cuda

        register_sunsky()
        print(json.dumps({"batched": batched_bench(prt_cuda.DeviceCuda(0))}))
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
