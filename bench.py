"""Benchmark of the splat rasteriser on B200.

Workload: 1.5M clustered Gaussians (SH degree 3), views at 1920x1080 on a
circular walk of radius 3 around the cloud (vertical fov 60 degrees), 16x16
tiles, black background. One step draws every view of the batch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank draws its own batch of views (weak scaling: the views
are independent, the Gaussians replicated; no collective on the forward path).
Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(count=1_500_000, width=1920, height=1080, views=8, clustered=True, sh_degree=3, vfov=60.0)
METRIC = "fwd+bwd ms/view, 1.5M Gaussians 1080p, batched+BF16 vs plain FP32, err<=1e-4"


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """nvidia-smi sampled every 200 ms over the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_scene(seed: int):
    from athenea_b200 import scenes
    recs, enc = scenes.records(WORKLOAD["count"], WORKLOAD["clustered"], seed, WORKLOAD["sh_degree"])
    return recs, enc


def view_cameras(views: int, first: int = 0):
    import athenea_b200 as A
    from athenea_b200 import scenes
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    out = []
    for v in range(first, first + views):
        eye = scenes.circle_eye(v, max(views, 1) * 4, 3.0, 0.3)
        cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, WORKLOAD["vfov"])
        out.append(cam.projection_for(W, H))
    return out


# ---------------------------------------------------------------------------
def run_ours(args) -> dict | None:
    import torch
    import torch.distributed as dist

    import athenea_b200 as A

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    recs, enc = make_scene(20261203 + 1)
    cloud = A.CloudLoader.upload(torch.from_numpy(recs.reshape(-1)).to(dev), enc, 3)
    del recs
    torch.cuda.empty_cache()
    V = WORKLOAD["views"]
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    projs = view_cameras(V, first=rank * V)
    raster = A.TileRasterizer.create()
    settings = A.RenderSettings(width=W, height=H)
    targets = [A.RenderTargets.make(W, H, device=dev) for _ in range(V)]
    inst = [A.SplatInstance(cloud)]
    stream = torch.cuda.current_stream(dev)

    def step():
        for v in range(V):
            raster.render(projs[v], inst, settings, targets[v], stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()
    ms_per_step = ms / args.steps
    views_total = V * world

    # e2e: through the public API from host memory -- each view's camera goes
    # in, its image comes back to pinned host memory.
    host = [torch.empty((W * H, 4), dtype=torch.float32, pin_memory=True) for _ in range(V)]
    e2e_start, e2e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e2e_start.record(stream)
    for _ in range(args.steps):
        for v in range(V):
            raster.render(projs[v], inst, settings, targets[v], stream=stream)
            host[v].copy_(targets[v].colour, non_blocking=True)
    e2e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2e_start.elapsed_time(e2e_end) / args.steps

    # per-stage times of one frame (events between the stages, waited for)
    timed = A.RenderSettings(width=W, height=H, time_stages=True)
    st = raster.render(projs[0], inst, timed, targets[0], stream=stream)
    stages = {"project_ms": st.project_ms, "emit_ms": st.emit_ms, "sort_and_ranges_ms": st.tile_sort_ms,
              "blend_ms": st.blend_ms}
    passes = math.ceil((24 + max(1, math.ceil(math.log2(max(2, ((W + 15) // 16) * ((H + 15) // 16)))))) / 8)
    launches_per_view = 5 + passes   # project, emit, histogram, passes, ranges, blend
    out = dict(ms_per_step=ms_per_step, views=views_total, stats=st, stages=stages, e2e_ms=e2e_ms,
               clocks=clocks.summary(), launches=launches_per_view * V * args.steps,
               sh_words=cloud.sh_words, count=cloud.count, passes=passes)
    if world > 1:
        dist.destroy_process_group()
    return out if rank == 0 else None


def cpu_baseline(threads: int = 0) -> dict:
    """The CPU restatement (oracle/, the reference's method in C++) timed on one view."""
    from oracle import oracle as O
    O.build()
    recs, enc = make_scene(20261203 + 1)
    e = dict(stride=enc["stride"], x=0, y=1, z=2, opacity=enc["opacity"], scale0=enc["scale0"],
             scale1=enc["scale1"], scale2=enc["scale2"], rotW=enc["rot_w"], rotX=enc["rot_x"], rotY=enc["rot_y"],
             rotZ=enc["rot_z"], dc0=enc["dc0"], dc1=enc["dc1"], dc2=enc["dc2"], restBase=enc["rest_base"],
             filePerColour=enc["file_per_colour"])
    pos, shape, sh, _, shw = O.decode(recs.reshape(-1), e, 15)
    del recs
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    from athenea_b200 import scenes
    eye = scenes.circle_eye(0, WORKLOAD["views"] * 4, 3.0, 0.3)
    cam = O.looking_at(eye, (0, 0, 0))
    cam.focal = cam.haperture * ((H * 0.5) / math.tan(math.radians(WORKLOAD["vfov"]) * 0.5)) / W
    proj = O.projection_for(cam, W, H)
    t0 = time.perf_counter()
    out = O.render([(pos, shape, sh, 15, shw, np.eye(4), 0)], proj, W, H, threads=threads)
    dt = time.perf_counter() - t0
    cores = threads or os.cpu_count()
    return dict(ms=dt * 1000.0, cores=cores, evaluated=out["evaluated"], pairs=out["binned"]["pairs"],
                visible=out["binned"]["visible"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--views", type=int, default=WORKLOAD["views"], help="views a GPU draws a step")
    ap.add_argument("--gaussians", type=int, default=WORKLOAD["count"], help="Gaussians in the scene")
    args = ap.parse_args()
    WORKLOAD["views"] = args.views
    WORKLOAD["count"] = args.gaussians
    args.warmup = max(args.warmup, 3)
    rank, world, _ = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return
        runs = []
        for _ in range(args.warmup if args.warmup < 1 else 1):
            cpu_baseline()
        for _ in range(args.steps):
            runs.append(cpu_baseline())
        ms = statistics.median(r["ms"] for r in runs)
        line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms/view", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "clustered-1.5M-1920x1080, forward of one view, CPU restatement",
                           "gaussians": WORKLOAD["count"], "width": WORKLOAD["width"], "height": WORKLOAD["height"]},
                "cpu_baseline": {"value": ms, "unit": "ms/view", "cores": runs[0]["cores"], "kind": "port",
                                 "sample": "one 1920x1080 view of the 1.5M-Gaussian scene, forward"},
                "e2e": {"value": ms, "unit": "ms/view", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    res = run_ours(args)
    if rank != 0 or res is None:
        return
    P = peaks()
    st = res["stats"]
    stages = res["stages"]
    dominant = max(stages, key=stages.get)
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    # algorithmic bytes a launch, per stage (DESIGN.md states each figure)
    per_slot_read = 16 + 16 + 4 * res["sh_words"]
    bytes_ = {
        "project_ms": res["count"] * (per_slot_read + 4 + 4) + st.visible * (48 + 8),
        "emit_ms": st.visible * (48 + 8 + 8) + st.pairs * 12,
        "sort_and_ranges_ms": st.pairs * (8 + 24 * res["passes"] + 8 + 8),
    }
    cpu = None if args.no_cpu else cpu_baseline()
    if dominant == "blend_ms":
        flops = (cpu["evaluated"] if cpu else st.pairs * 256) * 20
        achieved = flops / (stages[dominant] * 1e-3) / 1e12
        fp32_peak = 148 * 128 * 2 * (P.get("sm_max_mhz", 1965.0) * 1e6) / 1e12
        roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak, "traffic": None, "kernel": "blendKernel",
                    "peak_source": "nominal FP32 FMA rate at the measured max SM clock (no FP32 peak is measured)"}
    else:
        achieved = bytes_[dominant] / (stages[dominant] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": P["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / P["hbm_gbs"], "traffic": None, "kernel": dominant,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
    ms_view = res["ms_per_step"] / WORKLOAD["views"]
    line = {
        "metric": METRIC, "value": ms_view, "unit": "ms/view", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no dataset)",
        "config": {"workload": "clustered-1.5M-1920x1080", "gaussians": WORKLOAD["count"], "width": W, "height": H,
                   "views_per_gpu": WORKLOAD["views"], "sh_degree": 3, "tile": 16, "path": "plain forward, FP32",
                   "parallelism": f"views sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (packed Gaussians 186 MB > 126 MB)",
                   "note": "forward only: the backward and the batched/mixed path are not in this measurement"},
        "stages_ms": stages, "visible": st.visible, "pairs": st.pairs,
        "roofline": roofline,
        "e2e": {"value": res["e2e_ms"] / WORKLOAD["views"], "unit": "ms/view", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": W * H * 16 * WORKLOAD["views"]},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["ms"], "unit": "ms/view", "cores": cpu["cores"], "kind": "port",
                                "sample": "one 1920x1080 view of the same scene, forward (project, bin, blend)"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
