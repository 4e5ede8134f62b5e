"""Benchmark of the splat rasteriser's training step on B200.

Workload: 1.5M clustered Gaussians (SH degree 3), 8 views at 1920x1080 a GPU on
a circular walk of radius 3 around the cloud (vertical fov 60 degrees), black
background, mean-L2 loss against targets uniform in [0,1]^3.

The headline `value` is the batched mixed-precision step (forward, loss and
backward of every view, one launch a stage, replayed from a CUDA graph; SH in
BF16 / FP8 e4m3) in ms a view. The plain FP32 path (one differentiable frame, the
loss and the backward a view) runs on the same scene and views and is reported
beside it with the speed-up.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank draws its own views (weak scaling: views are
independent, the Gaussians replicated) and the gradients are summed over ranks
in 4 buckets, each bucket's all-reduce posted on a side stream while the step's
projection adjoint computes the later buckets. Rank 0 prints one JSON line.
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

WORKLOAD = dict(count=1_500_000, width=1920, height=1080, views=8, clustered=True, sh_degree=3, vfov=60.0,
                name="clustered-1.5M-1920x1080", mixed_sizes=False)
# gradient buckets of a multi-GPU step: each bucket's all-reduce overlaps the later buckets' adjoint
BUCKETS = 4
METRIC = "fwd+bwd ms/view, 1.5M Gaussians 1080p, batched+BF16 vs plain FP32, err<=1e-4"


# DRAM bytes a launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# batched kernels, from an ncu capture of this workload at 2 views (tile 32,
# 128 records a batch), scaled by 4 to its 8 views: records and pairs grow
# with the views.
NCU_TRAFFIC: dict = {
    "blendStepKernel": 4 * 147.60e6,
    "projectEmitKernel": 4 * 473.22e6,
}


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "fallback": True}


class ClockSampler:
    """The SM clock, its maximum and the throttle reasons over the timed region: read
    through NVML every 10 ms from a thread (the device found by its UUID, which
    CUDA_VISIBLE_DEVICES does not renumber), or, without NVML, nvidia-smi every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []          # (sm MHz, max sm MHz, {reason names})
        self.stop = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.device)
        uuid = str(getattr(props, "uuid", "") or "")
        if uuid:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            reasons_of = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = [getattr(nv, "nvmlClocksEventReason" + n, getattr(nv, "nvmlClocksThrottleReason" + n, 0))
                    for n in ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
            self.stop = threading.Event()

            def sample():
                while not self.stop.is_set():
                    try:
                        r = reasons_of(h)
                        self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                          nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                                          {self.NAMES[k] for k in range(4) if r & bits[k]}))
                    except Exception:
                        pass
                    self.stop.wait(0.01)

            self.thread = threading.Thread(target=sample, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
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
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if self.thread is None and self.path:
            try:
                for line in open(self.path):
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        self.rows.append((float(parts[1]), float(parts[2]) if parts[2].replace(".", "").isdigit()
                                          else None, {self.NAMES[k] for k in range(4)
                                                      if parts[5 + k].lower().startswith("active")}))
            finally:
                try:
                    os.unlink(self.path)
                except OSError:
                    pass
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        maxima = [m for _, m, _ in self.rows if m]
        return {"sm_mhz": statistics.median(float(r[0]) for r in self.rows),
                "sm_max_mhz": float(max(maxima)) if maxima else None,
                "reasons": sorted(set().union(*(r[2] for r in self.rows))), "samples": len(self.rows),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


def sort_passes(bits: int) -> int:
    """The onesweep's passes over `bits` key bits: eight bits a pass, or nine where that saves a pass."""
    eights, nines = (bits + 7) // 8, (bits + 8) // 9
    return min(eights, nines)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_scene(seed: int):
    from athenea_b200 import scenes
    recs, enc = scenes.records(WORKLOAD["count"], WORKLOAD["clustered"], seed, WORKLOAD["sh_degree"])
    return recs, enc


def view_specs(views: int, first: int = 0):
    """[(projection, width, height)] of views first .. first + views - 1 of the workload's walk."""
    import athenea_b200 as A
    from athenea_b200 import scenes
    total = max(first + views, 1)
    sizes = (scenes.view_sizes(total, scenes.SEED) if WORKLOAD["mixed_sizes"]
             else [(WORKLOAD["width"], WORKLOAD["height"])] * total)
    out = []
    for v in range(first, first + views):
        W, H = sizes[v]
        eye = scenes.circle_eye(v, max(views, 1) * 4, 3.0, 0.3)
        cam = A.pinhole_for_vertical_fov(eye, (0, 0, 0), W, H, WORKLOAD["vfov"])
        out.append((cam.projection_for(W, H), W, H))
    return out


# ---------------------------------------------------------------------------
class PlainTrainer:
    """The plain FP32 path: per view, a differentiable frame (ath_raster_render_params),
    the mean-L2 loss's gradient (ath_l2_loss) and the backward (ath_raster_backward), one
    view after another, gradients added into one set."""

    def __init__(self, params, views, targets_dev, dev):
        import torch
        import athenea_b200 as A
        self.A = A
        self.P = params
        self.views = views
        self.targets = targets_dev
        self.raster = A.TileRasterizer.create()
        self.frames, self.dl = {}, {}
        for _, W, H in views:
            if (W, H) not in self.frames:
                self.frames[(W, H)] = A.RenderTargets.make(W, H, device=dev)
                self.dl[(W, H)] = torch.empty((W * H, 4), dtype=torch.float32, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.grads = params.zeros_like()

    def step(self, stream, targets=None, check=False):
        """One step over every view; `check` waits for each frame (and redraws one whose pairs
        outgrew the handle's capacity), which a warm-up step does so that the capacity covers
        every view before the timed steps, which do not wait."""
        targets = targets if targets is not None else self.targets
        self.loss.zero_()
        for g in (self.grads.means, self.grads.scales, self.grads.quats, self.grads.sh):
            g.zero_()
        stats = None
        for v, (proj, W, H) in enumerate(self.views):
            frames, dl = self.frames[(W, H)], self.dl[(W, H)]
            stats = self.raster.render_params(proj, self.P, self.A.RenderSettings(width=W, height=H), frames,
                                              stream=stream, do_check=check)
            self.A.l2_loss(frames.colour, targets[v], dl, self.loss, stream=stream)
            self.raster.backward(dl, self.grads, stream=stream)
        return stats


def _timed(fn, steps: int, stream, world: int, dev) -> float:
    """K calls of `fn` between CUDA events on `stream`, a barrier and a
    synchronize on both sides; ms per call, max over ranks."""
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms / steps


def run_ours(args) -> dict | None:
    """The batched mixed-precision step (ath_batch_train_step: every view of the
    batch in one launch a stage, the step replayed from a CUDA graph) and, beside
    it, the plain FP32 path one view at a time, on the same scene and views."""
    import torch
    import torch.distributed as dist

    import athenea_b200 as A
    from athenea_b200 import scenes

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    V = WORKLOAD["views"]
    p = scenes.params(WORKLOAD["count"], WORKLOAD["clustered"], 20261203 + 1, WORKLOAD["sh_degree"])
    params = A.Params(*[torch.from_numpy(p[k]).to(dev) for k in ("means", "scales", "quats", "sh")],
                      sh_degree=p["sh_degree"])
    del p
    mixed = A.MixedParams.from_params(params)
    # weak scaling: every rank draws V views of its own, views rank*V .. rank*V + V - 1
    shard = A.shard_views(V * world, rank, world)
    views = view_specs(len(shard), first=shard.start)
    pixel_base = np.cumsum([0] + [W * H for _, W, H in views])
    gen = torch.Generator().manual_seed(20261203 + 7 + rank)
    host_target = torch.rand((int(pixel_base[-1]), 3), generator=gen).pin_memory()
    target = host_target.to(dev)
    stream = torch.cuda.current_stream(dev)

    # ---- the batched mixed-precision step ----------------------------------
    bt = A.BatchTrainer()
    bt.set_views(views)
    colour = torch.empty((bt.pixels, 4), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    # the gradients in one flat buffer; on more than one GPU they are summed over
    # ranks (every rank's views) bucket by bucket, each bucket's all-reduce posted on
    # a side stream as soon as the step's projection adjoint has finished it
    grads = A.GradientBuffer(params.count, int(params.sh.shape[1]), params.sh_degree, device=dev).params
    if args.tile:
        bt.set_tuning(args.tile, args.block_batch)
        tuned = {"tile": args.tile, "block_batch": args.block_batch}
    else:
        tuned = bt.tune(mixed, target, colour, loss, grads, repeats=2)
    buckets = None
    if world > 1:
        buckets = A.BucketedGradients(params.count, BUCKETS, int(params.sh.shape[1]), params.sh_degree, device=dev)
        bucket_done = [torch.cuda.Event() for _ in range(BUCKETS)]
        side = torch.cuda.Stream(dev)
        bt.set_buckets(buckets, bucket_done)
        grads = None

    def exchange():
        """Every bucket's all-reduce on the side stream, each after its bucket's event;
        the step's stream waits for the last."""
        if buckets is None:
            return
        for k, e in enumerate(bucket_done):
            side.wait_event(e)
            with torch.cuda.stream(side):
                buckets.allreduce_bucket(k)
        stream.wait_stream(side)

    def batched_step():
        bt.step(mixed, target, colour, loss, grads, stream=stream)
        exchange()

    for _ in range(args.warmup):
        batched_step()
    bt.check()
    with ClockSampler(local) as clocks:
        ms_batched = _timed(batched_step, args.steps, stream, world, dev)
    stats = bt.check()   # raises if a timed step overflowed its buffers or a wait gave up
    stages = bt.time_stages(mixed, target, colour, loss, grads, stream=stream)
    stats = bt.check()
    buf = bt.buffers()   # the pairs' form the sizing chose
    pair_form = ("wide: 64-bit (tile, depth) key and 32-bit Gaussian" if buf["sorted_values"] is not None else
                 "packed 64-bit word, 24-bit depth key" if buf["depth_bits"] >= 24 else
                 f"packed 64-bit word, depth exponent renumbered ({buf['depth_bits']}-bit depth field)")

    # e2e through the public API: each step's target images copied in from pinned
    # host memory into one of two device buffers on a copy stream (overlapping the
    # step before, and the step's own projection and sort: only its blends wait for
    # the copy, ath_batch_train_step_after), the step reading that buffer directly
    # (the library keeps one captured step for each); the loss read back to pinned
    # host memory.
    copy = torch.cuda.Stream(dev)
    staging = [torch.empty_like(target), torch.empty_like(target)]
    h2d_done = [torch.cuda.Event(), torch.cuda.Event()]
    used = [torch.cuda.Event(), torch.cuda.Event()]
    loss_host = torch.empty(1, dtype=torch.float32, pin_memory=True)

    def upload(k):
        copy.wait_event(used[k % 2])
        with torch.cuda.stream(copy):
            staging[k % 2].copy_(host_target, non_blocking=True)
            h2d_done[k % 2].record(copy)

    def e2e_step(k):
        bt.step(mixed, staging[k % 2], colour, loss, grads, stream=stream, target_ready=h2d_done[k % 2])
        exchange()
        used[k % 2].record(stream)
        loss_host.copy_(loss, non_blocking=True)

    for e in used:
        e.record(stream)
    # one untimed step on each buffer first: its graph is captured then
    for k in range(2):
        upload(k)
        e2e_step(k)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_start, e2e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_start.record(stream)
    copy.wait_stream(stream)
    upload(0)
    for k in range(args.steps):
        if k + 1 < args.steps:
            upload(k + 1)
        e2e_step(k)
    e2e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2e_start.elapsed_time(e2e_end) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    loss_batched = float(loss_host.item())

    # the batched forward alone (ath_batch_render: every view's colour, no loss or backward)
    for _ in range(2):
        bt.render(mixed, colour, stream=stream)   # the first captures its graph
    torch.cuda.synchronize()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for _ in range(args.steps):
        bt.render(mixed, colour, stream=stream)
    r1.record(stream)
    torch.cuda.synchronize()
    ms_render = r0.elapsed_time(r1) / args.steps
    if world > 1:
        t = torch.tensor([ms_render], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_render = float(t.item())
    bt.check()
    del bt, staging

    # ---- the plain FP32 path, one view at a time, same scene and views --------
    ms_plain, plain_stages = None, None
    if not args.no_plain:
        dev_targets = [target[int(pixel_base[v]):int(pixel_base[v + 1])] for v in range(len(views))]
        plain = PlainTrainer(params, views, dev_targets, dev)
        for w in range(args.warmup):
            plain.step(stream, check=w == 0)
        ms_plain = _timed(lambda: plain.step(stream), args.steps, stream, world, dev)
        proj0, W0, H0 = views[0]
        timed = A.RenderSettings(width=W0, height=H0, time_stages=True)
        frames0, dl0 = plain.frames[(W0, H0)], plain.dl[(W0, H0)]
        st = plain.raster.render_params(proj0, params, timed, frames0, stream=stream)
        bw0, bw1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        A.l2_loss(frames0.colour, dev_targets[0], dl0, plain.loss, stream=stream)
        bw0.record(stream)
        plain.raster.backward(dl0, plain.grads, stream=stream)
        bw1.record(stream)
        torch.cuda.synchronize()
        plain_stages = {"project_ms": st.project_ms, "emit_ms": st.emit_ms, "sort_and_ranges_ms": st.tile_sort_ms,
                        "blend_ms": st.blend_ms, "backward_ms": bw0.elapsed_time(bw1)}

    T = tuned["tile"]
    total_tiles = sum(((W + T - 1) // T) * ((H + T - 1) // T) for _, W, H in views)
    passes = sort_passes(buf["depth_bits"] + max(1, math.ceil(math.log2(max(2, total_tiles)))))
    # the step's kernels: begin, projectEmit, histogram, the sort's passes, ranges,
    # the tile order, the blends (forward, loss and adjoint), and for each gradient
    # bucket the two grouping kernels and the projection adjoint (memsets are not counted)
    launches = (2 + 1 + passes + 1 + 1 + 1 + 3 * (BUCKETS if world > 1 else 1)) * args.steps
    arith = A.measure_peaks(5, stream=stream)   # the blends' denominators: FP32 FMA and ex2 rates, measured here
    out = dict(ms_batched=ms_batched, ms_plain=ms_plain, e2e_ms=e2e_ms, stages=stages, plain_stages=plain_stages,
               arith=arith,
               ms_render=ms_render,
               stats=stats, tuned=tuned, clocks=clocks.summary(), launches=launches, passes=passes,
               count=params.count, loss=loss_batched, h2d=host_target.numel() * 4, d2h=4, pair_form=pair_form,
               pixels=int(pixel_base[-1]), sizes=sorted({(W, H) for _, W, H in views}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


def cpu_baseline(threads: int = 0) -> dict:
    """The CPU restatement (oracle/: the reference's method in C++, OpenMP) on one view of the
    same workload: the forward from the same FP32 parameters, the mean-L2 loss's gradient, and
    the reference's own backward, the per-Gaussian colour gradient of its blend's
    contributionMode 4 (splat_blend.slang:381-398)."""
    from oracle import oracle as O
    from athenea_b200 import scenes
    O.build()
    p = scenes.params(WORKLOAD["count"], WORKLOAD["clustered"], 20261203 + 1, WORKLOAD["sh_degree"])
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    eye = scenes.circle_eye(0, WORKLOAD["views"] * 4, 3.0, 0.3)
    cam = O.looking_at(eye, (0, 0, 0))
    cam.focal = cam.haperture * ((H * 0.5) / math.tan(math.radians(WORKLOAD["vfov"]) * 0.5)) / W
    proj = O.projection_for(cam, W, H)
    target = np.random.default_rng(20261203 + 7).uniform(0, 1, size=(W * H, 3)).astype(np.float32)
    t0 = time.perf_counter()
    f = O.frame_for(proj, np.eye(4), W, H, rest_per_colour=15, sh_words=23)
    pr = O.project_params(f, p["means"], p["scales"], p["quats"], p["sh"], p["sh"].shape[1], threads=threads)
    binned = O.bin_(f, pr)
    out = O.blend(f, binned, pr, threads=threads)
    err = out["colour"][:, :3] - target
    dl = np.zeros((W * H, 4), np.float32)
    dl[:, :3] = 2.0 * err / (3.0 * W * H)
    O.colour_gradient(f, binned, pr, dl)
    dt = time.perf_counter() - t0
    cores = threads or os.cpu_count()
    return dict(ms=dt * 1000.0, cores=cores, evaluated=out["evaluated"], pairs=binned["pairs"],
                visible=binned["visible"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--views", type=int, default=WORKLOAD["views"], help="views a GPU draws a step")
    ap.add_argument("--gaussians", type=int, default=WORKLOAD["count"], help="Gaussians in the scene")
    ap.add_argument("--tile", type=int, choices=[8, 16, 32], default=0,
                    help="fix the batched step's tile size instead of autotuning")
    ap.add_argument("--block-batch", type=int, choices=[64, 128, 256, 512], default=256,
                    help="records a block stages at once, with --tile")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison")
    ap.add_argument("--workload", type=int, choices=[0, 1, 2, 3, 4], default=1,
                    help="0: 100k uniform, one 960x540 view; 1: 1.5M clustered, 8 views of 1920x1080 (the "
                         "headline); 2: 500k clustered, one 1280x720 view; 3: 2.36M clustered, 64 views of mixed "
                         "sizes; 4: 50M clustered, 8 views of 3840x2160")
    args = ap.parse_args()
    if args.workload != 1:
        from athenea_b200 import scenes
        w = scenes.WORKLOADS[args.workload]
        WORKLOAD.update(count=w.count, width=w.width, height=w.height, views=w.views, clustered=w.clustered,
                        name=w.name, mixed_sizes=args.workload == 3)
    else:
        WORKLOAD["views"] = args.views
        WORKLOAD["count"] = args.gaussians
    args.warmup = max(args.warmup, 3)
    rank, world, _ = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return
        runs = []
        for _ in range(args.warmup):   # untimed: builds the checker, pages the scene in
            cpu_baseline()
        for _ in range(args.steps):
            runs.append(cpu_baseline())
        ms = statistics.median(r["ms"] for r in runs)
        line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms/view", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD["name"], "gaussians": WORKLOAD["count"],
                           "width": WORKLOAD["width"], "height": WORKLOAD["height"],
                           "path": "the CPU restatement of the reference's path (oracle/, OpenMP): forward, "
                                   "mean-L2 loss gradient, the reference's colour-gradient backward"},
                "cpu_baseline": {"value": ms, "unit": "ms/view", "cores": runs[0]["cores"], "kind": "port",
                                 "sample": f"one {WORKLOAD['width']}x{WORKLOAD['height']} view of the "
                                           f"{WORKLOAD['count']}-Gaussian scene a step"},
                "e2e": {"value": ms, "unit": "ms/view", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    res = run_ours(args)
    if rank != 0 or res is None:
        return
    P = peaks()
    W, H, V = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["views"]
    headline = args.workload == 1 and WORKLOAD["count"] == 1_500_000 and V == 8
    stats, stages = res["stats"], res["stages"]
    dominant = max(stages, key=stages.get)
    fp32_peak = res["arith"]["fp32_tflops"]
    # algorithmic work a launch, per stage: bytes a unit times the units, or FLOPs counted on the
    # device. The blends' FLOPs: a forward evaluation 8 (offsets, the quadratic form, the cutoff
    # test) and 12 more when it blends (weight, three colour FMAs, transmittance, stop test); an
    # adjoint evaluation 8, and 37 more when it blends (alpha, the behind-colour recursion, the
    # transmittance recovery, the nine gradient sums)
    fwd_flops = 8 * stats["evaluated"] + 12 * stats["blended"]
    adj_flops = 8 * stats["adjoint_visited"] + 37 * stats["adjoint_live"]
    ex2_ops = stats["blended"] + 2 * stats["adjoint_live"]   # an exp a blend, an exp and a reciprocal an adjoint
    mixed_bytes = 16 + 16 + 16 + 24 + 36 + 4          # a Gaussian in the mixed layout
    work = {
        "project_emit": ("hbm", res["count"] * mixed_bytes + stats["kept"] * 48 + stats["pairs"] * 8),
        "sort": ("hbm", stats["pairs"] * (8 + 16 * res["passes"])),
        "ranges": ("hbm", stats["pairs"] * 8 + stats["pairs"] // 16 * 8),
        "blends": ("fp32", fwd_flops + adj_flops),
        "project_adjoint": ("hbm", res["count"] * (mixed_bytes + 60 * 4) + stats["kept"] * 40),
    }
    bound, amount = work[dominant]
    secs = stages[dominant] * 1e-3
    kernel_names = {"project_emit": "projectEmitKernel", "sort": "onesweepKernel", "ranges": "rangesBatchKernel",
                    "blends": "blendStepKernel", "project_adjoint": "projectAdjointBatchKernel"}
    if bound == "hbm":
        achieved = amount / secs / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": P["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / P["hbm_gbs"], "peak_source": "of measured (MEASURED_PEAKS.json hbm_gbs)"}
    else:
        achieved = amount / secs / 1e12
        roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak,
                    "peak_source": "of measured: ath_measure_peaks' FP32 FMA rate on this GPU in this run",
                    "flops": {"forward": fwd_flops, "adjoint": adj_flops},
                    "ex2": {"achieved_gops": ex2_ops / secs / 1e9, "peak_gops": res["arith"]["ex2_gops"],
                            "frac": ex2_ops / secs / 1e9 / res["arith"]["ex2_gops"]}}
    roofline["kernel"] = kernel_names[dominant]
    roofline["traffic"] = NCU_TRAFFIC.get(kernel_names[dominant]) if headline else None
    roofline["stage_share"] = stages[dominant] / sum(stages.values())
    cpu = None if args.no_cpu else cpu_baseline()
    ms_view = res["ms_batched"] / V
    line = {
        "metric": METRIC, "value": ms_view, "unit": "ms/view", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["ms_batched"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (SH bf16/e4m3)", "data": "synthetic (seeded; no dataset)",
        "config": {"workload": WORKLOAD["name"], "gaussians": WORKLOAD["count"],
                   "sizes": [f"{w}x{h}" for w, h in res["sizes"]], "pixels_per_gpu": res["pixels"],
                   "views_per_gpu": V, "sh_degree": 3, "tile": res["tuned"]["tile"],
                   "block_batch": res["tuned"]["block_batch"], "pair_form": res["pair_form"],
                   "path": "batched mixed-precision step: every view in one launch a stage, replayed from a CUDA "
                           "graph; forward, mean-L2 loss, backward to FP32 gradients",
                   "loss": "mean L2 a view against a target uniform in [0,1]^3, summed over views",
                   "parallelism": (f"views sharded over {world} GPU(s), gradients all-reduced in {BUCKETS} "
                                   "overlapped buckets") if world > 1 else "1 GPU",
                   "l2": f"inputs larger than L2 (records {V * WORKLOAD['count'] * 48 / 1e6:.0f} MB, pairs "
                         f"{stats['pairs'] * 8 / 1e6:.0f} MB, targets {res['pixels'] * 12 / 1e6:.0f} MB > 126 MB)"},
        "plain_fp32": None if res["ms_plain"] is None else {
            "ms_per_view": res["ms_plain"] / V, "speedup": res["ms_plain"] / res["ms_batched"],
            "stages_ms": res["plain_stages"],
            "path": "ath_raster_render_params + ath_l2_loss + ath_raster_backward a view, same scene and views"},
        "batched_render": {"ms_per_view": res["ms_render"] / V,
                           "path": "ath_batch_render: every view's forward alone (colour), no loss or backward, "
                                   "same scene and views"},
        "stages_ms": stages, "pairs": stats["pairs"], "kept": stats["kept"], "evaluated": stats["evaluated"],
        "blended": stats["blended"], "adjoint_visited": stats["adjoint_visited"],
        "adjoint_live": stats["adjoint_live"], "warp_visits": {
            "forward": stats["warp_visits_forward"], "adjoint": stats["warp_visits_adjoint"],
            "adjoint_summed": stats["warp_visits_adjoint_summed"]}, "records_staged": stats["records_staged"],
        "arith_peaks": res["arith"],
        "degenerate_fp64": stats["degenerate"], "loss": res["loss"],
        "roofline": roofline,
        "e2e": {"value": res["e2e_ms"] / V, "unit": "ms/view", "h2d_bytes_per_step": res["h2d"],
                "d2h_bytes_per_step": res["d2h"]},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["ms"], "unit": "ms/view", "cores": cpu["cores"], "kind": "port",
                                "sample": f"one {WORKLOAD['width']}x{WORKLOAD['height']} view of the same scene: "
                                          "forward, loss gradient and the reference's colour-gradient backward"}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
