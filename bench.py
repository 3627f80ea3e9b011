"""Benchmark: textured 2DGS forward+backward Mpix/s on one B200 per rank.

Workload (one "step" = one forward + backward of
rasterization_textured_gaussians over one batch of cameras):
  mixture1m -- 1,000,000 Gaussians drawn from a 64-component mixture (seed 3),
  32x32 RGBA low-frequency textures, four 1600x1200 cameras (fx=fy=1200) on a
  radius-25 Fibonacci sphere, tile 16, upstream dL/d(rgb, alpha) ~ N(0,1).
Inputs are seeded synthetic data of those shapes (no dataset exists here).

Arms:
  --impl ours (default): value = Mpix/s of the BF16-texture form (textures
      sampled from a BF16 copy, FP32 master and FP32 gradients), inputs
      resident in HBM; the FP32 plain drop-in is timed beside it
      (`plain_fp32`).  e2e = the same call with host inputs copied in each
      step from pinned memory and the call's results (image, alpha, loss,
      per-Gaussian gradients) copied back.
  --impl reference: the reference has no CPU textured rasterizer; this arm
      times its own PyTorch stages (projection, SH, intersection, offsets,
      from its install under baseline/_ref) and the CPU oracle (this
      repository's C++ restatement of its compositor kernels, OpenMP on all
      host cores) on a bounded tile sample.  Beside that CPU value it times the
      reference's own CUDA path on this GPU (`reference_cuda`: its kernels
      built from its sources into oracle/_ref, driven through its public
      renderer) at the largest workload that path accepts.

Timing: CUDA events on the bench's stream; inputs (textures 8.4 GB BF16 /
16.8 GB FP32) exceed the 126 MB L2; Python's cyclic GC is paused inside timed
loops (each step reads the intersection count back once, as the reference
does, so a host pause would show up as GPU idle time).

Multi-GPU (torchrun): every rank renders its own four cameras of the same
scene (replicas, weak scaling); time = max over ranks, value = all pixels /
time.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import contextlib
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "textured 2DGS fwd+bwd Mpix/s at 1M splats: bf16-tex vs fp32 plain, same B200"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------- workload
def make_scene(rank: int, world: int, n_splats: int, n_cams: int):
    from textured_gaussians_b200 import scenes

    rng = np.random.default_rng(3)
    n_comp = 64
    u = rng.normal(size=(n_comp, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    centres = u * (10.0 * rng.uniform(0, 1, size=(n_comp, 1)) ** (1.0 / 3.0))
    comp = rng.integers(0, n_comp, size=n_splats)
    means = centres[comp] + rng.normal(0, 0.5, size=(n_splats, 3))
    ls = rng.normal(-3.5, 0.6, size=(n_splats, 2))
    scales = np.exp(np.concatenate([ls, ls[:, 1:2]], 1))
    q = rng.normal(size=(n_splats, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opac = 1.0 / (1.0 + np.exp(-rng.normal(0.5, 1.0, size=n_splats)))
    colors = rng.uniform(0, 1, size=(n_splats, 1, 3))
    dirs = scenes.fibonacci_dirs(n_cams * world)[rank * n_cams:(rank + 1) * n_cams]
    V = np.stack([scenes.look_at(25.0 * d) for d in dirs])
    K = np.stack([scenes.intrinsics(1200, 800, 600)] * n_cams)
    f32 = lambda x: x.astype(np.float32)
    return dict(means=f32(means), quats=f32(q), scales=f32(scales), opacities=f32(opac), colors=f32(colors),
                viewmats=f32(V), Ks=f32(K), width=1600, height=1200)


def gpu_textures(n_splats, R, device, seed=3):
    """Low-frequency RGBA textures, 0.5 + 4x4 DCT-II content (coefficients N(0, 0.3)), clamped to [0, 1]."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    xs = torch.arange(R, device=device, dtype=torch.float32)
    basis = torch.cos(math.pi * (2 * xs[:, None] + 1) * torch.arange(4, device=device)[None, :] / (2 * R))  # [R,4]
    out = torch.empty((n_splats, R, R, 4), device=device, dtype=torch.float32)
    step = 1 << 16
    for s in range(0, n_splats, step):
        n = min(step, n_splats - s)
        a = torch.randn((n, 4, 4, 4), generator=g, device=device) * 0.3
        out[s:s + n] = (0.5 + torch.einsum("yv,xu,nvuc->nyxc", basis, basis, a)).clamp_(0.0, 1.0)
    return out


@contextlib.contextmanager
def no_gc():
    """Python's cyclic GC paused for a timed loop (collected just before): each step waits once on the host for
    the intersection count, so a host-side GC pause would otherwise show up as GPU idle time."""
    gc.collect()
    was = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.marked = False

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.first = threading.Event()
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (NVML initialisation) can stall the driver for tens of ms: let it finish
            # before any timed work
            self.first.wait(timeout=10)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.first.set()
            if self.marked:  # only samples taken from the timed region on
                self.rows.append([x.strip() for x in line.split(",")])

    def mark(self):
        """Start keeping samples (the timed region begins)."""
        self.marked = True

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[4:8]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------- distributed
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------- algorithmic bytes
def compositor_bytes(meta, D, R, s_t, N, C, H, W):
    """Compulsory HBM bytes of one compositor forward / backward launch:
    per visible splat its parameters (60 + 4D B) and one read of its texture
    (4 R^2 s_t B) per view, 4 B per intersection and per tile, the per-pixel
    outputs; the backward adds upstream gradients and saved state per pixel,
    per-splat gradient writes (68 + 4D B) and the FP32 texture-gradient
    zero-fill + write (N 4R^2 * 4 * 2 B)."""
    import torch

    visible = int((meta["radii"] > 0).sum().item())
    I = int(meta["isect_ids"].numel())
    T = int(meta["tile_width"] * meta["tile_height"] * C)
    P = C * H * W
    fwd = visible * (60 + 4 * D) + visible * 4 * R * R * s_t + 4 * I + 4 * T + P * (4 * D + 32)
    bwd = (visible * (60 + 4 * D) + visible * 4 * R * R * s_t + 4 * I + 4 * T + P * (4 * D + 32 + 4 * D + 24)
           + visible * (68 + 4 * D) + N * 4 * R * R * 4 * 2)
    return fwd, bwd, dict(visible=visible, isects=I, tiles=T, pixels=P)


# ---------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch

    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one explicit stream for torch ops, library kernels and timing events alike
    with torch.cuda.stream(torch.cuda.Stream(dev)):
        _run_ours(args, rank, world, local, dev)


def _run_ours(args, rank, world, local, dev):
    import torch
    from textured_gaussians_b200 import _backend as B
    from textured_gaussians_b200 import rasterization_textured_gaussians
    from textured_gaussians_b200.cuda import make_texture_storage

    sc = make_scene(rank, world, args.splats, args.cameras)
    T = lambda x: torch.from_numpy(x).to(dev)
    means, quats, scales, opac, colors = (T(sc[k]).requires_grad_() for k in
                                          ("means", "quats", "scales", "opacities", "colors"))
    viewmats, Ks = T(sc["viewmats"]), T(sc["Ks"])
    W, H, C, N, R = sc["width"], sc["height"], args.cameras, args.splats, args.tex
    tex32 = gpu_textures(N, R, dev).requires_grad_()
    store, _ = make_texture_storage(tex32.detach(), "bf16")
    g = torch.Generator(device=dev)
    g.manual_seed(7 + rank)
    w_rgb = torch.randn((C, H, W, 3), generator=g, device=dev)
    w_a = torch.randn((C, H, W, 1), generator=g, device=dev)

    def step(storage, tile_size, per_view, depth=0, persistent=False, filtering="bilinear", tex_scales=None):
        for t in (means, quats, scales, opac, colors, tex32):
            t.grad = None
        views = [slice(c, c + 1) for c in range(C)] if per_view else [slice(0, C)]
        for v in views:  # the plain drop-in renders one camera per call, as the reference must (C > 1 misindexes)
            out = rasterization_textured_gaussians(means, quats, scales, opac, colors, tex32, viewmats[v], Ks[v], W, H,
                                                   sh_degree=0, far_plane=100.0, tile_size=tile_size,
                                                   texture_storage=storage,
                                                   tile_order=args.tile_order, batch_depth=depth,
                                                   persistent=persistent, filtering=filtering,
                                                   texture_scales=tex_scales)
            loss = (out[0] * w_rgb[v]).sum() + (out[1] * w_a[v]).sum()
            loss.backward()
        return out, loss

    timed_info = {}

    def timed(storage, tile_size, per_view, steps, warmup, depth=0, filtering="bilinear", tex_scales=None,
              fresh=False):
        if fresh:  # another form's cached blocks released first, so its warm-up settles this form's allocations
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        for _ in range(warmup):
            step(storage, tile_size, per_view, depth, filtering=filtering, tex_scales=tex_scales)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        l0 = B.lib().tg_kernel_launch_count()
        seg0 = torch.cuda.memory_stats().get("segment.all.allocated", 0)
        B.TIMERS.enable(True)
        with no_gc():
            t0.record()
            for i in range(steps):
                starts[i].record()
                out = None  # the previous step's outputs are released before this step allocates its own
                out, _ = step(storage, tile_size, per_view, depth, filtering=filtering, tex_scales=tex_scales)
                ends[i].record()
            t1.record()
            torch.cuda.synchronize()
        # device segments the caching allocator had to add inside the timed steps (0 = every step reused memory)
        timed_info["segments_allocated"] = torch.cuda.memory_stats().get("segment.all.allocated", 0) - seg0
        launches = B.lib().tg_kernel_launch_count() - l0
        stages = B.TIMERS.summary()
        B.TIMERS.enable(False)
        barrier(world)
        total_ms = t0.elapsed_time(t1)
        per = [a.elapsed_time(b) for a, b in zip(starts, ends)]
        return total_ms, per, stages, launches, out

    # headline form: BF16 texture storage (FP32 master + gradients), all views in one call, tile size and
    # batch depth autotuned
    from textured_gaussians_b200.tuning import autotune_compositor

    # the clock sampler starts before tuning and warm-up, so its own start-up never overlaps the timed steps
    with ClockSampler(local) as clk:
        if args.tile:
            (tile, depth), tune_ms = (args.tile, args.depth), {}
        else:
            (tile, depth), tune_ms = autotune_compositor(("bench", N, C, W, H, R),
                                                         lambda ts, d: step(store, ts, False, d))
            tile = int(max_over_ranks(float(tile), world))  # every rank uses the same configuration
            depth = int(max_over_ranks(float(depth), world))
        clk.mark()
        total_bf16, per_bf16, stages_bf16, launches, out = timed(store, tile, False, args.steps, args.warmup, depth)
        segments_bf16 = timed_info["segments_allocated"]
    total_bf16 = max_over_ranks(total_bf16, world)
    fwd_b, bwd_b, counts = compositor_bytes(out[-1], 3, R, 2, N, C, H, W)
    del out  # no live autograd graph may reach the leaves when a CUDA graph is captured
    # the same form with the persistent compositor launch (CTAs take tiles from a work counter)
    pers_ms = timed_plain(lambda: step(store, tile, False, depth, True), args.steps)
    graphed = None
    if not args.no_graph:
        graphed = time_graphed(lambda: step(store, tile, False, depth), args.steps, C * H * W * world)
    # FP32 plain drop-in on the same GPU: FP32 textures, one camera per call, tile 16
    total_f32, per_f32, stages_f32, launches_f32, _ = timed(None, 16, True, args.steps, args.warmup)
    total_f32 = max_over_ranks(total_f32, world)
    # the precision form on its own: FP32 texture storage in the headline form (one call, same tile and depth),
    # so bf16 / fp32 compares storage precision alone
    total_f32_one, _, stages_f32_one, _, out_one = timed(None, tile, False, args.steps, args.warmup, depth)
    del out_one
    total_f32_one = max_over_ranks(total_f32_one, world)
    # the same headline form with the other texture filters: mipmapped2 (coarse levels built and folded back
    # every step) and anisotropic_bilinear (each pixel's footprint integrated over the texel cells it covers)
    # (at most 5 timed steps each: an anisotropic_bilinear step takes about a second)
    filters = {}
    if not args.no_filters:
        f_tile = min(tile, 16)
        f_steps = min(args.steps, 5)
        for filt in ("mipmapped2", "anisotropic_bilinear"):
            # anisotropic_bilinear at its own default batch depth (ANISO_BATCH_DEPTH)
            f_depth = depth if f_tile == tile and filt != "anisotropic_bilinear" else 0
            total_f, per_f, stages_f, _, out_f = timed(store, f_tile, False, f_steps, args.warmup, f_depth, filt,
                                                       fresh=True)
            del out_f
            total_f = max_over_ranks(total_f, world)
            filters[filt] = {
                "value": round(C * H * W * world * f_steps / (total_f / 1e3) / 1e6, 2), "unit": "Mpix/s",
                "ms_per_step": round(total_f / f_steps, 3), "steps": f_steps, "tile_size": f_tile,
                "batch_depth": f_depth or "default",
                "per_step_ms": [round(x, 3) for x in per_f],
                "allocator_segments_in_timed_steps": timed_info["segments_allocated"],
                "stage_ms": {k: round(statistics.mean(v), 4) for k, v in stages_f.items()}}

    # the other texture storage forms of the headline configuration (same tile, depth and filter)
    storage_forms = {}
    if not args.no_filters:
        for fmt in ("fp16", "fp8"):
            st_f, sc_f = make_texture_storage(tex32.detach(), fmt)
            total_s, _, stages_s, _, out_s = timed(st_f, tile, False, args.steps, args.warmup, depth,
                                                   tex_scales=sc_f, fresh=True)
            del out_s, st_f
            total_s = max_over_ranks(total_s, world)
            storage_forms[fmt] = {
                "value": round(C * H * W * world * args.steps / (total_s / 1e3) / 1e6, 2), "unit": "Mpix/s",
                "ms_per_step": round(total_s / args.steps, 3),
                "stage_ms": {k: round(statistics.mean(v), 4) for k, v in stages_s.items()}}

    # the same forms at the largest workload the reference's own CUDA path accepts (its arm times that path
    # there: `reference_cuda` of --impl reference), for a like-for-like comparison on this GPU
    same_n = None
    n_ref = reference_cuda_splats(N, R)
    if n_ref < N and not args.no_filters:
        sc_r = make_scene(rank, world, n_ref, C)
        tex_r = gpu_textures(n_ref, R, dev)
        store_r, _ = make_texture_storage(tex_r.detach(), "bf16")
        pix_r = C * sc_r["width"] * sc_r["height"]
        ms_plain = max_over_ranks(time_renderer(rasterization_textured_gaussians, sc_r, tex_r, dev, 16, 5, 2, True),
                                  world)
        ms_head = max_over_ranks(time_renderer(rasterization_textured_gaussians, sc_r, tex_r, dev, tile, 5, 2, False,
                                               texture_storage=store_r, batch_depth=depth,
                                               tile_order=args.tile_order), world)
        same_n = {"splats": n_ref,
                  "plain_fp32": {"value": round(pix_r * world / (ms_plain / 1e3) / 1e6, 2), "unit": "Mpix/s",
                                 "ms_per_step": round(ms_plain, 3), "form": "FP32 textures, one call per camera, tile 16"},
                  "bf16_one_call": {"value": round(pix_r * world / (ms_head / 1e3) / 1e6, 2), "unit": "Mpix/s",
                                    "ms_per_step": round(ms_head, 3),
                                    "form": f"BF16 storage, one call, tile {tile}, batch depth {depth or tile * tile}"}}
        # the other filters on the same splats as the reference arm times them (anisotropic_bilinear on the
        # splats whose footprints stay convex in every view): FP32 textures one call per camera, and BF16
        # storage in one call
        same_n["filters"] = {}
        for filt in ("mipmapped2", "anisotropic_bilinear"):
            n_f = reference_cuda_splats(N, R, filt)
            scf, texf = sc_r, tex_r
            if n_f != n_ref:
                scf = make_scene(rank, world, n_f, C)
                texf = gpu_textures(n_f, R, dev)
            if filt == "anisotropic_bilinear":
                keep = aniso_safe_subset(scf, dev)
                scf = dict(scf, **{k: np.ascontiguousarray(scf[k][keep]) for k in
                                   ("means", "quats", "scales", "opacities", "colors")})
                texf = gpu_textures(keep.size, R, dev)
            storef, _ = make_texture_storage(texf.detach(), "bf16")
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            f_tile = min(tile, 16)
            f_depth = depth if f_tile == tile and filt != "anisotropic_bilinear" else 0
            ms_p = max_over_ranks(time_renderer(rasterization_textured_gaussians, scf, texf, dev, 16, 3, 2, True,
                                                filtering=filt), world)
            ms_o = max_over_ranks(time_renderer(rasterization_textured_gaussians, scf, texf, dev, f_tile, 3, 2,
                                                False, filtering=filt, texture_storage=storef, batch_depth=f_depth,
                                                tile_order=args.tile_order), world)
            same_n["filters"][filt] = {
                "splats": int(scf["means"].shape[0]),
                "fp32_per_camera": {"value": round(pix_r * world / (ms_p / 1e3) / 1e6, 2), "unit": "Mpix/s",
                                    "ms_per_step": round(ms_p, 3), "form": "FP32 textures, one call per camera, tile 16"},
                "bf16_one_call": {"value": round(pix_r * world / (ms_o / 1e3) / 1e6, 2), "unit": "Mpix/s",
                                  "ms_per_step": round(ms_o, 3), "form": f"BF16 storage, one call, tile {f_tile}"}}
            del storef
            if texf is not tex_r:
                del texf
        del tex_r, store_r
        torch.cuda.empty_cache()

    pix_per_step = C * H * W * world
    value = pix_per_step * args.steps / (total_bf16 / 1e3) / 1e6
    value_f32 = pix_per_step * args.steps / (total_f32 / 1e3) / 1e6
    value_f32_one = pix_per_step * args.steps / (total_f32_one / 1e3) / 1e6

    # roofline of the dominant kernel (the compositor adjoint call)
    peaks, peaks_kind = load_peaks()
    bwd_ms = statistics.mean(stages_bf16["tg_rasterize_bwd"])
    achieved = bwd_b / (bwd_ms / 1e3) / 1e9
    roofline = {"kernel": "tg_rasterize_bwd (compositor adjoint: gradient zero-fill + adjoint kernel + densify)",
                "bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks_kind,
                "traffic": traffic_bytes(args, N, C, R, tile, depth), "algorithmic_bytes": bwd_b,
                "launch_ms": round(bwd_ms, 4)}
    # the forward compositor beside it: algorithmic and (headline workload) measured bytes over its event time
    fwd_ms = statistics.mean(stages_bf16["tg_rasterize_fwd"])
    fwd_traffic = FORWARD_KERNEL_DRAM_BYTES if traffic_bytes(args, N, C, R, tile, depth) is not None else None
    roofline_fwd = {"kernel": "tg_rasterize_fwd (compositor forward)", "bound": "hbm",
                    "achieved": round(fwd_b / (fwd_ms / 1e3) / 1e9, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": round(fwd_b / (fwd_ms / 1e3) / 1e9 / peaks["hbm_gbs"], 4), "traffic": fwd_traffic,
                    "traffic_frac": (round(fwd_traffic / (fwd_ms / 1e3) / 1e9 / peaks["hbm_gbs"], 4)
                                     if fwd_traffic else None),
                    "algorithmic_bytes": fwd_b, "launch_ms": round(fwd_ms, 4)}
    stage_ms = {k: round(statistics.mean(v), 4) for k, v in stages_bf16.items()}
    stage_ms_f32 = {k: round(statistics.mean(v), 4) for k, v in stages_f32.items()}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, sc, tex32, store, w_rgb, w_a, dev, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, sample_tiles=args.cpu_sample)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_bf16 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, shapes of the workload)",
        "config": {"workload": f"mixture1m: N={N:,} splats, {R}x{R} RGBA textures sampled from BF16 storage "
                               f"(FP32 master + FP32 gradients), {C} cameras 1600x1200 per GPU in one call, "
                               f"tile {tile}, batch depth {depth or tile * tile} (autotuned), fwd+bwd",
                   "texture_storage": "bf16", "tile_size": tile, "batch_depth": depth or tile * tile,
                   "tuning_ms": tune_ms, "splats": N,
                   "tile_order": args.tile_order,
                   "cameras_per_gpu": C, "width": W, "height": H,
                   "l2": "inputs larger than L2 (BF16 textures 8.4 GB, FP32 master 16.8 GB)",
                   "parallelism": f"replicas x{world}"},
        "splats_per_s": round(N * C * world * args.steps / (total_bf16 / 1e3), 1),
        "plain_fp32": {"value": round(value_f32, 2), "unit": "Mpix/s", "ms_per_step": round(total_f32 / args.steps, 3),
                       "form": "FP32 textures, one camera per call, tile 16 (the drop-in as the reference is used)",
                       "stage_ms": stage_ms_f32},
        "bf16_over_fp32": round(value / value_f32, 3),
        "fp32_one_call": {"value": round(value_f32_one, 2), "unit": "Mpix/s",
                          "ms_per_step": round(total_f32_one / args.steps, 3),
                          "form": f"FP32 texture storage, all cameras in one call, tile {tile}, batch depth "
                                  f"{depth or tile * tile} (the headline form with FP32 storage)",
                          "stage_ms": {k: round(statistics.mean(v), 4) for k, v in stages_f32_one.items()}},
        "bf16_over_fp32_one_call": round(value / value_f32_one, 3),
        "at_reference_cuda_splats": same_n,
        "stage_ms": stage_ms, "per_step_ms": [round(x, 3) for x in per_bf16],
        "allocator_segments_in_timed_steps": segments_bf16,
        "median_ms_per_step": round(statistics.median(per_bf16), 3),
        "median_value": round(pix_per_step / (statistics.median(per_bf16) / 1e3) / 1e6, 2),
        "graphed": graphed, "persistent_ms_per_step": round(pers_ms, 3), "filters": filters,
        "storage_forms": storage_forms,
        "counts": counts, "roofline": roofline, "roofline_forward": roofline_fwd, "gpu_launches": int(launches),
        "clocks": clk.summary(), "e2e": e2e, "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


# DRAM bytes of one compositor-adjoint call on the headline workload (1M splats, 32x32 textures, four 1600x1200
# views, tile 8, batch depth 64), measured with ncu in one pass (dram__bytes_read.sum + dram__bytes_write.sum):
# adjoint kernel 53.763 GB read + 9.741 GB written, densification kernel 0.288 + 0.022 GB; the gradient zero-fill
# (a memset, not a kernel) writes its N * R^2 * 16 bytes.
ADJOINT_KERNEL_DRAM_BYTES = 53.763221e9 + 9.741255e9 + 0.288009e9 + 0.021744e9
# the forward compositor kernel on the same workload, same capture: 36.358 GB read + 0.806 GB written
FORWARD_KERNEL_DRAM_BYTES = 36.358471e9 + 0.806166e9


def traffic_bytes(args, N, C, R, tile, depth):
    """Measured DRAM traffic of the adjoint call for the workload it was measured on, else the --traffic-bytes
    value (None when absent)."""
    if args.traffic_bytes is not None:
        return args.traffic_bytes
    if (N, C, R, tile, depth or tile * tile, args.workload) == (1_000_000, 4, 32, 8, 64, "mixture1m"):
        return ADJOINT_KERNEL_DRAM_BYTES + N * R * R * 16
    return None


def timed_plain(fn, steps, warmup=1):
    """Mean CUDA-event ms per call of fn() after `warmup` calls (current stream)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with no_gc():
        t0.record()
        for _ in range(steps):
            fn()
        t1.record()
        torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps


def time_graphed(fn, steps, pixels):
    """The same step captured once in a CUDA graph (forward, loss and backward; intersection buffers sized by
    capacity, no host synchronisation) and replayed `steps` times."""
    import torch
    from textured_gaussians_b200.graph import GraphedStep

    g = GraphedStep(fn)
    g.replay()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with no_gc():
        t0.record()
        for _ in range(steps):
            g.replay()
        t1.record()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    over = g.overflowed()
    out = {"value": round(pixels / (ms / 1e3) / 1e6, 2), "unit": "Mpix/s", "ms_per_step": round(ms, 3),
           "capacities": g.capacities, "recorded_sizes": g.sizes, "overflowed": over}
    del g
    torch.cuda.empty_cache()
    return out


def run_e2e(args, sc, tex32, store, w_rgb, w_a, dev, world):
    """Same metric through the public call with host inputs and host results: pinned-host -> device copies of
    every input each step (BF16 textures), forward + backward, and device -> host copies of the call's
    results -- the rendered image and alpha, the loss, and the gradients of means, quats, scales, opacities
    and colours.  The FP32 texture gradient (16.8 GB at 1M splats) stays on the device: the optimizer step
    that consumes it (SelectiveAdam, which also refreshes the BF16 copy the compositor samples) runs there,
    so a training loop never moves it to the host."""
    import torch

    from textured_gaussians_b200 import rasterization_textured_gaussians

    host = {k: torch.from_numpy(sc[k]).pin_memory() for k in ("means", "quats", "scales", "opacities", "colors",
                                                                "viewmats", "Ks")}
    host["textures"] = store.cpu().pin_memory()
    host["w_rgb"] = w_rgb.cpu().pin_memory()
    host["w_a"] = w_a.cpu().pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    W, H = sc["width"], sc["height"]
    C = len(sc["viewmats"])
    res_host = {"image": torch.empty((C, H, W, 3)), "alpha": torch.empty((C, H, W, 1)), "loss": torch.empty((1,))}
    for k in ("means", "quats", "scales", "opacities", "colors"):
        res_host["v_" + k] = torch.empty(sc[k].shape)
    res_host = {k: v.pin_memory() for k, v in res_host.items()}
    d2h = sum(t.numel() * t.element_size() for t in res_host.values())
    back = torch.cuda.Stream(dev)

    # a step's inputs are copied on a copy stream while the previous step computes (a prefetching input
    # pipeline, as a training loop's loader would run); every step's copies are inside the timed region
    compute = torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(dev)

    def fetch():
        copy.wait_stream(compute)  # the buffers being overwritten are free once the compute stream is past them
        with torch.cuda.stream(copy):
            d = {k: v.to(dev, non_blocking=True) for k, v in host.items()}
            ev = torch.cuda.Event()
            ev.record(copy)
        return d, ev

    def step(d, ev):
        compute.wait_event(ev)
        for t in d.values():
            t.record_stream(compute)
        leaves = {k: d[k].requires_grad_() for k in ("means", "quats", "scales", "opacities", "colors", "textures")}
        out = rasterization_textured_gaussians(leaves["means"], leaves["quats"], leaves["scales"],
                                               leaves["opacities"], leaves["colors"], leaves["textures"],
                                               d["viewmats"], d["Ks"], W, H, sh_degree=0, far_plane=100.0)
        loss = (out[0] * d["w_rgb"]).sum() + (out[1] * d["w_a"]).sum()
        loss.backward()
        # the results go back to the host on their own stream, overlapping the next step's compute
        res = {"image": out[0].detach(), "alpha": out[1].detach(), "loss": loss.detach().reshape(1)}
        for k in ("means", "quats", "scales", "opacities", "colors"):
            res["v_" + k] = leaves[k].grad
        back.wait_stream(compute)
        with torch.cuda.stream(back):
            for k, t in res.items():
                t.record_stream(back)
                res_host[k].copy_(t, non_blocking=True)

    def run(n):
        nxt = fetch()
        for i in range(n):
            cur, nxt = nxt, (fetch() if i + 1 < n else None)
            step(*cur)
            del cur

    run(max(1, min(args.warmup, 2)))
    torch.cuda.synchronize()
    barrier(world)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    steps = max(2, min(args.steps, 5))
    t0.record()
    run(steps)
    compute.wait_stream(back)  # the timed region ends once the last step's results are on the host
    t1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    pix = C * W * H * world
    return {"value": round(pix * steps / (ms / 1e3) / 1e6, 2), "unit": "Mpix/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": steps, "ms_per_step": round(ms / steps, 3),
            "path": "rasterization_textured_gaussians(textures=BF16 host tensor) + loss.backward(); each step's "
                    "host-to-device copies on a copy stream, overlapping the previous step's compute; image, "
                    "alpha, loss and the per-Gaussian gradients (not the texture gradient) copied back to "
                    "pinned host memory on a third stream"}


# ---------------------------------------------------------------- CPU arm (reference torch stages + oracle)
def reference_cpu():
    """The reference's own pure-PyTorch stages (textured_gaussians/cuda/_torch_impl.py, _torch_impl_2dgs.py)
    from its install under baseline/_ref, or None where it is not installed.  They run on the CPU as they are;
    the reference has no CPU textured compositor."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "textured_gaussians")):
        return None
    if path not in sys.path:
        sys.path.append(path)
    from textured_gaussians.cuda import _torch_impl, _torch_impl_2dgs

    return _torch_impl, _torch_impl_2dgs


def reference_cpu_stages(sc, V, K, W, H, tile, isect_n=20_000):
    """Seconds of the reference's CPU stages on one camera of the scene, with every host thread: the 2DGS
    projection and SH (degree 0) of all splats and the offset encoding of the sorted intersections, run in
    full; its tile intersection (a Python loop over splats) on the first `isect_n` splats, charged per splat."""
    import torch

    mods = reference_cpu()
    if mods is None:
        return None
    ti, ti2 = mods
    torch.set_num_threads(os.cpu_count() or 1)
    means, quats, scales = (torch.from_numpy(sc[k]) for k in ("means", "quats", "scales"))
    Vt, Kt = torch.from_numpy(V), torch.from_numpy(K)
    N = means.shape[0]
    out = {}
    t0 = time.perf_counter()
    radii, means2d, depths, _, _ = ti2._fully_fused_projection_2dgs(means, quats, scales, Vt, Kt, W, H, 0.01, 100.0)
    out["projection_s"] = time.perf_counter() - t0
    cam = torch.linalg.inv(Vt)[:, :3, 3]
    dirs = means[None] - cam[:, None]
    t0 = time.perf_counter()
    ti._spherical_harmonics(0, dirs, torch.from_numpy(sc["colors"])[None].expand(1, -1, -1, -1))
    out["sh_s"] = time.perf_counter() - t0
    radii = radii.int()
    n = min(isect_n, N)
    tw, th = -(-W // tile), -(-H // tile)
    t0 = time.perf_counter()
    _, ids, _ = ti._isect_tiles(means2d[:, :n].contiguous(), radii[:, :n].contiguous(), depths[:, :n].contiguous(),
                                tile, tw, th)
    out["isect_s"] = (time.perf_counter() - t0) * N / n
    out["isect_sampled_splats"] = n
    t0 = time.perf_counter()
    ti._isect_offset_encode(ids, 1, tw, th)
    out["offsets_s"] = (time.perf_counter() - t0) * N / n
    out["threads"] = torch.get_num_threads()
    return out


_CPU_CAMERA = {}


def cpu_baseline(args, sample_tiles: int = 16, tile: int = 8):
    """The workload's CPU cost on one camera, at the GPU arm's tile size: the reference's own CPU stages
    (projection, SH, intersection, offsets: reference_cpu_stages) where its install is present, else the
    oracle's; and the oracle's compositor forward + backward (FP32, OpenMP over tiles) on every
    `sample_tiles`-th tile row.  The per-camera stages are charged in proportion to the sampled pixels; they
    are timed on the first call and reused by later calls on the same workload, which re-time the
    compositor sample only."""
    from oracle import oracle as O

    sc = make_scene(0, 1, args.splats, args.cameras)
    rng = np.random.default_rng(3)
    N, R = args.splats, args.tex
    W, H = sc["width"], sc["height"]
    V, K = sc["viewmats"][:1], sc["Ks"][:1]
    tw, th = -(-W // tile), -(-H // tile)
    key = (N, args.cameras, tile)
    if key not in _CPU_CAMERA:
        t0 = time.perf_counter()
        proj = O.project_fwd(sc["means"], sc["quats"], sc["scales"], V, K, W, H, 0.01, 100.0)
        t_proj_port = time.perf_counter() - t0
        t0 = time.perf_counter()
        _, ids, fl = O.isect_tiles(proj[1], proj[0], proj[2], tile, tw, th, 1)
        off = O.isect_offset_encode(ids, 1, tw, th)
        t_isect_port = time.perf_counter() - t0
        _CPU_CAMERA[key] = (proj, fl, off, t_proj_port, t_isect_port, reference_cpu_stages(sc, V, K, W, H, tile))
    (radii, m2d, dep, M, nrm), fl, off, t_proj_port, t_isect_port, ref = _CPU_CAMERA[key]
    if ref is not None:
        t_cam = ref["projection_s"] + ref["sh_s"] + ref["isect_s"] + ref["offsets_s"]
    else:
        t_cam = t_proj_port + t_isect_port
    # textures for the splats touched by the sampled tiles only (keeps host memory bounded)
    mask = np.zeros((1, th, tw), np.uint8)
    mask[0, ::sample_tiles, :] = 1
    frac = mask.mean()
    tex = np.full((N, R, R, 4), 0.5, np.float32) if N * R * R * 16 <= 4 << 30 else None
    if tex is None:
        # 16.8 GB would not be reasonable on the host; a 0.5-grey texture table of the same shape is
        # replaced by a shared constant texture, which does not change the compositor's work
        tex = np.full((1, R, R, 4), 0.5, np.float32)
        gid = np.zeros(m2d.shape[1], np.int64)
    else:
        gid = None
    cols = np.broadcast_to(sc["colors"][:, 0][None], (1, N, 3)).copy()
    op = sc["opacities"][None]
    t1 = time.perf_counter()
    if gid is None:
        fwd = O.raster_fwd(m2d, M, cols, op, nrm, tex, off, fl, W, H, tile, masks=mask)
    else:
        fwd = O.raster_fwd(m2d[0], M[0], cols[0], op[0], nrm[0], tex, off, fl, W, H, tile, masks=mask,
                           gaussian_ids=gid, n_gauss=1)
    vc = rng.normal(size=(1, H, W, 3)).astype(np.float32)
    va = rng.normal(size=(1, H, W, 1)).astype(np.float32)
    z1 = np.zeros((1, H, W, 1), np.float32)
    z3 = np.zeros((1, H, W, 3), np.float32)
    if gid is None:
        O.raster_bwd(m2d, M, cols, op, nrm, tex, off, fl, W, H, tile, fwd, vc, va, z3, z1, z1, masks=mask)
    else:
        O.raster_bwd(m2d[0], M[0], cols[0], op[0], nrm[0], tex, off, fl, W, H, tile, fwd, vc, va, z3, z1, z1,
                     masks=mask, gaussian_ids=gid, n_gauss=1)
    t_raster = time.perf_counter() - t1
    est = t_cam * frac + t_raster
    mpix = W * H * frac / est / 1e6
    stages = "reference torch stages" if ref is not None else "oracle stages"
    out = {"value": round(mpix, 4), "unit": "Mpix/s", "cores": os.cpu_count(), "kind": "port",
           "sample": f"one 1600x1200 camera of the workload at tile {tile}: projection, SH, intersection and offsets "
                     f"of all {N:,} splats ({stages}, {t_cam:.2f} s, charged x{frac:.3f}), compositor fwd+bwd "
                     f"(FP32 oracle, OpenMP) on every {sample_tiles}th tile row ({frac * 100:.1f}% of pixels, "
                     f"{t_raster:.2f} s)",
           "stage_s": {"camera_stages": round(t_cam, 3), "compositor_sample": round(t_raster, 3),
                       "oracle_projection": round(t_proj_port, 3), "oracle_isect_sort_offsets": round(t_isect_port, 3)}}
    if ref is not None:
        out["reference_stages_s"] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in ref.items()}
    return out


# ---------------------------------------------------------------- batching form (64 uneven views, 3 scenes)
BATCH_SIZES = [(400, 300), (800, 600), (1297, 840), (1600, 1200)]


def make_batch_workload(n_views=64, scene_sizes=(200_000, 500_000, 1_000_000), seed=4):
    """Three mixture scenes (as the 1M workload, seeds 4, 5, 6), 64 views with resolutions drawn uniformly from
    BATCH_SIZES (fx = fy = W, principal point at the centre), view c showing scene c % 3 from the
    (c // 3)-th of that scene's radius-25 Fibonacci directions."""
    from textured_gaussians_b200 import scenes

    parts = []
    for s, n in enumerate(scene_sizes):
        sc = make_scene_seeded(n, seed + s)
        parts.append(sc)
    rng = np.random.default_rng(seed)
    sizes = [BATCH_SIZES[i] for i in rng.integers(0, len(BATCH_SIZES), size=n_views)]
    view_scenes = [c % len(scene_sizes) for c in range(n_views)]
    per_scene = [sum(1 for v in view_scenes if v == s) for s in range(len(scene_sizes))]
    dirs = [scenes.fibonacci_dirs(k) for k in per_scene]
    V = np.stack([scenes.look_at(25.0 * dirs[view_scenes[c]][c // len(scene_sizes)]) for c in range(n_views)])
    K = np.stack([scenes.intrinsics(w, w / 2, h / 2) for w, h in sizes])
    cat = {k: np.concatenate([p[k] for p in parts]) for k in ("means", "quats", "scales", "opacities", "colors")}
    offs = np.cumsum([0] + list(scene_sizes)).tolist()
    return cat, offs, V.astype(np.float32), K.astype(np.float32), sizes, view_scenes


def make_scene_seeded(n_splats: int, seed: int):
    """The mixture scene of make_scene with its own seed (Gaussians only)."""
    rng = np.random.default_rng(seed)
    n_comp = 64
    u = rng.normal(size=(n_comp, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    centres = u * (10.0 * rng.uniform(0, 1, size=(n_comp, 1)) ** (1.0 / 3.0))
    comp = rng.integers(0, n_comp, size=n_splats)
    means = centres[comp] + rng.normal(0, 0.5, size=(n_splats, 3))
    ls = rng.normal(-3.5, 0.6, size=(n_splats, 2))
    scales = np.exp(np.concatenate([ls, ls[:, 1:2]], 1))
    q = rng.normal(size=(n_splats, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opac = 1.0 / (1.0 + np.exp(-rng.normal(0.5, 1.0, size=n_splats)))
    colors = rng.uniform(0, 1, size=(n_splats, 1, 3))
    f32 = lambda x: x.astype(np.float32)
    return dict(means=f32(means), quats=f32(q), scales=f32(scales), opacities=f32(opac), colors=f32(colors))


def run_batch(args):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    with torch.cuda.stream(torch.cuda.Stream(dev)):
        _run_batch(args, dev)


def _run_batch(args, dev):
    """Config of the batching form: one call renders all 64 views (BF16 texture storage, heaviest tiles first,
    tile autotuned) against the FP32 plain drop-in called once per view at tile 16."""
    import torch
    from textured_gaussians_b200 import _backend as B
    from textured_gaussians_b200 import rasterization_textured_gaussians
    from textured_gaussians_b200.batch import ViewTable, rasterization_textured_gaussians_batch
    from textured_gaussians_b200.cuda import make_texture_storage
    from textured_gaussians_b200.tuning import autotune_compositor

    cat, offs, V, K, sizes, vs = make_batch_workload(n_views=args.views)
    T = lambda x: torch.from_numpy(x).to(dev)
    L = {k: T(v).requires_grad_() for k, v in cat.items()}
    R = args.tex
    N = offs[-1]
    tex32 = torch.cat([gpu_textures(offs[s + 1] - offs[s], R, dev, seed=4 + s) for s in range(len(offs) - 1)])
    tex32.requires_grad_()
    store, _ = make_texture_storage(tex32.detach(), "bf16")
    viewmats, Ks = T(V), T(K)
    widths, heights = [w for w, _ in sizes], [h for _, h in sizes]
    n_pix = sum(w * h for w, h in sizes)
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    w_flat = torch.randn((n_pix, 4), generator=g, device=dev)
    pix_base = np.cumsum([0] + [w * h for w, h in sizes]).tolist()
    tables = {}

    def zero():
        for t in list(L.values()) + [tex32]:
            t.grad = None

    def step_batch(tile, order, depth=0, persistent=False):
        zero()
        vt = tables.get(tile)
        if vt is None:
            vt = tables[tile] = ViewTable(widths, heights, tile, dev)
        out = rasterization_textured_gaussians_batch(
            L["means"], L["quats"], L["scales"], L["opacities"], L["colors"], tex32, offs, viewmats, Ks, widths,
            heights, vs, sh_degree=0, far_plane=100.0, tile_size=tile, texture_storage=store, tile_order=order,
            view_table=vt, batch_depth=depth, persistent=persistent)
        meta = out[-1]
        loss = (meta["flat_colors"] * w_flat[:, :3]).sum() + (meta["flat_alphas"] * w_flat[:, 3:]).sum()
        loss.backward()
        return meta

    def step_per_view():
        zero()
        for c, (w, h) in enumerate(sizes):
            a, b = offs[vs[c]], offs[vs[c] + 1]
            out = rasterization_textured_gaussians(
                L["means"][a:b], L["quats"][a:b], L["scales"][a:b], L["opacities"][a:b], L["colors"][a:b],
                tex32[a:b], viewmats[c:c + 1], Ks[c:c + 1], w, h, sh_degree=0, far_plane=100.0, tile_size=16)
            wv = w_flat[pix_base[c]:pix_base[c + 1]]
            loss = (out[0].reshape(-1, 3) * wv[:, :3]).sum() + (out[1].reshape(-1, 1) * wv[:, 3:]).sum()
            loss.backward()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        l0 = B.lib().tg_kernel_launch_count()
        B.TIMERS.enable(True)
        with no_gc():
            t0.record()
            for _ in range(steps):
                fn()
            t1.record()
            torch.cuda.synchronize()
        stages = {k: round(statistics.mean(v), 3) for k, v in B.TIMERS.summary().items()}
        B.TIMERS.enable(False)
        return t0.elapsed_time(t1) / steps, stages, B.lib().tg_kernel_launch_count() - l0

    # the workload's tuning grid: tile size in {8, 16, 32} x Gaussian batch depth in {64, 128, 256}
    (tile, depth), tune_ms = autotune_compositor(("batch", N, len(sizes)),
                                                 lambda ts, d: step_batch(ts, "heaviest_first", d),
                                                 depths=(64, 128, 256), repeats=1)
    with ClockSampler(0) as clk:
        clk.mark()
        ms_b, stages_b, launches_b = timed(lambda: step_batch(tile, "heaviest_first", depth), args.steps, args.warmup)
    ms_launch, _, _ = timed(lambda: step_batch(tile, "launch", depth), args.steps, 1)
    ms_pers = timed_plain(lambda: step_batch(tile, "heaviest_first", depth, True), args.steps)
    graphed = (None if args.no_graph
               else time_graphed(lambda: step_batch(tile, "heaviest_first", depth), args.steps, n_pix))
    ms_pv, stages_pv, launches_pv = timed(step_per_view, args.steps, 1)
    line = {
        "metric": "textured 2DGS fwd+bwd Mpix/s, batching form: 64 uneven views over 3 scenes in one call",
        "value": round(n_pix / (ms_b / 1e3) / 1e6, 2), "unit": "Mpix/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_b, 3), "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": f"3 mixture scenes N=200k/500k/1M ({N:,} splats), {R}x{R} RGBA textures in BF16 "
                               f"storage, {len(sizes)} views drawn from {BATCH_SIZES}, {n_pix:,} pixels, "
                               f"tile {tile}, batch depth {depth or tile * tile} (autotuned), heaviest tiles first, "
                               f"fwd+bwd",
                   "tuning_ms": tune_ms, "views": len(sizes), "pixels": n_pix, "splats": N},
        "splats_per_s": round(sum(offs[s + 1] - offs[s] for s in vs) / (ms_b / 1e3), 1),
        "launch_order_ms_per_step": round(ms_launch, 3), "persistent_ms_per_step": round(ms_pers, 3),
        "per_view_fp32": {"value": round(n_pix / (ms_pv / 1e3) / 1e6, 2), "unit": "Mpix/s",
                          "ms_per_step": round(ms_pv, 3), "form": "FP32 plain drop-in, one call per view, tile 16",
                          "stage_ms": stages_pv, "gpu_launches": int(launches_pv)},
        "batch_over_per_view_fp32": round(ms_pv / ms_b, 3), "graphed": graphed,
        "stage_ms": stages_b, "gpu_launches": int(launches_b), "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


# The reference indexes textures through 32-bit packed accessors and refuses a texture tensor of more than
# 2^31 - 1 elements (1,000,000 x 32 x 32 x 4 is 4.2e9): its CUDA path is timed at the largest splat count in
# steps of 100,000 that it accepts (500,000 at 32x32), and this arm's own form is timed there too.
def reference_cuda_splats(n_splats: int, R: int, filtering: str = "bilinear") -> int:
    """The most splats (in 100,000s) the reference's compositor takes: it refuses texture tensors of 2^31
    elements or more -- for mipmapped2 its full pyramid, (4^(L+1) - 1) / 3 texels a splat."""
    texels = R * R
    if filtering == "mipmapped2":
        texels = (4 * R * R - 1) // 3
    cap = (2**31 - 1) // (texels * 4)
    return min(n_splats, cap // 100_000 * 100_000 if cap >= 100_000 else cap)


def load_reference_package():
    """The reference's Python package (baseline/_ref) with its _C module bound to its own kernels as built
    from its sources into oracle/_ref (the package's own loader would compile every kernel it ships)."""
    import types

    from oracle import build_ref

    mod = build_ref.load()
    pkg = os.path.join(ROOT, "baseline", "_ref")
    if mod is None or not os.path.isdir(os.path.join(pkg, "textured_gaussians")):
        return None
    if pkg not in sys.path:
        sys.path.append(pkg)
    stub = types.ModuleType("textured_gaussians.cuda._backend")
    stub._C = mod
    sys.modules["textured_gaussians.cuda._backend"] = stub
    from textured_gaussians import rendering

    return rendering


def time_renderer(render, sc, tex, dev, tile, steps, warmup, per_view, **kw):
    """ms per fwd+bwd step of `render` (a rasterization_textured_gaussians) over the scene's cameras."""
    import torch

    T = lambda x: torch.from_numpy(x).to(dev)
    leaves = [T(sc[k]).requires_grad_() for k in ("means", "quats", "scales", "opacities", "colors")]
    tex = tex.requires_grad_()
    V, K = T(sc["viewmats"]), T(sc["Ks"])
    C, W, H = V.shape[0], sc["width"], sc["height"]
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    w_rgb = torch.randn((C, H, W, 3), generator=g, device=dev)

    def step():
        for t in leaves + [tex]:
            t.grad = None
        views = [slice(c, c + 1) for c in range(C)] if per_view else [slice(0, C)]
        for v in views:
            out = render(*leaves, tex, V[v], K[v], W, H, sh_degree=0, far_plane=100.0, tile_size=tile, **kw)
            (out[0] * w_rgb[v]).sum().backward()

    return timed_plain(step, steps, warmup)


def aniso_safe_subset(sc, dev, tile=16):
    """Indices of the splats whose footprint quads stay convex on every pixel of every tile they touch, in
    every view.  The reference's anisotropic_bilinear clipping keeps at most 8 vertices in fixed arrays
    (filters/anisotropic_bilinear.cuh:80-160); a pixel whose corner rays meet the splat's plane on both
    sides gives a self-intersecting quad that can need more (undefined behaviour), so its timing runs only
    on splats that stay 1.5 (radius + tile + 2) pixels from that line, z(px, py) = 0, in all views."""
    import torch

    from textured_gaussians_b200.cuda import fully_fused_projection_2dgs

    T = lambda x: torch.from_numpy(x).to(dev)
    with torch.no_grad():
        radii, m2d, _, M, _ = fully_fused_projection_2dgs(
            T(sc["means"]), T(sc["quats"]), T(sc["scales"]), T(sc["viewmats"]), T(sc["Ks"]), sc["width"],
            sc["height"], 0.3, 0.01, 100.0, 0.0)
    r = radii.cpu().numpy().astype(np.float64)
    M = M.cpu().numpy().astype(np.float64)
    c = m2d.cpu().numpy().astype(np.float64)
    M0, M1, M2 = M[..., 0, :], M[..., 1, :], M[..., 2, :]

    def cz(u, v):
        return u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0]

    a, b, c0 = -cz(M2, M1), -cz(M0, M2), cz(M0, M1)
    dist = np.abs(a * c[..., 0] + b * c[..., 1] + c0) / np.maximum(np.hypot(a, b), 1e-300)
    keep = ((r <= 0) | (dist >= 1.5 * (r + tile + 2))).all(axis=0)
    return np.flatnonzero(keep)


def reference_cuda(args):
    """The reference's own CUDA path on this GPU: its renderer, FP32 textures, one call per camera (the only
    defined form), at reference_cuda_splats() splats; None where its build or install is absent."""
    import torch

    if not torch.cuda.is_available():
        return None
    R = args.tex
    n = reference_cuda_splats(args.splats, R)
    ref = load_reference_package()
    if ref is None:
        return None
    dev = torch.device("cuda", 0)
    sc = make_scene(0, 1, n, args.cameras)
    out = {"splats": n, "texture": f"{R}x{R} FP32", "cameras": args.cameras, "form": "one call per camera",
           "why_reduced": f"the reference refuses texture tensors of more than 2^31 - 1 elements "
                          f"({args.splats:,} x {R}x{R}x4 = {args.splats * R * R * 4:.3g})"}
    pix = args.cameras * sc["width"] * sc["height"]
    for tile in (16, 8):
        tex = gpu_textures(n, R, dev)
        ms = time_renderer(ref.rasterization_textured_gaussians, sc, tex, dev, tile, 5, 2, True)
        out[f"tile{tile}"] = {"value": round(pix / (ms / 1e3) / 1e6, 2), "unit": "Mpix/s", "ms_per_step": round(ms, 3)}
        del tex
        torch.cuda.empty_cache()
    # the other texture filters, same form: mipmapped2 (a zero background: its adjoint returns a background
    # gradient for a None background, which autograd rejects) and anisotropic_bilinear on the splats whose
    # footprints stay convex in every view (aniso_safe_subset)
    out["filters"] = {}
    bg = torch.zeros((1, 3), device=dev)
    for filt in ("mipmapped2", "anisotropic_bilinear"):
        nf = reference_cuda_splats(args.splats, R, filt)
        scf = sc if nf == n else make_scene(0, 1, nf, args.cameras)
        if filt == "anisotropic_bilinear":
            keep = aniso_safe_subset(sc, dev)
            scf = dict(scf, **{k: np.ascontiguousarray(scf[k][keep]) for k in
                               ("means", "quats", "scales", "opacities", "colors")})
        nf = scf["means"].shape[0]
        tex = gpu_textures(nf, R, dev)
        steps, warm = (2, 1) if filt == "anisotropic_bilinear" else (5, 2)
        res = {"splats": nf}
        for tile in ((16,) if filt == "anisotropic_bilinear" else (16, 8)):  # bounded: about 1 s a step
            ms = time_renderer(ref.rasterization_textured_gaussians, scf, tex, dev, tile, steps, warm, True,
                               filtering=filt, backgrounds=bg)
            res[f"tile{tile}"] = {"value": round(pix / (ms / 1e3) / 1e6, 2), "unit": "Mpix/s",
                                  "ms_per_step": round(ms, 3)}
        out["filters"][filt] = res
        del tex
        torch.cuda.empty_cache()
    return out


def cpu_config_table():
    """The CPU cost of the small workloads run whole, and of one camera of the views8 workload, on the host's
    cores: the reference's own torch stages (projection, SH, intersection, offsets) plus the oracle's FP32
    compositor forward + backward.  Printed by --impl reference --cpu-configs (one JSON line)."""
    import torch

    from oracle import oracle as O
    from textured_gaussians_b200 import scenes

    mods = reference_cpu()
    ti, ti2 = mods if mods is not None else (None, None)
    torch.set_num_threads(os.cpu_count() or 1)
    rows = {}
    for name, make in (("config0_small", scenes.small), ("config2_adjoint", scenes.adjoint),
                       ("config1_views8_camera0", lambda: scenes.views8(with_textures=False))):
        s = make()
        V, K = s.viewmats[:1], s.Ks[:1]
        N, W, H, ts = s.means.shape[0], s.width, s.height, s.tile_size
        tw, th = -(-W // ts), -(-H // ts)
        st = {}
        if ti2 is not None:
            means, quats, scales = (torch.from_numpy(x) for x in (s.means, s.quats, s.scales))
            t0 = time.perf_counter()
            radii_t, m2d_t, dep_t, _, _ = ti2._fully_fused_projection_2dgs(means, quats, scales, torch.from_numpy(V),
                                                                          torch.from_numpy(K), W, H, s.near_plane,
                                                                          s.far_plane)
            st["ref_projection"] = time.perf_counter() - t0
            cam = torch.linalg.inv(torch.from_numpy(V))[:, :3, 3]
            t0 = time.perf_counter()
            ti._spherical_harmonics(s.sh_degree, means[None] - cam[:, None], torch.from_numpy(s.colors)[None])
            st["ref_sh"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            _, ids_t, _ = ti._isect_tiles(m2d_t, radii_t.int(), dep_t, ts, tw, th)
            st["ref_isect"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            ti._isect_offset_encode(ids_t, 1, tw, th)
            st["ref_offsets"] = time.perf_counter() - t0
        radii, m2d, dep, M, nrm = O.project_fwd(s.means, s.quats, s.scales, V, K, W, H, s.near_plane, s.far_plane)
        _, ids, fl = O.isect_tiles(m2d, radii, dep, ts, tw, th, 1)
        off = O.isect_offset_encode(ids, 1, tw, th)
        cam = np.linalg.inv(V.astype(np.float64))[:, :3, 3]
        cols = np.maximum(O.sh_fwd(s.sh_degree, (s.means[None] - cam[:, None]).astype(np.float32), s.colors,
                                   masks=radii > 0) + 0.5, 0).astype(np.float32)
        R = s.textures.shape[1] if s.textures is not None else s.extra["texture_res"]
        if s.textures is not None:
            tex, gid, ng = s.textures, None, None
        else:  # 12 GB of textures would not be reasonable on the host: one shared texture, the same work
            tex, gid, ng = np.full((1, R, R, 4), 0.5, np.float32), np.zeros(N, np.int64), 1
        args = (m2d, M, cols, s.opacities[None], nrm, tex, off, fl, W, H, ts)
        kw = {} if gid is None else dict(gaussian_ids=gid, n_gauss=ng)
        if gid is not None:
            args = (m2d[0], M[0], cols[0], s.opacities, nrm[0]) + args[5:]
        rng = np.random.default_rng(0)
        up = [rng.normal(size=(1, H, W, c)).astype(np.float32) for c in (3, 1, 3, 1, 1)]
        t0 = time.perf_counter()
        fo = O.raster_fwd(*args, backgrounds=s.backgrounds, **kw)
        O.raster_bwd(*args, fo, *up, backgrounds=s.backgrounds, **kw)
        st["oracle_compositor_fwd_bwd"] = time.perf_counter() - t0
        total = sum(st.values())
        rows[name] = {"splats": N, "texture": f"{R}x{R}", "pixels": W * H, "tile": ts,
                      "stage_s": {k: round(v, 4) for k, v in st.items()},
                      "value": round(W * H / total / 1e6, 4), "unit": "Mpix/s"}
    return {"cpu_configs": rows, "cores": os.cpu_count(), "cpu": _cpu_model()}


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.cpu_configs:
        print(json.dumps(cpu_config_table()), flush=True)
        return
    samples = []
    for _ in range(args.warmup + args.steps):
        samples.append(cpu_baseline(args, sample_tiles=args.cpu_sample))
    vals = [s["value"] for s in samples[args.warmup:]]
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, shapes of the workload)",
        "config": {"workload": f"mixture1m: N={args.splats:,} splats, {args.tex}x{args.tex} RGBA textures, "
                               f"1600x1200 cameras, tile 8, fwd+bwd (CPU sample)"},
        "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": samples[-1]["cores"], "kind": "port",
                         "sample": samples[-1]["sample"],
                         "reference_stages_s": samples[-1].get("reference_stages_s")},
        "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": reference_cuda(args),
        "note": "the reference has no CPU textured compositor: this arm times the reference's own PyTorch "
                "stages (projection, SH, intersection, offsets) from its install and the C++ restatement of its "
                "compositor kernels on the host cores",
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20,
                    help="timed steps: value from their total time, median_value from their median")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--splats", type=int, default=1_000_000)
    ap.add_argument("--cameras", type=int, default=4)
    ap.add_argument("--tex", type=int, default=32)
    ap.add_argument("--cpu-sample", type=int, default=16)
    ap.add_argument("--tile", type=int, default=0,
                    help="tile size of the headline form (0 = autotune tile over 8, 16, 32 and the batch depth)")
    ap.add_argument("--depth", type=int, default=0, help="batch depth with --tile (0 = tile^2)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay timing")
    ap.add_argument("--no-filters", action="store_true",
                    help="skip the timing of the other texture filters and storage forms")
    ap.add_argument("--workload", default="mixture1m", choices=["mixture1m", "batch"],
                    help="mixture1m: the headline workload; batch: 64 uneven views over 3 scenes (batching form)")
    ap.add_argument("--views", type=int, default=64, help="views of the batch workload")
    ap.add_argument("--tile-order", default="heaviest_first", choices=["launch", "heaviest_first"],
                    help="compositor tile order of the headline form")
    ap.add_argument("--cpu-configs", action="store_true",
                    help="with --impl reference: time the small workloads whole on the CPU (reference torch stages "
                         "+ oracle compositor) instead of the benchmark line")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="DRAM bytes of one compositor-adjoint launch from an ncu capture, reported as roofline.traffic")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
