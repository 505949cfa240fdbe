"""Benchmark of the splat render path on B200.

Headline workload ("frame"): 1M splats, SH degree 3 (16 coefficients per
channel), means from 8 Gaussian clusters, 1920x1080, cameras on a 30-view
radius-4 orbit. A step renders one frame (project, binned intersection build:
per-tile counts, placement, per-tile sort by depth; rasterize) through
sf_render_frames, the orbit's 30 cameras per call: the frames are enqueued
back to back and each frame's intersection total is checked at the call's
one host sync.

  value   frames/s, all ranks, device-timed with CUDA events on the launch
          stream, inputs resident in HBM (236 MB of splat planes > 126 MB L2,
          so no L2 flush is needed between frames);
  e2e     the same frames through sf_render_frames_to_host (the orbit's
          30 cameras per call): each camera goes in from host memory and each
          frame's RGBA8 image comes back into pinned host memory inside the
          timed region (wall clock), the read-back of one frame overlapping
          the next frame; e2e.single_frame is sf_render_to_host, one frame per
          call with its read-back after it;
  roofline the rasterizer (the largest kernel) against the FP32 pipe: 24
          FP32 operations per visited (pixel, splat) pair, pairs counted by
          the kernel itself;
  backward the adjoint (forward that keeps per-pixel state, then the
          backward) on one frame of the same scene;
  eig_round a 20-view 512x512 segmentation round, batched into one CUDA
          graph vs the plain per-view calls;
  cpu_baseline the CPU oracle (a C++/OpenMP restatement of the reference's
          kernels) on one frame of the same workload on this host's cores.

--impl reference runs that CPU implementation alone as the reference arm (the
reference itself is Rust on wgpu and cannot run on this machine).
Multi-GPU: replicas only (each rank renders its share of the orbit); rank 0
prints the one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SPLATS, SH_PER_CH, WIDTH, HEIGHT, N_CAMS, RADIUS = 1_000_000, 16, 1920, 1080, 30, 4.0
WORKLOAD = ("frame: 1M splats SH3 (8 Gaussian clusters sigma 0.3 in [-2,2]^3), 1920x1080, "
            "30-camera radius-4 orbit")
METRIC = "1080p frames/s @1M splats"
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 lanes x FMA x 1.965 GHz
# DRAM bytes (read + write) of one rasterizer launch of this workload, from an
# ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, orbit camera 3:
# 47.40 MB + 1.59 MB). Traffic far above the gathered records would mean
# re-reads; here it is the walked entries' records and ids.
RASTER_TRAFFIC_BYTES = 48.99e6
RASTER_FLOPS_PER_PAIR = 24
RESERVE_ISECTS = 1 << 24


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples taken while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def make_scene():
    from splatfield_b200 import synth

    return synth.scene_clustered(N_SPLATS, SH_PER_CH, seed=0)


def orbit(make_look_at):
    from splatfield_b200 import synth

    return synth.orbit_cameras(N_CAMS, RADIUS, WIDTH, HEIGHT, make_look_at)


def cpu_frame_time(attr, sh, max_frames=3, budget_s=30.0):
    """Seconds per frame of the CPU oracle on this host (all OpenMP threads)."""
    import oracle as O

    cams = orbit(O.look_at)
    times = []
    t_total = 0.0
    for i in range(max_frames):
        t0 = time.perf_counter()
        prep = O.prepare(cams[i % len(cams)], WIDTH, HEIGHT, attr, sh, SH_PER_CH)
        O.rasterize(prep, 0, want_float=False)
        dt = time.perf_counter() - t0
        times.append(dt)
        t_total += dt
        if t_total > budget_s:
            break
    return float(np.median(times)), len(times), O.num_threads()


def time_backward(sf, splats, scratch, attr, sh, cam, stream, args):
    """Adjoint workload: the frame scene, one camera, L2 loss against the render
    of a copy with means + N(0, 0.01) and opacity logits + N(0, 0.2). Times
    sf_render_forward (the float frame that keeps per-pixel state) and
    sf_render_backward (raster replay + projection adjoint) with CUDA events."""
    import torch

    from splatfield_b200 import synth

    size = (WIDTH, HEIGHT)
    target_splats = sf.Splats(synth.perturbed(attr, N_SPLATS, seed=0), sh, splats.ctx)
    target_scratch = sf.RenderScratch(N_SPLATS, size, splats.ctx)
    target = target_splats.render_forward(target_scratch, cam, size, stream=stream).read()
    img = splats.render_forward(scratch, cam, size, stream=stream).read()
    dl = sf.DeviceBuffer.from_array((2.0 * (img - target)).astype(np.float32), splats.ctx)
    del target_splats, target_scratch
    d_attr = sf.DeviceBuffer.empty(11 * N_SPLATS, np.float32, splats.ctx)
    d_sh = sf.DeviceBuffer.empty(3 * SH_PER_CH * N_SPLATS, np.float32, splats.ctx)
    reps = max(3, min(args.steps // 30, 50))
    fwd_ms, bwd_ms = [], []
    for i in range(reps + 2):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        splats.render_forward(scratch, cam, size, stream=stream)
        e1.record(stream)
        splats.render_backward_into(scratch, cam, size, dl, d_attr, d_sh, stream=stream)
        e2.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            fwd_ms.append(e0.elapsed_time(e1))
            bwd_ms.append(e1.elapsed_time(e2))
    f, b = float(np.median(fwd_ms)), float(np.median(bwd_ms))
    return {"workload": "adjoint: frame scene, 1 camera, L2 vs perturbed-copy render",
            "forward_ms": f, "backward_ms": b, "ratio": b / f, "target_ratio": 3.0, "reps": reps,
            "note": "device-timed; forward = sf_render_forward (keeps per-pixel T and last "
                    "contributor), backward = sf_render_backward into device gradient buffers"}


ROUND_VIEWS, ROUND_SIDE, ROUND_RADIUS = 20, 512, 3.5


def time_eig_round(sf, splats, ctx, stream, args):
    """Segmentation round on the frame scene: 20 candidate views at 512x512 on
    a radius-3.5 sphere, posterior a, b log-uniform in [1, 1024]. Per view the
    responsibility render and its EIG.

    plain   the reference's Segmenter::select_view loop: per view
            sf_render_responsibility (one host sync for the intersection
            total) then sf_beta_eig (one sync for the sum);
    batched sf_round_eig: all views in one CUDA graph, one sync per round
            (lanes and raster form chosen by sf_round_autotune, untimed).
    The evidence + EIG form (the C2 round) lifts each view's fg / bg words
    under a 1-3 ellipse mask and reduces its EIG over fg + bg (prepare +
    masked sf_accumulate_prepared + sf_beta_eig per view vs
    sf_round_evidence); the words stay on the device in both arms and are
    compared once after timing, the EIGs every round.
    Rounds are timed on the host clock around a synchronised round (the plain
    path's host syncs are part of its cost); results must agree exactly."""
    import torch

    from splatfield_b200 import synth

    size = (ROUND_SIDE, ROUND_SIDE)
    a, b = synth.beta_posterior(N_SPLATS, seed=1)
    beta = sf.BetaState.from_host(a, b, ctx)
    cams = synth.sphere_cameras(ROUND_VIEWS, ROUND_RADIUS, 2, sf.look_at)
    masks = [sf.Mask.from_bytes(size, synth.ellipse_mask(ROUND_SIDE, ROUND_SIDE, seed=100 + v), ctx)
             for v in range(ROUND_VIEWS)]
    scratch = sf.RenderScratch(N_SPLATS, size, ctx)
    acc = sf.Accumulators(N_SPLATS, ctx)
    rnd = sf.Round(N_SPLATS, [size] * ROUND_VIEWS, ctx)
    reps = max(3, min(args.steps // 100, 15))

    def plain_round(mode, evidence, keep=None):
        out = []
        for v in range(ROUND_VIEWS):
            if evidence:
                isects = splats.prepare_isects(scratch, cams[v], size, stream=stream)
                splats.accumulate_prepared(scratch, isects, size, acc, masks[v], stream=stream)
                if keep is not None:
                    keep.append((acc.fg.read(stream), acc.bg.read(stream)))
                out.append(beta.eig(acc, mode, stream=stream))
            else:
                splats.render_responsibility(scratch, acc, cams[v], size, stream=stream)
                out.append(beta.eig(acc, mode, stream=stream))
        return np.array(out)

    def batched_round(mode, evidence):
        if evidence:
            return rnd.evidence(splats, beta, cams, masks, mode, stream=stream)
        return rnd.eig(splats, beta, cams, mode, stream=stream)

    def timed(fn, *a):
        fn(*a)
        times = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn(*a)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return float(np.median(times)), out

    tuning, tune_ms = rnd.autotune(splats, beta, cams, sf.EIG_FP64, stream=stream)
    result = {"workload": f"round: frame scene, {ROUND_VIEWS} views {ROUND_SIDE}x{ROUND_SIDE} on a "
                          f"radius-{ROUND_RADIUS} sphere, a,b log-uniform [1,1024]",
              "tuning": tuning, "reps": reps}
    for name, mode, evidence in (("responsibility_lut_f32", sf.EIG_LUT_F32, False),
                                 ("responsibility_fp64", sf.EIG_FP64, False),
                                 ("evidence_eig_lut_f32", sf.EIG_LUT_F32, True)):
        tp, ep = timed(plain_round, mode, evidence)
        tb, eb = timed(batched_round, mode, evidence)
        entry = {"plain_views_per_s": ROUND_VIEWS / tp, "batched_views_per_s": ROUND_VIEWS / tb,
                 "plain_ms_per_round": 1e3 * tp, "batched_ms_per_round": 1e3 * tb, "speedup": tp / tb,
                 "eig_identical": bool(np.array_equal(ep, eb))}
        if evidence:
            # Checked once, outside the timed rounds: every view's fg and bg
            # words (the masked evidence lift of the C2 round).
            kept = []
            plain_round(mode, True, kept)
            rnd.evidence(splats, beta, cams, masks, mode, stream=stream)
            entry["words_identical"] = all(
                np.array_equal(kept[v][0], rnd.evidence_words(v)[0].read(stream))
                and np.array_equal(kept[v][1], rnd.evidence_words(v)[1].read(stream)) for v in range(ROUND_VIEWS))
        result[name] = entry
    return result


UNEVEN_SPLATS, UNEVEN_SH, UNEVEN_VIEWS, UNEVEN_SIDES = 3_000_000, 4, 64, (256, 384, 512, 768, 1024)


def time_uneven_round(sf, ctx, stream, args):
    """The uneven batched lift (C4): 3M splats with SH degree 1 (clustered as
    the frame scene), 64 views whose sides are drawn from 256..1024, each
    with a 1-3 ellipse mask; per view the masked evidence lift and its FP64
    EIG (over fg + bg), as one batched graph (sf_round_evidence) against the
    plain per-view calls (one scratch per side, so the plain arm never
    reallocates). Responsibilities are the u32 lift; the adjoint's per-splat
    feature gradient is checked against it in the tests."""
    import torch

    from splatfield_b200 import synth

    attr, sh = synth.scene_clustered(UNEVEN_SPLATS, UNEVEN_SH, seed=7)
    splats = sf.Splats(attr, sh, ctx)
    del attr, sh
    rng = np.random.default_rng(11)
    sides = [int(x) for x in rng.choice(UNEVEN_SIDES, UNEVEN_VIEWS)]
    cams = synth.sphere_cameras(UNEVEN_VIEWS, ROUND_RADIUS, 9, sf.look_at)
    masks = [sf.Mask.from_bytes((s, s), synth.ellipse_mask(s, s, seed=300 + v), ctx) for v, s in enumerate(sides)]
    a, b = synth.beta_posterior(UNEVEN_SPLATS, seed=5)
    beta = sf.BetaState.from_host(a, b, ctx)
    acc = sf.Accumulators(UNEVEN_SPLATS, ctx)
    scratches = {s: sf.RenderScratch(UNEVEN_SPLATS, (s, s), ctx) for s in UNEVEN_SIDES}
    rnd = sf.Round(UNEVEN_SPLATS, [(s, s) for s in sides], ctx)
    rnd.set_tuning(lanes=8, raster_cull=1, raster_order=sf.ORDER_HYBRID)
    reps = 3

    def plain():
        out = []
        for v, s in enumerate(sides):
            isects = splats.prepare_isects(scratches[s], cams[v], (s, s), stream=stream)
            splats.accumulate_prepared(scratches[s], isects, (s, s), acc, masks[v], stream=stream)
            out.append(beta.eig(acc, sf.EIG_FP64, stream=stream))
        return np.array(out)

    def batched():
        return rnd.evidence(splats, beta, cams, masks, sf.EIG_FP64, stream=stream)

    def timed(fn):
        fn()
        times, out = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        return float(np.median(times)), out

    tp, ep = timed(plain)
    tb, eb = timed(batched)
    sizes = {str(s): sides.count(s) for s in UNEVEN_SIDES}
    return {"workload": f"uneven round: {UNEVEN_SPLATS // 1_000_000}M splats SH1 (8 Gaussian clusters), "
                        f"{UNEVEN_VIEWS} views with sides in {list(UNEVEN_SIDES)}, ellipse masks, "
                        "evidence lift + FP64 EIG per view",
            "views_per_side": sizes, "reps": reps,
            "plain_views_per_s": UNEVEN_VIEWS / tp, "batched_views_per_s": UNEVEN_VIEWS / tb,
            "plain_ms_per_round": 1e3 * tp, "batched_ms_per_round": 1e3 * tb, "speedup": tp / tb,
            "eig_identical": bool(np.array_equal(ep, eb))}


def cpu_other_configs(attr, sh, budget_s=25.0):
    """The CPU oracle on the other configs' plain paths, on the host's cores:
    one C0 frame (100k SH0 splats uniform in [-1,1]^3, 512x512, fov 60 deg)
    and the C2 round (per view: prepare, masked evidence lift, LUT EIG over
    fg + bg), as many of its 20 views as fit the budget."""
    import oracle as O

    from splatfield_b200 import synth

    a0, s0 = synth.scene_uniform(100_000, 1, 0)
    cam0 = O.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam0.fov[0], cam0.fov[1] = synth.fov_for(512, 512)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        O.rasterize(O.prepare(cam0, 512, 512, a0, s0, 1), 0, want_float=False)
        times.append(time.perf_counter() - t0)
    c0_ms = 1e3 * float(np.median(times))
    size = (ROUND_SIDE, ROUND_SIDE)
    a, b = synth.beta_posterior(N_SPLATS, seed=1)
    cams = synth.sphere_cameras(ROUND_VIEWS, ROUND_RADIUS, 2, O.look_at)
    scale = O.scale_for(*size)
    t0 = time.perf_counter()
    done = 0
    for v in range(ROUND_VIEWS):
        prep = O.prepare(cams[v], ROUND_SIDE, ROUND_SIDE, attr, sh, SH_PER_CH)
        fg, bg = O.evidence(prep, synth.ellipse_mask(ROUND_SIDE, ROUND_SIDE, seed=100 + v))
        O.eig(a, b, fg + bg, scale, 0)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    per_view = (time.perf_counter() - t0) / done
    return {"kind": "port", "cores": O.num_threads(),
            "c0_frame": {"ms": c0_ms, "sample": "3 frames of 100k SH0 splats at 512x512, median"},
            "c2_round": {"views_per_s": 1.0 / per_view, "ms_per_round": 1e3 * per_view * ROUND_VIEWS,
                         "sample": f"{done} of the round's {ROUND_VIEWS} views (evidence lift + LUT EIG)"}}


def run_reference(args, rank, world):
    """The reference arm: the CPU implementation of the path on this host."""
    if rank != 0:
        return
    import oracle as O

    attr, sh = make_scene()
    cams = orbit(O.look_at)
    budget_s = 120.0  # the whole arm stays within a few minutes at any --steps
    t_start = time.perf_counter()
    for i in range(min(args.warmup, 3)):
        prep = O.prepare(cams[i % N_CAMS], WIDTH, HEIGHT, attr, sh, SH_PER_CH)
        O.rasterize(prep, 0, want_float=False)
    t0 = time.perf_counter()
    done = 0
    for i in range(args.steps):
        prep = O.prepare(cams[i % N_CAMS], WIDTH, HEIGHT, attr, sh, SH_PER_CH)
        O.rasterize(prep, 0, want_float=False)
        done += 1
        if time.perf_counter() - t_start > budget_s:
            break
    dt = time.perf_counter() - t0
    fps = done / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "steps_run": done, "warmup": args.warmup, "ms_per_step": 1e3 * dt / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": WORKLOAD, "parallelism": "host cores"},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": O.num_threads(), "kind": "port",
                         "sample": f"{done} full frames of the workload (stops after {budget_s:.0f} s)"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "suous/splatfield runs only on wgpu (no Rust toolchain and no graphics stack here); "
                "its kernels are timed as the C++/OpenMP restatement used as the parity oracle",
    }
    print(json.dumps(line), flush=True)


def run_round_only(args):
    """Profiling mode: the eig_round workload's batched round alone, with the
    tuning the autotuner picks for it fixed, timed on the host clock."""
    import torch

    import splatfield_b200 as sf
    from splatfield_b200 import synth

    torch.cuda.set_device(0)
    ctx = sf.Context(0)
    attr, sh = make_scene()
    splats = sf.Splats(attr, sh, ctx)
    size = (ROUND_SIDE, ROUND_SIDE)
    a, b = synth.beta_posterior(N_SPLATS, seed=1)
    beta = sf.BetaState.from_host(a, b, ctx)
    cams = synth.sphere_cameras(ROUND_VIEWS, ROUND_RADIUS, 2, sf.look_at)
    rnd = sf.Round(N_SPLATS, [size] * ROUND_VIEWS, ctx)
    rnd.set_tuning(lanes=8, raster_cull=1, raster_order=sf.ORDER_HYBRID)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        rnd.eig(splats, beta, cams, sf.EIG_LUT_F32, stream=stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rnd.eig(splats, beta, cams, sf.EIG_LUT_F32, stream=stream)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.median(times))
    print(json.dumps({"round_only": args.steps, "ms_per_round": ms, "views_per_s": ROUND_VIEWS / (ms / 1e3)}))


def run_ours(args, rank, world):
    import torch

    import splatfield_b200 as sf
    from splatfield_b200 import _lib, replicas

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist = dist_mod
    ctx = sf.Context(local)
    attr, sh = make_scene()
    splats = sf.Splats(attr, sh, ctx)
    scratch = sf.RenderScratch(N_SPLATS, (WIDTH, HEIGHT), ctx)
    # Intersection capacity sized up front (the orbit's frames need up to
    # about 8.4M), so no reallocation falls inside a timed region.
    scratch.reserve(RESERVE_ISECTS)
    cams = orbit(sf.look_at)
    my_cams = replicas.replica_share(cams, rank, world)
    stream = torch.cuda.current_stream()
    size = (WIDTH, HEIGHT)

    for i in range(max(args.warmup, 3)):
        splats.render_with(scratch, my_cams[i % N_CAMS], size, stream=stream)
    torch.cuda.synchronize()
    if args.frames_only:
        # Profiling mode: just `steps` more frames, nothing else launched.
        for i in range(args.steps):
            splats.render_with(scratch, my_cams[i % N_CAMS], size, stream=stream)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"frames_only": args.steps, "kernels_per_frame":
                              (_lib.lib().sf_kernel_launches()) / (args.steps + max(args.warmup, 3))}))
        return

    # ---- device-timed frames
    launches0 = _lib.lib().sf_kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    path = [my_cams[i % N_CAMS] for i in range(N_CAMS)]
    with ClockSampler(local) as clocks:
        start.record(stream)
        done = 0
        while done < args.steps:
            k = min(N_CAMS, args.steps - done)
            splats.render_frames(scratch, path[:k], size, stream=stream)
            done += k
        end.record(stream)
        torch.cuda.synchronize()
    launches = _lib.lib().sf_kernel_launches() - launches0
    ms = replicas.max_over_ranks(start.elapsed_time(end), dist)
    fps = world * args.steps / (ms / 1e3)

    # ---- per-stage split: prepare (everything before the rasterizer) vs rasterizer
    prep_ms, rast_ms, stats = [], [], None
    for i in range(min(args.steps, 10)):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        isects = splats.prepare_isects(scratch, my_cams[i % N_CAMS], size, stream=stream)
        e1.record(stream)
        splats.finalize_rgb(scratch, isects, size, stream=stream)
        e2.record(stream)
        torch.cuda.synchronize()
        prep_ms.append(e0.elapsed_time(e1))
        rast_ms.append(e1.elapsed_time(e2))
        st = scratch.stats(stream)
        stats = st if stats is None else {k: stats[k] + st[k] for k in st}
    n_split = min(args.steps, 10)
    raster_ms = float(np.mean(rast_ms))
    pairs = stats["pairs_visited"] / n_split
    # Per-pair diagnostics from the counting form of the rasterizer (untimed).
    scratch.set_tuning(raster_detail=1)
    detail = None
    for i in range(n_split):
        isects = splats.prepare_isects(scratch, my_cams[i % N_CAMS], size, stream=stream)
        splats.finalize_rgb(scratch, isects, size, stream=stream)
        st = scratch.stats(stream)
        detail = st if detail is None else {k: detail[k] + st[k] for k in st}
    scratch.set_tuning()
    achieved = pairs * RASTER_FLOPS_PER_PAIR / (raster_ms / 1e3) / 1e12

    # ---- end to end through the host-facing calls: the camera path in
    # batches of N_CAMS frames (each image's read-back overlapping the next
    # frame), and one frame per call (read-back after each frame)
    batch_out = sf.pinned_empty((N_CAMS, HEIGHT, WIDTH), np.uint32)
    host_out = batch_out[0]
    path = [my_cams[i % N_CAMS] for i in range(N_CAMS)]
    for i in range(2):
        splats.render_to_host(scratch, my_cams[i], size, out=host_out, stream=stream)
    splats.render_frames_to_host(scratch, path, size, out=batch_out, stream=stream)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        k = min(N_CAMS, args.steps - done)
        splats.render_frames_to_host(scratch, path[:k], size, out=batch_out, stream=stream)
        done += k
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, dist)
    e2e_fps = world * args.steps / e2e_s
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        splats.render_to_host(scratch, my_cams[i % N_CAMS], size, out=host_out, stream=stream)
    single_s = replicas.max_over_ranks(time.perf_counter() - t0, dist)
    single_fps = world * args.steps / single_s
    del batch_out, host_out

    bwd = time_backward(sf, splats, scratch, attr, sh, my_cams[0], stream, args)
    eig_round = time_eig_round(sf, splats, ctx, stream, args)
    del scratch
    uneven = time_uneven_round(sf, ctx, stream, args)

    if rank != 0:
        return
    cpu_s, cpu_frames, cores = cpu_frame_time(attr, sh)
    cpu_more = cpu_other_configs(attr, sh)
    clk = clocks.summary()
    peaks, which = measured_peaks()
    line = {
        "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "splats": N_SPLATS, "sh_per_ch": SH_PER_CH, "width": WIDTH,
                   "height": HEIGHT, "cameras": N_CAMS,
                   "l2": "inputs larger than L2: 236 MB of splat planes read per frame vs 126 MB L2",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": 36,
                "d2h_bytes_per_step": WIDTH * HEIGHT * 4,
                "path": f"sf_render_frames_to_host ({N_CAMS}-camera path per call, camera by value, each RGBA8 "
                        "image to pinned host memory, read-back overlapping the next frame)",
                "single_frame": {"value": single_fps, "unit": "frames/s",
                                 "path": "sf_render_to_host (one frame per call, read-back after the frame)"}},
        "roofline": {"kernel": "raster_kernel<RGB>", "bound": "fp32", "achieved": achieved,
                     "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": achieved / FP32_PEAK_TFLOPS,
                     "traffic": RASTER_TRAFFIC_BYTES,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch, camera 3",
                     "pairs_per_frame": pairs,
                     "flops_per_pair": RASTER_FLOPS_PER_PAIR,
                     "pairs_processed_per_frame": detail["pairs_processed"] / n_split,
                     "accounting": "algorithmic pairs = 256 per tile-list entry walked before the "
                                   "tile's early exit (the reference's per-pixel loop); the kernel "
                                   "skips, per warp, the pairs it proves alpha < 1/255 for",
                     "peak_source": "derived: 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz (no measured FP32 peak)"},
        "stages_ms": {"prepare": float(np.mean(prep_ms)), "raster": raster_ms},
        "raster_stats": {k: v / n_split for k, v in detail.items()},
        "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": f"{cpu_frames} full frame(s) of the workload, median"},
        "cpu_other_configs": cpu_more,
        "backward": bwd,
        "eig_round": eig_round,
        "uneven_round": uneven,
        "clocks": clk,
        "gpu_launches": int(launches),
        "peaks": {"source": which, "hbm_gbs": peaks.get("hbm_gbs")},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames-only", action="store_true",
                    help="render warmup + steps frames and exit (for profilers)")
    ap.add_argument("--round-only", action="store_true",
                    help="run warmup + steps batched segmentation rounds (8 lanes, culling, hybrid order) "
                         "and exit (for profilers)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.round_only:
            run_round_only(args)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
