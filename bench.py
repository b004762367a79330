"""Benchmark: tetrahedral-cage deform + render frames on B200.

Workload (the reference's tet-cage configuration): 1,100,000 Gaussians drawn
from the seeded synthetic distribution with means scaled into [-1, 1]^3, a
5x5x5-cube / 750-tet / 216-vertex cage driven by the spring solver (bottom
layer pinned, stiffness 40, damping 4/s, dt 1/60), 1920x1080, a camera
orbiting at radius 4. One step = one frame: a host spring step, then Stage 1
(deform), Stage 2 (project), Stage 3 (bin + sort) and Stage 4 (composite).

The default line also carries, at 1 GPU: `stage4` ((pixel, entry) pairs/s and
the compositor's FP32 issue fraction), `error_floor` (a float64 evaluation of
the frame's formulas on a sample, against the f32 frame), `mvc` (the
polygon-cage leg below, with fewer frames) and `views` (the multi-view leg
below); `--no-legs` leaves them out. `e2e` runs the same frames through the C
ABI with the cage vertices uploaded and the RGBA8 frame read back every step,
three timed runs of K frames of which the median is reported (all three are
listed), and reports the host time per step by part.

Arms:
  python bench.py [--gpus N --steps K --warmup W]     this library (CUDA, sm_100a)
  python bench.py --impl reference ...                the reference's CPU path
                                                      (its Rayon backend restated
                                                      in oracle/, all host threads)
Multi-GPU (torchrun, one process per GPU): replicas; each rank renders its own
views (frames rank, rank+N, ...), no data exchange; value = all frames / max
rank time (weak scaling).

  python bench.py --workload views [--steps K --warmup W]
Batched multi-view workload (2,000,000 Gaussians drawn as above without
rescaling, the spring-driven tet cage deforming them once per step, 64 views
on a spiral, radius 3-5, elevation -30..60 degrees, resolutions cycling
640x360 / 1280x720 / 1920x1080): views/s of one step rendered as per-view
frame calls, as one batched call with per-view launches, and as one replayed
CUDA graph. One JSON line, 1 GPU.

  python bench.py --workload large [--steps K --warmup W]
Large-scene workload (6,000,000 Gaussians in the quantized f16 layout, four
384-tet spring cages over the upper half, the learned polygon cage for the
rest, 7680x4320 with 64-bit keys, camera orbiting at radius 4): frames/s and
per-stage times. One JSON line, 1 GPU.

  python bench.py --workload mvc [--steps K --warmup W]
Polygon-cage workload (3,000,000 Gaussians uniform in the unit ball, level-3
icosphere cage of radius 1.15 displaced by a smooth random field of amplitude
0.1, moved every frame by another such field, 1920x1080): Stage 1 with exact
stored MVC bindings against Stage 1 with the learned weight field trained on
2,000,000 interior points with exact weights, on the same frames; the learned
deformation's error is judged by the exact one. One JSON line, 1 GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "ms/frame per stage & views/s; learned vs exact MVC deform time at ≤1e-3 err"
UNIT = "views/s"
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0


def radix_digits(args) -> str:
    """Digit widths of the entry sort's passes over the tile bits, e.g. "7+6"."""
    tw, th = {0: (16, 16), 1: (8, 8), 2: (32, 16)}[getattr(args, "tile_shape", 0)]
    tiles = ((args.width + tw - 1) // tw) * ((args.height + th - 1) // th)
    tile_bits = max(1, (tiles - 1).bit_length())
    rb = args.radix_bits
    if rb == 0:
        passes = (tile_bits + 7) // 8
        rb = max(4, -(-tile_bits // passes))
    widths, left = [], tile_bits
    while left > 0:
        widths.append(min(rb, left))
        left -= rb
    return "+".join(str(w) for w in widths)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["tet", "mvc", "views", "large"], default="tet")
    ap.add_argument("--views", type=int, default=64)
    ap.add_argument("--gaussians", type=int, default=None,
                    help="default 1,100,000 (tet) or 3,000,000 (mvc)")
    ap.add_argument("--train-points", type=int, default=2_000_000)
    ap.add_argument("--train-steps", type=int, default=6000)
    ap.add_argument("--fallback-quantile", type=float, default=0.99,
                    help="residual quantile above which bound Gaussians keep exact weights")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="default workload only: skip the error floor and the MVC and "
                         "multi-view legs")
    ap.add_argument("--entry-sort", type=int, default=0,
                    help="tile-entry sort: 0 auto, 1 radix passes, 2 one-pass tile transpose")
    ap.add_argument("--radix-bits", type=int, default=0,
                    help="entry-sort digit width (0 = balanced digits of at most 8 bits)")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (a stable launch list for profiling)")
    ap.add_argument("--tile-shape", type=int, default=0,
                    help="screen tile: 0 = 16x16 (the reference's), 1 = 8x8, 2 = 32x16")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload(args):
    from cindergs_b200 import workloads
    return workloads.tet_cage_orbit(n=args.gaussians or 1_100_000, width=args.width,
                                    height=args.height)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        mx.append(float(parts[2]))
                    except ValueError:
                        continue
                    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                             "sw_power_cap"]
                    for name, v in zip(names, parts[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(name)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_frames(wl, bind_tet, bind_w, frames, start_frame=0):
    """Renders `frames` frames with the restated reference CPU backend; returns
    (seconds per frame list, threads)."""
    import oracle
    m = wl.cage.mesh
    times = []
    for f in range(frames):
        cam = wl.camera(start_frame + f)
        comp = wl.compositor(cam)
        t0 = time.perf_counter()
        oracle.ref_frame(wl.scene.as_dict(), cam.to_array(), wl.width, wl.height,
                         np.asarray(comp.background_color, np.float32),
                         np.asarray(comp.camera_position, np.float32), wl.sh_degree,
                         cage=dict(verts=wl.cage.vertices(), elems=m.elements, inv_dm=m.inv_dm,
                                   bind_tet=bind_tet, bind_w=bind_w),
                         split_thr=wl.strain_split_threshold, mip=wl.mip_filter_3d_var)
        times.append(time.perf_counter() - t0)
        wl.step()
    return times, oracle.threads()


def config_dict(args, wl, world):
    return {"workload": "tet-cage deform + render, orbit camera",
            "gaussians": wl.scene.count, "width": args.width, "height": args.height,
            "cage": "5x5x5 cubes x 6 tets (750 tets, 216 vertices), springs k=40 c=4 dt=1/60",
            "sh_degree": 3, "keys": "32-bit tile|depth", "radix_digits": radix_digits(args),
            "entry_sort": ["auto (radix)", "radix", "tile transpose"][args.entry_sort],
            "tile": ["16x16", "8x8", "32x16"][args.tile_shape],
            "l2": "inputs larger than L2 (resident scene 255 MB + 26M tile entries)",
            "parallelism": f"replicas x{world} (views sharded, no exchange)"}


def run_reference(args):
    """--impl reference: the reference's CPU path (restated) on host cores."""
    world, rank, local = dist_setup(args)
    if rank != 0:
        return 0
    import oracle
    from cindergs_b200 import workloads  # noqa: F401
    wl = workload(args)
    m = wl.cage.mesh
    bt, bw = oracle.bind_points(wl.scene.positions, m.rest_vertices, m.elements, m.inv_dm,
                                m.bounds())
    for _ in range(args.warmup):
        wl.step()
    times, threads = cpu_reference_frames(wl, bt, bw, args.steps)
    total = sum(times)
    value = args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(args, wl, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full frames of the workload"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args)
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from cindergs_b200 import GpuPipelineState
    from cindergs_b200.replicas import max_over_ranks

    wl = workload(args)
    stream = torch.cuda.Stream(device=local)
    st = GpuPipelineState(local, stream=stream.cuda_stream)
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    frame = rank

    def render(profile=False, timings=True):
        nonlocal frame
        wl.step()
        cam = wl.camera(frame)
        frame += world
        return st.execute_frame_gpu(wl.scene, cages, cam, wl.compositor(cam),
                                    wl.strain_split_threshold, wl.mip_filter_3d_var,
                                    1.0 / 255.0, 0.5, profile_stages=profile,
                                    stage_timings=timings, radix_bits=args.radix_bits,
                                    entry_sort=args.entry_sort, tile_shape=args.tile_shape)

    for _ in range(max(args.warmup, 3)):
        render()
    # Kernel launch shapes (block sizes) chosen by the autotuner on the
    # workload's current frame; every shape renders the same frame.
    from cindergs_b200 import autotune
    cam_t = wl.camera(frame)
    if args.no_tune:
        shape = {k: v[0] for k, v in autotune.LAUNCH_CHOICES.items()}
        st.set_launch_shape(**shape)
    else:
        shape, _ = autotune.tune_launch_shape(st, wl.scene, cages, cam_t, wl.compositor(cam_t),
                                              radix_bits=args.radix_bits,
                                              entry_sort=args.entry_sort,
                                              tile_shape=args.tile_shape)
    # Per-stage device times of a few representative frames (not timed).
    stage_rows = [render(profile=True, timings=True) for _ in range(3)]
    st.synchronize()

    def barrier():
        torch.cuda.synchronize(local)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)

    # ---- timed region: inputs resident in HBM, CUDA events on the library
    # stream around K frames as a caller runs them (no per-kernel events);
    # then K more frames with an event pair around every launch, for the
    # per-kernel device times (their own total is reported beside `value`)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    clock = ClockSampler(local)
    barrier()
    with clock:
        start.record(stream)
        for _ in range(args.steps):
            render(profile=False, timings=False)
        end.record(stream)
        barrier()
        st.kernel_profile_reset()
        pstart = torch.cuda.Event(enable_timing=True)
        pend = torch.cuda.Event(enable_timing=True)
        pstart.record(stream)
        for _ in range(args.steps):
            render(profile=True, timings=False)
        pend.record(stream)
        barrier()
    ms = max_over_ranks(start.elapsed_time(end), device=f"cuda:{local}")
    ms_profiled = max_over_ranks(pstart.elapsed_time(pend), device=f"cuda:{local}")
    kp = st.kernel_profile()
    value = world * args.steps / (ms / 1000.0)

    # ---- e2e: through the C ABI with host buffers, copies inside the timed
    # region. Per step: the host spring step, the cage vertices uploaded
    # (cgs_cage_vertices_update), the frame enqueued (cgs_execute_frame, no
    # host wait), and the RGBA8 frame read back into page-locked host memory
    # (cgs_readback_rgba8_async: frame i's copy runs while frame i + 1
    # renders; each image is waited for before it is reused). Cameras and
    # compositor blocks are host inputs prepared like the caller's own
    # structs; the host time per step is reported by part.
    import ctypes
    from cindergs_b200 import _abi
    lib, ctx = st._lib, st.handle
    params_c = _abi.CgsFrameParams(float(wl.strain_split_threshold), float(wl.mip_filter_3d_var),
                                   1.0 / 255.0, 0.5, 0, 0, 0, int(args.radix_bits),
                                   int(args.entry_sort), int(args.tile_shape))
    pinned_out = [torch.empty((args.height, args.width, 4), dtype=torch.uint8).pin_memory()
                  for _ in range(2)]
    out_ptr = [ctypes.c_void_p(t.data_ptr()) for t in pinned_out]
    nverts = wl.cage.mesh.rest_vertices.shape[0]
    vert_host = np.empty((nverts, 3), np.float32)
    ticket = ctypes.c_uint64()

    def e2e_run(frame0):
        """K frames through the C ABI; returns (ms over ranks, host ms by part, wall, device)."""
        e2e_frames = [frame0 + world * i for i in range(args.steps)]
        cams_c = [st._camera(wl.camera(f)) for f in e2e_frames]
        comps_c = [st._compositor(wl.compositor(wl.camera(f))) for f in e2e_frames]
        host_ms = {"spring_step": 0.0, "enqueue": 0.0, "readback_wait": 0.0}
        barrier()
        t0 = time.perf_counter()
        e2e_start = torch.cuda.Event(enable_timing=True)
        e2e_end = torch.cuda.Event(enable_timing=True)
        e2e_start.record(stream)
        prev_ticket = None
        for step in range(args.steps):
            ta = time.perf_counter()
            wl.step()
            vert_host[:] = wl.cage.vertices()
            tb = time.perf_counter()
            _abi.check(lib.cgs_cage_vertices_update(ctx, vert_host.ctypes.data_as(ctypes.c_void_p),
                                                    nverts), "cgs_cage_vertices_update", ctx)
            _abi.check(lib.cgs_execute_frame(ctx, ctypes.byref(cams_c[step]),
                                             ctypes.byref(comps_c[step]), ctypes.byref(params_c),
                                             None), "cgs_execute_frame", ctx)
            _abi.check(lib.cgs_readback_rgba8_async(ctx, out_ptr[step % 2], args.width,
                                                    args.height, ctypes.byref(ticket)),
                       "cgs_readback_rgba8_async", ctx)
            tc = time.perf_counter()
            if prev_ticket is not None:  # the previous frame's pixels are on the host
                _abi.check(lib.cgs_readback_wait(ctx, prev_ticket), "cgs_readback_wait", ctx)
            prev_ticket = ticket.value
            td = time.perf_counter()
            host_ms["spring_step"] += (tb - ta) * 1000.0
            host_ms["enqueue"] += (tc - tb) * 1000.0
            host_ms["readback_wait"] += (td - tc) * 1000.0
        if prev_ticket is not None:
            _abi.check(lib.cgs_readback_wait(ctx, prev_ticket), "cgs_readback_wait", ctx)
        e2e_end.record(stream)
        barrier()
        wall = (time.perf_counter() - t0) * 1000.0
        dev = e2e_start.elapsed_time(e2e_end)
        return max_over_ranks(max(dev, wall), device=f"cuda:{local}"), host_ms, wall, dev

    # One untimed run first (the readback path's first use: its snapshot
    # buffers, copy stream and page-locked staging), then three runs of K
    # frames each, every copy inside each timed region; the median run is
    # reported (the GPUs' host links are shared with other jobs, and one
    # stalled copy should not set the figure), all three are listed.
    e2e_run(frame)
    frame += world * args.steps
    e2e_runs = []
    for _ in range(3):
        e2e_runs.append(e2e_run(frame))
        frame += world * args.steps
    e2e_ms, host_ms, e2e_wall, e2e_dev = sorted(e2e_runs, key=lambda r: r[0])[1]
    e2e_value = world * args.steps / (e2e_ms / 1000.0)
    e2e_all = [world * args.steps / (r[0] / 1000.0) for r in e2e_runs]
    e2e_parts = {k: v / args.steps for k, v in host_ms.items()}
    e2e_parts["wall_ms_per_step"] = e2e_wall / args.steps
    e2e_parts["device_ms_per_step"] = e2e_dev / args.steps

    # ---- the same frames with 32x16 screen tiles (the autotuner's choice at
    # 1080p: fewer tile entries to bin and sort, more candidates per pixel)
    alt = None
    if args.tile_shape == 0:
        def render_alt(count_entries=False):
            nonlocal frame
            wl.step()
            cam = wl.camera(frame)
            frame += world
            return st.execute_frame_gpu(wl.scene, cages, cam, wl.compositor(cam),
                                        wl.strain_split_threshold, wl.mip_filter_3d_var,
                                        1.0 / 255.0, 0.5, stage_timings=count_entries,
                                        tile_shape=2)
        for _ in range(max(args.warmup, 3)):
            last_alt = render_alt(True)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        barrier()
        a0.record(stream)
        for _ in range(args.steps):
            render_alt()
        a1.record(stream)
        barrier()
        alt_ms = max_over_ranks(a0.elapsed_time(a1), device=f"cuda:{local}")
        alt = {"views_per_s": world * args.steps / (alt_ms / 1000.0),
               "ms_per_step": alt_ms / args.steps,
               "tile_entries": last_alt.total_tile_entries}

    # ---- one more frame of the workload with the f32 image written: the
    # float64 error floor of its formulas on a sample (1 GPU)
    floor = None
    if world == 1 and not args.no_legs and args.tile_shape == 0:
        from cindergs_b200 import error_floor
        wl.step()
        cam_f = wl.camera(frame)
        comp_f = wl.compositor(cam_f)
        st.execute_frame_gpu(wl.scene, cages, cam_f, comp_f, wl.strain_split_threshold,
                             wl.mip_filter_3d_var, 1.0 / 255.0, 0.5, force_stage3=True,
                             write_f32=True)
        floor = error_floor.frame_floor(st, wl.scene, cages, cam_f, comp_f)

    if rank == 0:
        hbm, peak_kind = peaks()
        kernels = {}
        for name, d in kp.items():
            if name == "clear" or d["launches"] == 0:
                continue
            avg_ms = d["ms"] / max(args.steps, 1)
            gbs = d["alg_bytes"] / (d["ms"] / 1000.0) / 1e9 if d["ms"] > 0 else 0.0
            kernels[name] = {"ms_per_frame": avg_ms, "launches": d["launches"],
                             "alg_bytes_per_frame": d["alg_bytes"] // max(args.steps, 1),
                             "achieved_gbs": gbs, "hbm_frac": gbs / hbm}
        dom = max(kernels, key=lambda k: kernels[k]["ms_per_frame"])
        dk = kernels[dom]
        per_launch_bytes = kp[dom]["alg_bytes"] / kp[dom]["launches"]
        per_launch_ms = kp[dom]["ms"] / kp[dom]["launches"]
        traffic = None
        tp = os.path.join(ROOT, "profiles", "dram_traffic.json")
        if os.path.exists(tp):
            try:
                traffic = json.load(open(tp)).get(dom)
            except Exception:
                traffic = None
        gpu_launches = sum(d["launches"] for n_, d in kp.items() if n_ != "clear")
        stages = {k: statistics.median(getattr(r, k) for r in stage_rows)
                  for k in ("stage1_deform_ms", "stage2_project_ms", "stage3_bin_sort_ms",
                            "stage4_composite_ms")}
        last = stage_rows[-1]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": dict(config_dict(args, wl, world),
                                                launch_shape=shape),
            "stages_ms": stages,
            "ms_per_step_with_kernel_events": ms_profiled / args.steps,
            "frame_counts": {"active_gaussians": last.active_gaussians,
                             "surviving_gaussians": last.surviving_gaussians,
                             "tile_entries": last.total_tile_entries},
            "kernels": kernels,
            "roofline": {"kernel": dom, "bound": "hbm",
                         "achieved": per_launch_bytes / (per_launch_ms / 1000.0) / 1e9,
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": (per_launch_bytes / (per_launch_ms / 1000.0) / 1e9) / hbm,
                         "traffic": traffic, "alg_bytes_per_launch": per_launch_bytes},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step":
                    int(wl.cage.mesh.rest_vertices.nbytes) + 96 + 48 + 40,
                    "d2h_bytes_per_step": int(args.width * args.height * 4 + 36),
                    "host_ms_per_step": e2e_parts,
                    "runs": e2e_all, "reported": "median of 3 timed runs of K frames",
                    "path": "C ABI: cage vertices up, frame, asynchronous RGBA8 readback"},
            "gpu_launches": gpu_launches,
            "clocks": clock.summary(),
        }
        if alt is not None:
            line["tile_32x16"] = alt
        # Stage 4 is FP32/SFU issue-bound: (pixel, entry) pairs per second,
        # from the entries the compositor gathered (its algorithmic bytes are
        # 52 B per gathered entry + 8 B per tile + 4 B per pixel), and the FP32
        # issue rate those pairs need at 24 FP32 operations each (the blend
        # loop's arithmetic per pair that passes the opacity and q cuts)
        # against 128 FP32 lanes per SM at the sampled SM clock.
        ck = kp.get("composite")
        if ck and ck["launches"]:
            tw, th = {0: (16, 16), 1: (8, 8), 2: (32, 16)}[args.tile_shape]
            tiles = ((args.width + tw - 1) // tw) * ((args.height + th - 1) // th)
            fetched = max(ck["alg_bytes"] / max(args.steps, 1) - 4 * args.width * args.height
                          - 8 * tiles, 0) / 52.0
            pairs = fetched * tw * th
            cms = ck["ms"] / max(args.steps, 1)
            clk = (line["clocks"].get("sm_mhz") or 1965.0) * 1e6
            pps = pairs / (cms / 1000.0)
            line["stage4"] = {"ms_per_frame": cms, "entries_gathered_per_frame": fetched,
                              "pixel_entry_pairs_per_frame": pairs, "pairs_per_s": pps,
                              "fp32_ops_per_pair": 24,
                              "fp32_issue_frac": pps * 24 / (148 * 128 * clk),
                              "hbm_frac": kernels.get("composite", {}).get("hbm_frac")}
        if floor is not None:
            line["error_floor"] = floor
        if world == 1 and not args.no_legs:
            st.close()
            st = None
            torch.cuda.empty_cache()
            # the legs' own CPU baselines run in their standalone workloads
            for name, fn, over in (("mvc", mvc_result, {"steps": min(args.steps, 10)}),
                                   ("views", views_result, {"steps": min(args.steps, 5)})):
                try:
                    sub = argparse.Namespace(**{**vars(args), **over, "gaussians": None,
                                                "no_cpu_baseline": True, "width": 1920,
                                                "height": 1080})
                    line[name] = fn(sub)
                except Exception as exc:  # a leg that fails is reported, not fatal
                    line[name] = {"failed": f"{type(exc).__name__}: {exc}"}
                torch.cuda.empty_cache()
        if world == 1 and not args.no_cpu_baseline:
            try:
                bt = cages.bind_tet
                bw = cages.bind_w
                times, threads = cpu_reference_frames(wl, bt, bw, 1, start_frame=frame)
                line["cpu_baseline"] = {"value": 1.0 / times[0], "unit": UNIT, "cores": threads,
                                        "kind": "port",
                                        "sample": "1 full frame of the workload (reference "
                                                  "CPU path restated in oracle/)"}
            except Exception as exc:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                        "kind": "port", "sample": f"failed: {exc}"}
        print(json.dumps(line), flush=True)
    if st is not None:
        st.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_mvc(args):
    """Exact vs learned MVC Stage 1 on the polygon-cage workload (1 GPU)."""
    print(json.dumps(mvc_result(args)), flush=True)
    return 0


def mvc_result(args) -> dict:
    """The polygon-cage leg: exact stored bindings vs the learned field
    (cached codes and per-frame network), the learned error judged by the
    exact deformation of the same frames."""
    import torch
    from cindergs_b200 import GpuPipelineState, _abi, workloads
    torch.cuda.set_device(0)
    n = args.gaussians or 3_000_000
    wl = workloads.mvc_cage_sphere(n=n, width=args.width, height=args.height)
    stream = torch.cuda.Stream(device=0)
    st = GpuPipelineState(0, stream=stream.cuda_stream)
    st.upload_scene(wl.scene)
    st.upload_cages(None)
    st.mvc_cage_upload(wl.cage)
    stage1 = ("mvc", "field", "deform")

    def timed(t0_event_fn):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = t0_event_fn()
        b.record(stream)
        torch.cuda.synchronize()
        return out, a.elapsed_time(b)

    def frames(first):
        """warm-up, then `steps` profiled frames from frame `first`; returns
        (per-kernel ms per frame, frame ms, deformed positions of frame `first`)."""
        def one(f, profile, timings):
            st.mvc_vertices_update(wl.vertices(f))
            cam = wl.camera(f)
            return st.execute_frame_gpu(wl.scene, None, cam, wl.compositor(cam), 0.0, 0.0,
                                        profile_stages=profile, stage_timings=timings)
        one(first, False, True)
        pos = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32).reshape(-1, 3).copy()
        for f in range(max(args.warmup, 3)):
            one(first + 1 + f, False, False)
        st.synchronize()
        st.kernel_profile_reset()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for f in range(args.steps):
            one(first + 1 + f, True, False)
        b.record(stream)
        st.synchronize()
        torch.cuda.synchronize()
        kp = st.kernel_profile()
        per = {k: dict(ms=d["ms"] / args.steps, alg_bytes=d["alg_bytes"] // args.steps,
                       alg_flops=d["alg_flops"] // args.steps, launches=d["launches"])
               for k, d in kp.items() if d["launches"]}
        return per, a.elapsed_time(b) / args.steps, pos

    # ---- exact: inside test + weights + central-difference gradients, stored
    nb, bind_ms = timed(st.mvc_bind)
    k_exact, frame_exact, pos_exact = frames(0)
    s1_exact = sum(k_exact.get(k, {}).get("ms", 0.0) for k in stage1)

    # ---- training data and training (exact weights from the MVC kernel)
    pts = torch.from_numpy(wl.training_points(args.train_points)).to("cuda:0")
    w, weights_ms = timed(lambda: st.mvc_weights(pts))
    st.mvc_field_create(seed=1)
    loss, train_ms = timed(lambda: st.mvc_field_train(pts, w, steps=args.train_steps, batch=4096,
                                                      lr=2e-3, lam=0.05, seed=5))
    del w, pts
    torch.cuda.empty_cache()

    # ---- learned bindings: fallback threshold at a quantile of the residuals
    _, _, enc = st.mvc_field_layout()
    s = 1.0 / float(enc[3])
    rng = np.random.default_rng(7)
    sample = wl.scene.positions[rng.choice(n, min(n, 200_000), replace=False)]
    raw, _ = st.mvc_field_infer(sample, rest=True)
    res = np.linalg.norm(raw - sample, axis=1) / s
    thr = float(np.quantile(res, args.fallback_quantile))
    (nbl, nfb), pf_bind_ms = timed(lambda: st.mvc_bind_learned(thr, per_frame=True))
    k_pf, frame_pf, pos_pf = frames(0)
    s1_pf = sum(k_pf.get(k, {}).get("ms", 0.0) for k in stage1)
    (nbl, nfb), learned_bind_ms = timed(lambda: st.mvc_bind_learned(thr))
    k_learned, frame_learned, pos_learned = frames(0)
    s1_learned = sum(k_learned.get(k, {}).get("ms", 0.0) for k in stage1)
    mode_diff = float((np.linalg.norm(pos_learned[:n].astype(np.float64) - pos_pf[:n], axis=1)
                       / (1.0 / float(enc[3]))).max())

    err = np.linalg.norm(pos_learned[:n].astype(np.float64) - pos_exact[:n], axis=1) / s
    cpu = None
    if not args.no_cpu_baseline:
        # the reference's CPU path for this step: deform_scene_cpu with stored
        # exact bindings (restated in oracle/, one thread), on a sample
        import oracle
        m = min(n, 10_000)
        sidx = np.random.default_rng(11).choice(n, m, replace=False)
        sp = wl.scene.positions[sidx]
        inside, wgs = oracle.mvc_bind(sp, wl.cage.rest_vertices, wl.cage.triangles)
        t0 = time.perf_counter()
        oracle.mvc_deform(sp, wl.scene.covariances_3d[sidx], wl.scene.opacities[sidx], inside,
                          wgs, wl.vertices(1))
        cpu_ms = (time.perf_counter() - t0) * 1000.0 * n / m
        cpu = {"value": cpu_ms, "unit": "ms/frame (Stage 1)", "cores": 1, "kind": "port",
               "sample": f"exact MVC deformation with stored bindings (deform_scene_cpu "
                         f"restated in oracle/) of {m:,} of the Gaussians, scaled to {n:,}"}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        pk["kind"] = "measured"
    except Exception:
        pk = {"hbm_gbs": FALLBACK_HBM_GBS, "bf16_tflops": FALLBACK_BF16_TFLOPS, "kind": "fallback"}
    fk = k_pf.get("field", {})
    ck = k_learned.get("field", {})
    code_gbs = ck["alg_bytes"] / (ck["ms"] / 1000.0) / 1e9 if ck.get("ms") else None
    field_tflops = fk["alg_flops"] / (fk["ms"] / 1000.0) / 1e12 if fk.get("ms") else None
    mk = k_exact.get("mvc", {})
    mvc_gbs = mk["alg_bytes"] / (mk["ms"] / 1000.0) / 1e9 if mk.get("ms") else None
    line = {
        "metric": "MVC Stage 1 ms/frame: learned weight field vs exact stored bindings",
        "value": s1_learned, "unit": "ms/frame", "higher_is_better": False, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "dtype": "bf16 MLP (fp32 accumulate)",
        "data": "synthetic",
        "config": {"workload": "polygon-cage MVC, exact vs learned", "gaussians": n,
                   "cage": "icosphere L3 r=1.15, 642 vertices / 1280 triangles, displaced 0.1",
                   "motion": "moving smooth random field, amplitude 0.1",
                   "width": args.width, "height": args.height,
                   "train_points": args.train_points, "train_steps": args.train_steps},
        "stage1_ms": {"exact": s1_exact, "learned": s1_learned,
                      "speedup": s1_exact / s1_learned if s1_learned else None,
                      "learned_per_frame_network": s1_pf,
                      "speedup_per_frame_network": s1_exact / s1_pf if s1_pf else None},
        "frame_ms": {"exact": frame_exact, "learned": frame_learned,
                     "learned_per_frame_network": frame_pf},
        "kernels_ms": {"exact": {k: v["ms"] for k, v in k_exact.items()},
                       "learned": {k: v["ms"] for k, v in k_learned.items()},
                       "learned_per_frame_network": {k: v["ms"] for k, v in k_pf.items()}},
        "modes": {"learned": "network codes kept per Gaussian (1 KB), output layer per frame",
                  "learned_per_frame_network": "whole network per Gaussian every frame",
                  "max_rel_position_difference": mode_diff},
        "exact_weights": {"bind_ms": bind_ms, "bound": nb,
                          "stored_bytes": nb * wl.cage.num_vertices * 16,
                          "train_weights_ms": weights_ms},
        "learned": {"bind_ms": learned_bind_ms, "bind_ms_per_frame_network": pf_bind_ms,
                    "bound": nbl, "fallbacks": nfb, "code_bytes": (nbl - nfb) * 1024,
                    "residual_threshold": thr, "train_ms": train_ms, "loss_terms": loss},
        "error": {"judge": "exact MVC deformation of the same frame",
                  "mean_rel_position": float(err.mean()),
                  "p99_rel_position": float(np.quantile(err, 0.99)),
                  "max_rel_position": float(err.max()), "relative_to": "cage half-extent s",
                  "s": s},
        "cpu_baseline": cpu,
        "roofline": {
            "field": {"bound": "tensor", "achieved": field_tflops,
                      "peak": pk.get("bf16_tflops"), "unit": "TFLOP/s",
                      "frac": field_tflops / pk["bf16_tflops"] if field_tflops else None,
                      "flops_per_launch": fk.get("alg_flops")},
            "field_codes": {"bound": "hbm", "achieved": code_gbs, "peak": pk.get("hbm_gbs"),
                            "unit": "GB/s",
                            "frac": code_gbs / pk["hbm_gbs"] if code_gbs else None,
                            "bytes_per_launch": ck.get("alg_bytes")},
            "mvc_exact": {"bound": "hbm", "achieved": mvc_gbs, "peak": pk.get("hbm_gbs"),
                          "unit": "GB/s", "frac": mvc_gbs / pk["hbm_gbs"] if mvc_gbs else None,
                          "bytes_per_launch": mk.get("alg_bytes")},
            "peak_kind": pk["kind"]},
    }
    st.close()
    return line


def run_views(args):
    """Per-view frames vs batched views vs a replayed CUDA graph (1 GPU)."""
    print(json.dumps(views_result(args)), flush=True)
    return 0


def views_result(args) -> dict:
    """The batched multi-view leg: 64 autotuned views per step as per-view
    frame calls, one batched call and one replayed CUDA graph."""
    import torch
    from cindergs_b200 import GpuPipelineState, workloads
    torch.cuda.set_device(0)
    n = args.gaussians or 2_000_000
    wl, cams, comps = workloads.multiview_cage(n=n, views=args.views)
    stream = torch.cuda.Stream(device=0)
    st = GpuPipelineState(0, stream=stream.cuda_stream)
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    imgs = st.view_images(comps)
    pixels = sum(c.screen_width * c.screen_height for c in comps)
    from cindergs_b200 import _abi, autotune
    wl.step()
    tuned = autotune.tune_views(st, wl.scene, cages, cams, comps)
    tss, rbs, ess = autotune.per_view(tuned, comps)

    def per_view_frames():
        wl.step()
        for v, (cam, comp) in enumerate(zip(cams, comps)):
            st.execute_frame_gpu(wl.scene, cages, cam, comp, force_stage3=True,
                                 stage_timings=False, radix_bits=rbs[v], entry_sort=ess[v],
                                 tile_shape=tss[v])

    def batched(graph):
        wl.step()
        return st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=graph,
                                radix_bits=rbs, entry_sort=ess, tile_shape=tss)

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        st.synchronize()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        out = [fn() for _ in range(args.steps)]
        b.record(stream)
        st.synchronize()
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1000.0 / args.steps
        return a.elapsed_time(b) / args.steps, wall, out

    # size the key buffers for the largest view (a frame waited for is
    # re-binned with grown buffers when its entries overflowed)
    wl.step()
    for v, (cam, comp) in enumerate(zip(cams, comps)):
        st.execute_frame_gpu(wl.scene, cages, cam, comp, force_stage3=True, stage_timings=True,
                             radix_bits=rbs[v], entry_sort=ess[v], tile_shape=tss[v])
    clock = ClockSampler(0)
    with clock:
        plain_ms, plain_wall, _ = timed(per_view_frames)
        eager_ms, eager_wall, _ = timed(lambda: batched(False))
        graph_ms, graph_wall, gst = timed(lambda: batched(True))
    replays = sum(1 for x in gst if x["graph_replayed"])
    nv = len(cams)
    # Per-kernel device time and algorithmic HBM bytes of one step of
    # per-view frames: the step's floor is the sum over kernels of bytes /
    # the measured copy bandwidth, a bound for any batching of the views.
    st.kernel_profile_reset()
    wl.step()
    for v, (cam, comp) in enumerate(zip(cams, comps)):
        st.execute_frame_gpu(wl.scene, cages, cam, comp, force_stage3=True, profile_stages=True,
                             radix_bits=rbs[v], entry_sort=ess[v], tile_shape=tss[v])
    st.synchronize()
    hbm = peaks()[0]
    per_kernel, floor_ms = {}, 0.0
    for name, k in st.kernel_profile().items():
        if k["launches"] == 0:
            continue
        f = k["alg_bytes"] / (hbm * 1e9) * 1e3
        floor_ms += f
        per_kernel[name] = {"ms": k["ms"], "launches": k["launches"],
                            "alg_bytes": k["alg_bytes"], "hbm_floor_ms": f,
                            "frac": f / k["ms"] if k["ms"] > 0 else None}
    cpu = None
    if not args.no_cpu_baseline:
        # one 1280x720 view through the restated reference CPU backend
        import oracle
        v = 1
        m = wl.cage.mesh
        _, _, _, flat_bt, flat_bw = cages.flatten()  # 0xFFFFFFFF marks unbound Gaussians
        t0 = time.perf_counter()
        oracle.ref_frame(wl.scene.as_dict(), cams[v].to_array(), comps[v].screen_width,
                         comps[v].screen_height, np.asarray(comps[v].background_color, np.float32),
                         np.asarray(comps[v].camera_position, np.float32), 3,
                         cage=dict(verts=wl.cage.vertices(), elems=m.elements, inv_dm=m.inv_dm,
                                   bind_tet=flat_bt, bind_w=flat_bw))
        cpu = {"value": 1.0 / (time.perf_counter() - t0), "unit": "views/s",
               "cores": __import__("oracle").threads(), "kind": "port",
               "sample": "one 1280x720 view of the step (reference CPU path restated in oracle/)"}
    line = {
        "metric": "views/s of a 64-view step: one replayed CUDA graph vs per-view frame launches",
        "value": nv / (graph_ms / 1000.0), "unit": "views/s", "higher_is_better": True,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": graph_ms,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched multi-view, tet cage per step", "gaussians": n,
                   "views": nv, "resolutions": "640x360 / 1280x720 / 1920x1080 cycling",
                   "pixels_per_step": pixels, "cameras": "spiral r 3-5, elevation -30..60"},
        "views_per_s": {"per_view_frames": nv / (plain_ms / 1000.0),
                        "batched_eager": nv / (eager_ms / 1000.0),
                        "graph": nv / (graph_ms / 1000.0)},
        "ms_per_step": {"per_view_frames": plain_ms, "batched_eager": eager_ms, "graph": graph_ms},
        "wall_ms_per_step": {"per_view_frames": plain_wall, "batched_eager": eager_wall,
                             "graph": graph_wall},
        "speedup_graph_vs_per_view_frames": plain_ms / graph_ms,
        "graph_replays": replays,
        "autotuned": {f"{w}x{h}": {"tile": "x".join(map(str, _abi.TILE_SHAPES[ts])),
                                  "radix_bits": rb, "entry_sort": ["auto", "radix", "transpose"][es],
                                  "stage34_ms": ms} for (w, h), (ts, rb, es, ms) in tuned.items()},
        "tile_entries_per_step": gst[-1]["total_tile_entries"] if gst else None,
        "per_kernel_one_step": per_kernel,
        "hbm_floor_ms_per_step": floor_ms,
        "max_speedup_over_per_view_frames_at_hbm_floor": plain_ms / floor_ms if floor_ms else None,
        "cpu_baseline": cpu,
        "clocks": clock.summary(),
    }
    st.close()
    return line


def run_large(args):
    """Quantized 6M scene, four tet cages + learned polygon cage, 8K (1 GPU)."""
    import torch
    from cindergs_b200 import CageScene, GpuPipelineState, workloads
    torch.cuda.set_device(0)
    n = args.gaussians or 6_000_000
    wl = workloads.large_multicage(n=n)
    stream = torch.cuda.Stream(device=0)
    st = GpuPipelineState(0, stream=stream.cuda_stream)
    st.upload_scene(wl.scene)
    cs = CageScene.auto_bind(wl.cages, st, n)
    st.upload_cages(cs)
    st.mvc_cage_upload(wl.poly.cage)
    pts = torch.from_numpy(wl.poly.training_points(args.train_points)).to("cuda:0")
    w = st.mvc_weights(pts)
    st.mvc_field_create(seed=1)
    loss = st.mvc_field_train(pts, w, steps=args.train_steps, batch=4096, lr=2e-3, lam=0.05,
                              seed=5)
    del w, pts
    torch.cuda.empty_cache()
    _, _, enc = st.mvc_field_layout()
    s_half = 1.0 / float(enc[3])
    rng = np.random.default_rng(7)
    sample = wl.scene.positions[rng.choice(n, min(n, 200_000), replace=False)]
    raw, _ = st.mvc_field_infer(sample, rest=True)
    thr = float(np.quantile(np.linalg.norm(raw - sample, axis=1) / s_half, args.fallback_quantile))
    nb, nfb = st.mvc_bind_learned(thr)
    tet_bound = int((cs.bind_cage != 0xFFFFFFFF).sum())
    frame = 0

    def render(profile=False, timings=True):
        nonlocal frame
        cs.step(1.0 / 60.0)
        st.mvc_vertices_update(wl.poly.vertices(frame))
        cam = wl.camera(frame)
        frame += 1
        return st.execute_frame_gpu(wl.scene, cs, cam, wl.compositor(cam), profile_stages=profile,
                                    stage_timings=timings)

    for _ in range(max(args.warmup, 3)):
        render()
    rows = [render(profile=True) for _ in range(2)]
    st.synchronize()
    st.kernel_profile_reset()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clock = ClockSampler(0)
    torch.cuda.synchronize()
    with clock:
        a.record(stream)
        for _ in range(args.steps):
            render(profile=True, timings=False)
        b.record(stream)
        st.synchronize()
        torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    kp = st.kernel_profile()
    hbm, _ = peaks()
    kernels = {k: {"ms_per_frame": d["ms"] / args.steps,
                   "hbm_frac": (d["alg_bytes"] / (d["ms"] / 1000.0) / 1e9 / hbm) if d["ms"] else 0.0}
               for k, d in kp.items() if d["launches"] and k != "clear"}
    dev = ctypes_device_bytes(st)
    last = rows[-1]
    line = {
        "metric": "frames/s of the large quantized multi-cage scene at 7680x4320",
        "value": 1000.0 / ms, "unit": "frames/s", "higher_is_better": True, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "dtype": "f32 (f16 storage)",
        "data": "synthetic",
        "config": {"workload": "quantized scene, 4 tet cages + learned polygon cage, 8K",
                   "gaussians": n, "width": wl.width, "height": wl.height, "orbit_radius": wl.radius,
                   "keys": "64-bit (tile, depth)" if last.used_64bit_keys else "32-bit"},
        "stages_ms": {k: getattr(last, k) for k in ("stage1_deform_ms", "stage2_project_ms",
                                                    "stage3_bin_sort_ms", "stage4_composite_ms")},
        "frame_counts": {"active_gaussians": last.active_gaussians,
                         "surviving_gaussians": last.surviving_gaussians,
                         "tile_entries": last.total_tile_entries},
        "kernels": kernels,
        "bindings": {"tet": tet_bound, "polygon_cage": nb, "polygon_fallbacks": nfb,
                     "field_loss_terms": loss},
        "device_bytes": dev,
        "clocks": clock.summary(),
    }
    print(json.dumps(line), flush=True)
    st.close()
    return 0


def ctypes_device_bytes(st) -> int:
    import ctypes
    v = ctypes.c_uint64(0)
    st._check(st._lib.cgs_ctx_device_bytes(st.handle, ctypes.byref(v)), "cgs_ctx_device_bytes")
    return int(v.value)


def main():
    args = parse()
    if args.workload == "large":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference CPU path at 8K with 6M Gaussians takes hours; "
                              "timed by the default workload's reference arm"}))
            return 0
        return run_large(args)
    if args.workload == "views":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference renders one view per call on its CPU path; "
                              "timed by the default workload's reference arm"}))
            return 0
        return run_views(args)
    if args.workload == "mvc":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference's MVC deformation is its CPU path; "
                              "exact GPU MVC is this leg's judge"}))
            return 0
        return run_mvc(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
