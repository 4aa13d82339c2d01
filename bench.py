"""Benchmark of the wavefront + persistent render path (Mrays/s).

Workload: the "displaced_icospheres" scene (3 level-8 displaced icospheres =
3,932,160 triangles + ground, medium box, area light, 2048x1024 procedural sky),
1920x1080, max depth 8, counter-based RNG. One step = one frame of the
workload's 16 samples per pixel (--spp-per-step), rendered by one C-ABI call
that traces several samples per wave (the library's automatic wave size);
K steps = 16 K spp (default K = 16, about a second of timed work).
Mrays/s = (extend rays + shadow rays) / device time, rays counted on the device.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference runs the UNMODIFIED reference (oracle/_ref/libmcref.so: the
reference's src/path_tracer.cu compiled for sm_100a) through its own
renderWithWavefront with --persistent semantics on the same scene.
Multi-GPU (torchrun): every rank renders its own K frames of the full image
(weak scaling) and the accumulation buffers are summed with one NCCL
all-reduce at the end, inside the timed region.
"""
import argparse
import copy
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "monocuda-pt_b200")]

WORKLOAD = {"workload": "displaced_icospheres", "triangles": 3932176, "width": 1920, "height": 1080, "max_depth": 8,
            "env_map": "2048x1024 procedural sky", "medium": "homogeneous box, sigma_t 0.5",
            "rng": "philox4x32-10 per (pixel, sample)", "l2": "inputs larger than L2 (BVH 252 MB + triangles 189 MB)"}
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "k_trace_displaced_icospheres.txt")
# algorithmic bytes per unit of the trace kernel: node visit (64 B binary / 128 B wide, scaled below),
# primitive test (48 B hot record), extend-ray I/O (ray in, hit out), shadow-ray I/O (entry, time, sample update)
NODE_BYTES, LEAF_BYTES, EXT_IO_BYTES, SHADOW_IO_BYTES = 64, 48, 48, 72
INGEST_BYTES = 224 + 36 + 192  # per triangle: AoS record read, hot and cold records written


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--spp-per-step", type=int, default=16, help="samples per pixel of one step (one frame)")
    ap.add_argument("--samples-per-wave", type=int, default=0,
                    help="samples traced together per wave (0 = the library's automatic choice, 1 = one per wave)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = the named workload)")
    ap.add_argument("--layout", default="wide4", choices=["binary", "wide4", "wide4q"], help="BVH node layout traversed")
    ap.add_argument("--builder", default="clustered", choices=["clustered", "lbvh"],
                    help="binary tree the wide layouts collapse: clustered (PLOC) or the reference's LBVH")
    ap.add_argument("--refill", type=int, default=0,
                    help="trace refill threshold; 0 = the library autotuner's choice (a fixed value keeps profiles "
                         "free of the autotuner's probe launches)")
    ap.add_argument("--resolution", default="",
                    help="WxH instead of the workload's 1920x1080 (same view, e.g. 480x270 for small ncu captures)")
    ap.add_argument("--trace-threads", type=int, default=0,
                    help="trace block size 128 or 256 (0 = the autotuner's choice, or 256 with a fixed --refill)")
    ap.add_argument("--stack-entries", type=int, default=0,
                    help="traversal stack entries per lane (0 = the autotuner's choice, or 64 with a fixed --refill; "
                         "-1 = what the 4-wide tree can need, 3 per level)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch and guiding summaries that the default 1-GPU line carries")
    ap.add_argument("--no-1m", action="store_true",
                    help="skip the second, ~1M-triangle line (level-7 icospheres, 983,056 triangles)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--profile", action="store_true",
                    help="warm-up and timed steps only (for ncu captures); prints the timed line without extras")
    ap.add_argument("--workload", default="icospheres",
                    choices=["icospheres", "batch", "guiding", "guided_waves", "mlp", "server"],
                    help="icospheres: the headline single-scene workload; batch: the 64-scene batched pipeline; "
                         "guiding: guided vs plain time to a fixed RMSE on the aperture room")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--guide-ref-spp", type=int, default=1024)
    ap.add_argument("--guide-plain-spp", type=int, default=64)
    ap.add_argument("--guide-chunk", type=int, default=8)
    ap.add_argument("--guide-lr", type=float, default=1e-3)
    ap.add_argument("--guide-steps", type=int, default=4, help="Adam steps per sample, each on 65536 records")
    ap.add_argument("--guide-vertices", type=int, default=0,
                    help="diffuse vertices per path that train the guide (0 = the library default, 3)")
    ap.add_argument("--guide-pretrain-spp", type=int, default=0,
                    help="diagnostic: train the guide on this many untimed samples first (the headline trains from "
                         "scratch inside the timed region)")
    ap.add_argument("--guide-batch", type=int, default=0, help="records per Adam step (0 = the library's 65536)")
    ap.add_argument("--guide-nee", type=int, default=0, choices=[0, 1],
                    help="guiding: the primary vertices' shadow rays also give training records")
    ap.add_argument("--guide-anchor", type=int, default=-1, choices=[-1, 0, 1],
                    help="guiding: lobe means offset by the direction input, so an untrained guide proposes around "
                         "the normal (1), raw means (0), or the library default, anchored (-1)")
    ap.add_argument("--guide-fold", action="store_true",
                    help="mirror guide directions below the surface up instead of ending those paths")
    ap.add_argument("--guide-weight-cap", type=float, default=0.0,
                    help="training: cap of a record's share of a step's weight, in units of 1 / records (0 = none)")
    ap.add_argument("--guide-depth", type=int, default=0,
                    help="bounces that sample the guide (0 = the library default, 4; deeper vertices sample the cosine "
                         "lobe alone)")
    ap.add_argument("--guide-dir", default="normal", choices=["normal", "ray"],
                    help="direction input of the guide: the face normal or the arriving ray's direction")
    ap.add_argument("--mlp-items", type=int, default=1 << 20)
    ap.add_argument("--server-rates", type=float, nargs="+", default=[1, 2, 4, 8, 16, 32, 64],
                    help="arrival rates (requests/s)")
    ap.add_argument("--server-repeats", type=int, default=3,
                    help="runs of each rate's trace (the schedule depends on host timing); medians and ranges reported")
    ap.add_argument("--server-requests", type=int, default=64,
                    help="requests per arrival rate (at most; max(24, 16 x rate) at low rates)")
    ap.add_argument("--server-sps", type=int, default=16, help="samples per server step")
    ap.add_argument("--server-wave-paths", type=int, default=0, help="paths per server wave (0 = 4M)")
    ap.add_argument("--server-scene-waves", action="store_true",
                    help="each step renders each scene's plain requests in a wave of their own")
    return ap.parse_args()


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if index < len(ids):
                index = ids[index]
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
            except (ValueError, IndexError):
                continue
        busy = [x for x in sm if mx and x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks(key="hbm_gbs"):
    """A measured peak from MEASURED_PEAKS.json (HBM GB/s or bf16 TFLOP/s), else the fallback."""
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p[key]), "measured"
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}.get(key, 0.0), "fallback"


def traffic_per_launch():
    """dram bytes (read + write) per trace launch from the committed ncu summary, or None."""
    try:
        with open(TRAFFIC_FILE) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def cpu_baseline(scene, args):
    """The oracle (CPU restatement of the same integrator) on a bounded band of
    rows of the same workload, all host threads, timed on this host."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import mcpt
    from helpers import oracle
    orc = oracle()
    tris = mcpt.host_triangles(scene)
    env = mcpt.host_env(scene)
    h = orc.orc_scene_create(C.addressof(tris), len(tris), None, 0, env.ctypes.data, scene.env_width,
                             scene.env_height, scene.env_intensity, 0.0)
    W, H = scene.width, scene.height
    threads = os.cpu_count() or 1
    acc = np.zeros(W * H * 3, np.float64)
    stats = np.zeros(2, np.float64)
    cam = scene.camera
    y0 = H // 2 - 4
    rows = 8
    t0 = time.perf_counter()
    orc.orc_render(h, C.addressof(cam), W, H, 1, 0, 8, 1234, 0, 0, 0, y0, W, y0 + rows, threads, acc.ctypes.data,
                   stats.ctypes.data)
    dt = time.perf_counter() - t0
    # size the sample to about --cpu-seconds: more rows first, then more samples per pixel
    per_row = max(dt, 1e-4) / rows
    rows = max(8, min(H, int(args.cpu_seconds / per_row)))
    spp = max(1, int(round(args.cpu_seconds / (per_row * rows)))) if rows == H else 1
    y0 = max(0, H // 2 - rows // 2)
    for attempt in range(2):
        acc[:] = 0
        t0 = time.perf_counter()
        orc.orc_render(h, C.addressof(cam), W, H, spp, 0, 8, 1234, 0, 0, 0, y0, W, y0 + rows, threads, acc.ctypes.data,
                       stats.ctypes.data)
        dt = time.perf_counter() - t0
        # the middle rows cost more than the average row: when the whole image
        # ran well short of the budget, rescale the samples once
        if rows < H or dt >= 0.5 * args.cpu_seconds:
            break
        spp = max(spp + 1, int(round(spp * args.cpu_seconds / max(dt, 1e-3))))
    orc.orc_scene_destroy(h)
    rays = stats[0] + stats[1]
    return {"value": round(rays / dt / 1e6, 4), "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": "%d rows x %d px x %d spp of the same workload (FP32 oracle, %d threads, %.1f s, %d rays)"
                      % (rows, W, spp, threads, dt, int(rays))}


def level_variant(ctx, level, steps, warmup, spp_per_step):
    """Mrays/s of the same workload with level-L icospheres (L = 7: 3 x 327,680
    triangles, the ~1M-triangle reading of the scene), device-timed like the
    headline: scene resident, autotuned refill, K frames of spp_per_step."""
    import torch

    import mcpt
    scene = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=level, seed=2)
    tris = mcpt.host_triangles(scene)
    ds = mcpt.DeviceScene(tris, env_rgba=mcpt.host_env(scene), env_intensity=scene.env_intensity)
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4, builder=mcpt.BUILDER_CLUSTERED)
    W, H = scene.width, scene.height
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    tuned = mcpt.render_params(scene.camera, W, H, spp_per_step, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234)
    mcpt.check(ctx.lib.mc_autotune(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(tuned), 4000))
    st = mcpt.RenderStats()

    def step(i):
        p = mcpt.render_params(scene.camera, W, H, spp_per_step, 8, persistent=bool(tuned.persistent),
                               rng=mcpt.RNG_PHILOX, seed=1234, first_sample=i * spp_per_step,
                               refill_threshold=tuned.refill_threshold, samples_per_wave=tuned.samples_per_wave,
                               trace_threads=tuned.trace_threads, stack_entries=tuned.stack_entries)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        return st.extend_rays + st.shadow_rays
    for i in range(warmup):
        step(1000 + i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rays = sum(step(i) for i in range(steps))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"workload": "displaced_icospheres level %d" % level, "triangles": int(len(tris)), "steps": steps,
           "spp_per_step": spp_per_step, "value": round(rays / (ms / 1e3) / 1e6, 2), "unit": "Mrays/s",
           "ms_per_step": round(ms / steps, 3),
           "autotuned": {"refill_threshold": int(tuned.refill_threshold), "trace_threads": int(tuned.trace_threads) or 256,
                         "stack_entries": int(tuned.stack_entries) or 64,
                         "samples_per_wave": int(tuned.samples_per_wave) or "automatic"}}
    bvh.close()
    ds.close()
    mcpt.free_scene(scene)
    return out


def run_ours(args):
    import torch

    import mcpt
    import sharding
    world, rank, local = dist_init(args)
    dev = "cuda:%d" % local
    torch.cuda.set_device(local)
    scene = mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=args.level, seed=2)
    tris = mcpt.host_triangles(scene)
    env = mcpt.host_env(scene)
    if args.resolution:
        rw, rh = (int(x) for x in args.resolution.lower().split("x"))
        cam = mcpt.Camera.from_buffer_copy(bytes(scene.camera))
        cam.image_width = rw
        cam.aspect_ratio = rw / float(rh)
        scene.camera = mcpt.camera_initialize(cam)
        scene.width, scene.height = rw, rh
    ctx = mcpt.Context(local)
    ds = mcpt.DeviceScene(tris, env_rgba=env, env_intensity=scene.env_intensity, device=dev)
    layout = {"binary": mcpt.LAYOUT_BINARY, "wide4": mcpt.LAYOUT_WIDE4, "wide4q": mcpt.LAYOUT_WIDE4Q}[args.layout]
    builder = {"clustered": mcpt.BUILDER_CLUSTERED, "lbvh": mcpt.BUILDER_LBVH}[args.builder]
    bvh = mcpt.Bvh(ctx, ds.view, layout=layout, builder=builder)
    W, H = scene.width, scene.height
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device=dev)
    K, Wm, S = args.steps, args.warmup, args.spp_per_step
    # step indices; step s renders samples [s * S, (s + 1) * S)
    timed_samples, warm_samples = sharding.sample_ranges(rank, world, K, Wm)

    # the library's autotuner picks the trace variant and refill threshold by
    # timing the wave that each step traces (untimed; the choice does not change the image)
    tuned = mcpt.render_params(scene.camera, W, H, S, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=1234,
                               refill_threshold=args.refill, samples_per_wave=args.samples_per_wave)
    if args.refill <= 0:
        mcpt.check(ctx.lib.mc_autotune(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(tuned), 4000))
    if args.trace_threads:
        tuned.trace_threads = args.trace_threads
    if args.stack_entries > 0:
        tuned.stack_entries = args.stack_entries
    elif args.stack_entries < 0:
        # what the 4-wide tree can need: 3 entries per level, rounded up to 8
        lv = bvh.info().wide_levels
        tuned.stack_entries = min(64, ((3 * lv + 7) // 8) * 8) if lv > 0 else 0

    def params(step, instrument=0):
        return mcpt.render_params(scene.camera, W, H, S, 8, persistent=bool(tuned.persistent), rng=mcpt.RNG_PHILOX,
                                  seed=1234, first_sample=step * S, instrument=instrument,
                                  refill_threshold=tuned.refill_threshold,
                                  samples_per_wave=args.samples_per_wave or tuned.samples_per_wave,
                                  trace_threads=tuned.trace_threads, stack_entries=tuned.stack_entries)

    st = mcpt.RenderStats()
    for s in warm_samples:
        p = params(s)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
    acc.zero_()
    clocks = Clocks(local) if rank == 0 else None
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    rays = ext = shd = 0
    trace_ms = 0.0
    trace_launches = launches = 0
    for s in timed_samples:
        p = params(s, instrument=2)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        ext += st.extend_rays
        shd += st.shadow_rays
        trace_ms += st.trace_ms
        trace_launches += st.trace_launches
        launches += st.kernel_launches
    sharding.reduce_accumulation(acc, world)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    ck = clocks.stop() if clocks else None
    rays = ext + shd
    if world > 1:
        t = torch.tensor([ms, float(rays)], dtype=torch.float64, device=dev)
        mx = t.clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        ms_max, rays_all = float(mx[0]), float(t[1])
    else:
        ms_max, rays_all = ms, float(rays)
    if args.profile:
        if rank == 0:
            print(json.dumps({"metric": "Mrays/s", "value": round(rays_all / (ms_max / 1e3) / 1e6, 2), "unit": "Mrays/s",
                              "steps": K, "profile": True, "level": args.level}), flush=True)
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    # untimed instrumented pass over the same samples: node visits and primitive tests
    visits = leaves = 0
    for s in timed_samples:
        p = params(s, instrument=1)
        tmp = torch.zeros_like(acc)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), tmp.data_ptr(),
                                               C.byref(st)))
        visits += st.node_visits
        leaves += st.leaf_tests

    # end to end through the C ABI with host buffers: each step renders one sample
    # and reads the accumulation buffer back into pinned host memory
    host_acc = torch.empty(W * H * 3, dtype=torch.float32, pin_memory=True)
    e2e_steps = K
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    e2e_rays = 0
    for s in timed_samples[:e2e_steps]:
        p = params(s)
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                               C.byref(st)))
        e2e_rays += st.extend_rays + st.shadow_rays
        host_acc.copy_(acc, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)

    # cold end to end: host triangles in, accumulation buffer out, one C-ABI call
    host_cold = torch.zeros(W * H * 3, dtype=torch.float32, pin_memory=True)
    pc = params(timed_samples.start)
    cold_stats = mcpt.RenderStats()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mcpt.check(ctx.lib.mc_render_host(ctx.handle, C.addressof(tris), len(tris), None, 0, C.byref(ds.env), C.byref(pc),
                                      host_cold.data_ptr(), C.byref(cold_stats)))
    cold_s = time.perf_counter() - t0
    # the same call again: the context's pinned staging and wave state exist now
    t0 = time.perf_counter()
    mcpt.check(ctx.lib.mc_render_host(ctx.handle, C.addressof(tris), len(tris), None, 0, C.byref(ds.env), C.byref(pc),
                                      host_cold.data_ptr(), None))
    cold2_s = time.perf_counter() - t0

    # the cold call's stages one by one, from the same pageable host array:
    # mc_scene_ingest_host (upload through the context's pinned staging, which
    # the cold call above allocated, then device ingestion; host clock), the
    # device ingestion alone from a device copy of the array (CUDA events,
    # including the light-count read-back), BVH build
    stages = {}
    i_hot = torch.empty(len(tris) * 36, dtype=torch.uint8, device=dev)
    i_cold = torch.empty(len(tris) * 192, dtype=torch.uint8, device=dev)
    i_lights = torch.empty(len(tris) * 64, dtype=torch.uint8, device=dev)
    i_nl, i_med = C.c_int32(), C.c_int32()
    for rep in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mcpt.check(ctx.lib.mc_scene_ingest_host(ctx.handle, C.addressof(tris), len(tris), None, 0, i_hot.data_ptr(),
                                                i_cold.data_ptr(), i_lights.data_ptr(), C.byref(i_nl), C.byref(i_med)))
        stages["ingest_host_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    aos = torch.frombuffer(tris, dtype=torch.uint8, count=len(tris) * 224).to(dev)
    for rep in range(3):
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        mcpt.check(ctx.lib.mc_scene_ingest(ctx.handle, aos.data_ptr(), len(tris), None, 0, i_hot.data_ptr(),
                                           i_cold.data_ptr(), i_lights.data_ptr(), C.byref(i_nl), C.byref(i_med)))
        g1.record()
        torch.cuda.synchronize()
    stages["ingest_device_ms"] = round(g0.elapsed_time(g1), 3)
    stages["ingest_device_GBps"] = round(len(tris) * INGEST_BYTES / (g0.elapsed_time(g1) / 1e3) / 1e9, 1)
    del aos, i_hot, i_cold, i_lights
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b2 = mcpt.Bvh(ctx, ds.view, layout=layout)
    torch.cuda.synchronize()
    stages["bvh_build_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    b2.close()

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    peak, peak_kind = peaks()
    node_bytes = 2 * NODE_BYTES if layout == mcpt.LAYOUT_WIDE4 else NODE_BYTES  # 128-byte wide, 64-byte binary / quantised
    alg_bytes = visits * node_bytes + leaves * LEAF_BYTES + ext * EXT_IO_BYTES + shd * SHADOW_IO_BYTES
    per_launch_bytes = alg_bytes / max(trace_launches, 1)
    per_launch_s = trace_ms / max(trace_launches, 1) / 1e3
    achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    traffic = traffic_per_launch()
    # DRAM fraction of the same launches: the captured DRAM bytes per launch
    # over this run's mean launch duration
    dram_gbs = traffic / per_launch_s / 1e9 if (traffic and per_launch_s > 0) else None
    value = rays_all / (ms_max / 1e3) / 1e6
    out = {
        "metric": "Mrays/s", "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": round(ms_max / K, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": dict(WORKLOAD, spp=K * S * world, spp_per_step=S, bvh_layout=args.layout, bvh_builder=args.builder,
                       bvh_wide_levels=int(bvh.info().wide_levels),
                       autotuned={"persistent": int(tuned.persistent), "refill_threshold": int(tuned.refill_threshold),
                                  "samples_per_wave": int(tuned.samples_per_wave) or "automatic",
                                  "trace_threads": int(tuned.trace_threads) or 256,
                                  "stack_entries": int(tuned.stack_entries) or 64, "graph": int(tuned.use_graph)},
                       parallelism="replicas x%d + final all-reduce" % world if world > 1 else "1 GPU",
                       samples_per_wave=args.samples_per_wave or "automatic",
                       samples_per_sec=round(W * H * K * S * world / (ms_max / 1e3), 1),
                       rays_per_path=round(rays_all / (W * H * K * S * world), 3)),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "kernel": "k_trace (persistent extend + shadow)",
                     "dram_gbs": round(dram_gbs, 1) if dram_gbs else None,
                     "dram_frac": round(dram_gbs / peak, 4) if dram_gbs else None,
                     "launches": trace_launches, "avg_launch_ms": round(trace_ms / max(trace_launches, 1), 4),
                     "trace_share": round(trace_ms / ms, 4),
                     "node_visits_per_ray": round(visits / max(rays, 1), 2),
                     "leaf_tests_per_ray": round(leaves / max(rays, 1), 2),
                     "algorithmic_bytes_per_launch": int(per_launch_bytes)},
        "e2e": {"value": round(e2e_rays / (e2e_ms / 1e3) / 1e6, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": C.sizeof(mcpt.RenderParams), "d2h_bytes_per_step": W * H * 12,
                "note": "scene and BVH resident; per step: render call with host params + accumulation read-back"},
        "e2e_cold": {"value": round((cold_stats.extend_rays + cold_stats.shadow_rays) / cold_s / 1e6, 2), "unit": "Mrays/s",
                     "seconds": round(cold_s, 3), "seconds_second_call": round(cold2_s, 3),
                     "h2d_bytes": len(tris) * 224, "d2h_bytes": W * H * 12,
                     "stages": stages,
                     "note": "mc_render_host: host triangles -> upload, device ingestion (bounds, lights, split), "
                             "BVH build, %d spp, read-back" % S},
        "gpu_launches": launches,
        "clocks": ck,
    }
    if not args.no_1m and args.level == 8 and world == 1:
        out["workload_1m"] = level_variant(ctx, 7, K, Wm, S)
    if not args.no_extras and args.level == 8 and world == 1 and not args.resolution:
        # the other workloads of the scope table, summarised in the same line:
        # the 64-scene batch against sequential renders, guided vs plain time
        # to plain's 64-spp RMSE on the aperture room (with the guide MLP's
        # kernel throughput)
        b = run_batch(args, emit=False)
        out["batch"] = {k: b[k] for k in ("value", "unit", "triangles", "build_ms", "render_ms", "sequential_mrays",
                                          "speedup_vs_sequential")}
        g = run_guiding(args, emit=False)
        out["guiding"] = {k: g[k] for k in ("metric", "value", "unit", "target_rmse", "plain_ms", "guided_ms_to_target",
                                            "guided_spp", "phase_split_ms")}
        out["guiding"]["mlp"] = {k: g["mlp"][k] for k in ("infer_queries_per_s", "infer_tflops", "infer_frac",
                                                          "train_records_per_s", "train_tflops", "train_frac",
                                                          "peak_tflops")}
        # the same measurement with a guide that has already trained on 1024
        # untimed samples of the view (what a resident scene's guide reaches
        # in the server): anchored lobes, guiding and training at the first
        # diffuse vertex only
        ta = copy.copy(args)
        ta.guide_anchor, ta.guide_depth, ta.guide_vertices, ta.guide_pretrain_spp = 1, 2, 1, 1024
        t = run_guiding(ta, emit=False, mlp=False)
        out["guiding_trained"] = {k: t[k] for k in ("value", "unit", "target_rmse", "plain_ms", "guided_ms_to_target",
                                                    "guided_spp", "pretrain_spp", "anchor_lobes", "guided_depth",
                                                    "train_vertices", "phase_split_ms")}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(scene, args)
    print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_batch(args, emit=True):
    """64 seeded scenes (log-normal triangle counts, median 50k, clipped to
    [1k, 2M]; resolutions from {256^2, 512^2, 1024^2}; spp from {4, 16, 64}):
    one batched BVH build and one batched, graph-replayed render, against
    the same scenes built and rendered one after another."""
    import torch

    import mcpt
    ctx = mcpt.Context(0)
    n = args.batch_scenes
    t0 = time.perf_counter()
    scenes = [mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=i, seed=3) for i in range(n)]
    gen_s = time.perf_counter() - t0
    devs = [mcpt.DeviceScene(mcpt.host_triangles(s)) for s in scenes]
    tris = sum(s.triangle_count for s in scenes)
    accs = [torch.zeros(s.width * s.height * 3, dtype=torch.float32, device="cuda") for s in scenes]

    def items():
        return [mcpt.BatchItem(d.view, mcpt.render_params(s.camera, s.width, s.height, s.spp, 8, persistent=True,
                                                           rng=mcpt.RNG_PHILOX, seed=3), a.data_ptr())
                for s, d, a in zip(scenes, devs, accs)]
    # warm-up
    b = mcpt.BatchBvh(ctx, [d.view for d in devs], layout=mcpt.LAYOUT_WIDE4)
    b.render(items(), use_graph=True)
    b.close()
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    b = mcpt.BatchBvh(ctx, [d.view for d in devs], layout=mcpt.LAYOUT_WIDE4)
    e1.record()
    st = b.render(items(), use_graph=True)
    e2.record()
    torch.cuda.synchronize()
    build_ms, render_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    rays = st.extend_rays + st.shadow_rays
    # the same scenes one request at a time (plain per-request wavefront),
    # after one untimed build and render that loads the single-scene kernels
    def single_render(s, d, a):
        single = mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4)
        p = mcpt.render_params(s.camera, s.width, s.height, s.spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=3)
        rs = mcpt.RenderStats()
        mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, single.handle, C.byref(d.view), C.byref(p), a.data_ptr(),
                                               C.byref(rs)))
        single.close()
        return rs.extend_rays + rs.shadow_rays
    single_render(scenes[0], devs[0], accs[0])
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    seq_rays = 0
    for s, d, a in zip(scenes, devs, accs):
        seq_rays += single_render(s, d, a)
    f1.record()
    torch.cuda.synchronize()
    seq_ms = f0.elapsed_time(f1)
    out = {"metric": "Mrays/s", "value": round(rays / ((build_ms + render_ms) / 1e3) / 1e6, 2), "unit": "Mrays/s",
           "n_gpus": 1, "workload": "batch_%d_scenes" % n, "triangles": tris,
           "paths": int(st.paths), "rays": int(rays), "build_ms": round(build_ms, 2), "render_ms": round(render_ms, 2),
           "render_only_mrays": round(rays / (render_ms / 1e3) / 1e6, 2),
           "sequential_ms": round(seq_ms, 2), "sequential_mrays": round(seq_rays / (seq_ms / 1e3) / 1e6, 2),
           "speedup_vs_sequential": round(seq_ms / (build_ms + render_ms), 3), "generation_s": round(gen_s, 1),
           "graph": True, "layout": "wide4"}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def mlp_throughput(ctx, guide, n=1 << 20):
    """Guide MLP kernels on n queries (inference) and n records (forward +
    backward + weight gradients), useful tensor-core FLOPs per item (padding
    excluded) over CUDA-event time."""
    import torch

    import mcpt
    q = torch.rand(n, 6, device="cuda")
    mix = torch.empty(n * 40, device="cuda")
    recs = torch.rand(n, 10, device="cuda")
    grad = torch.empty(mcpt.GUIDE_PARAM_COUNT, device="cuda")

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    infer_ms = timed(lambda: mcpt.check(ctx.lib.mc_guide_infer(guide.handle, q.data_ptr(), n, mix.data_ptr())))
    loss = C.c_double()
    train_ms = timed(lambda: mcpt.check(ctx.lib.mc_guide_gradient(guide.handle, recs.data_ptr(), n, grad.data_ptr(),
                                                                   C.byref(loss))))
    # useful FLOPs (padding excluded): forward, backward data, backward weights
    fwd_flop = 2 * (144 * 64 + 64 * 64 + 64 * 64 + 64 * 40)
    bwd_flop = 2 * (40 * 64 + 64 * 64 + 64 * 64) + 2 * (40 * 64 + 64 * 64 + 64 * 64 + 64 * 144)
    peak, peak_kind = peaks("bf16_tflops")
    infer_tf = n * fwd_flop / (infer_ms / 1e3) / 1e12
    train_tf = n * (fwd_flop + bwd_flop) / (train_ms / 1e3) / 1e12
    return {"items": n, "infer_ms": round(infer_ms, 3), "infer_queries_per_s": round(n / (infer_ms / 1e3)),
            "infer_tflops": round(infer_tf, 2), "train_ms": round(train_ms, 3),
            "train_records_per_s": round(n / (train_ms / 1e3)), "train_tflops": round(train_tf, 2),
            "peak_tflops": peak, "peak_kind": peak_kind, "infer_frac": round(infer_tf / peak, 4) if peak else None,
            "train_frac": round(train_tf / peak, 4) if peak else None, "flop_per_query": fwd_flop,
            "flop_per_record": fwd_flop + bwd_flop}


def run_mlp(args):
    """The guide MLP kernels alone (a small, self-contained case for profiling)."""
    import mcpt
    ctx = mcpt.Context(0)
    guide = mcpt.Guide(ctx, [-1.0, -1.0, -1.0], [1.0, 1.0, 1.0], seed=1)
    out = mlp_throughput(ctx, guide, n=args.mlp_items)
    out["metric"] = "guide MLP throughput"
    print(json.dumps(out), flush=True)
    guide.close()


def run_guiding(args, emit=True, mlp=True):
    """Time to a fixed RMSE, guided vs plain wavefront, on the aperture room
    (about 200k triangles, 1024x1024, light only through a 0.2 x 0.2 hole).
    The target RMSE is plain wavefront's at --guide-plain-spp; the guided
    renderer starts from an untrained guide (or, with --guide-pretrain-spp, one
    trained on that many untimed samples of the view), trains online
    (--guide-steps Adam steps per sample) and counts every sample and every
    training step in its time. The
    reference image is a plain render at --guide-ref-spp (its own noise adds
    the same amount to both MSEs). Firefly clamp off in all three (the clamp
    biases the estimators differently). Times are CUDA events around the
    render calls; the RMSE evaluation between chunks is not timed."""
    import numpy as np
    import torch

    import mcpt
    ctx = mcpt.Context(0)
    s = mcpt.generate_scene(mcpt.SCENE_GUIDING_ROOM)
    tris = mcpt.host_triangles(s)
    ds = mcpt.DeviceScene(tris)
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
    W, H = s.width, s.height
    raw = np.frombuffer(tris, dtype=np.uint8).reshape(len(tris), 224)
    verts = raw[:, :36].copy().view(np.float32).reshape(-1, 3)
    lo, hi = verts.min(0), verts.max(0)
    chunk = args.guide_chunk

    def params(spp, first):
        return mcpt.render_params(s.camera, W, H, spp, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX, seed=4,
                                  first_sample=first, disable_clamp=True)

    def render(acc, spp, first, guide=None, train=0):
        st = mcpt.RenderStats()
        p = params(spp, first)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if guide is None:
            mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), acc.data_ptr(),
                                                   C.byref(st)))
        else:
            mcpt.check(ctx.lib.mc_render_guided(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), guide.handle,
                                                train, acc.data_ptr(), C.byref(st)))
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), st

    # warm-up of both paths (kernels loaded, wave buffers reserved for a chunk),
    # the guided one with the timed guide's configuration
    tmp = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    render(tmp, chunk, 999999)
    gdir = mcpt.GUIDE_DIR_NORMAL if args.guide_dir == "normal" else mcpt.GUIDE_DIR_RAY
    warm_guide = mcpt.Guide(ctx, lo.tolist(), hi.tolist(), seed=1, learning_rate=args.guide_lr,
                            train_steps=args.guide_steps, train_vertices=args.guide_vertices, direction_input=gdir,
                            guided_depth=args.guide_depth, weight_cap=args.guide_weight_cap,
                            fold_below=args.guide_fold, anchor_lobes=None if args.guide_anchor < 0 else bool(args.guide_anchor),
                            batch_capacity=args.guide_batch,
                            nee_records=bool(args.guide_nee))
    render(tmp, chunk, 999998, warm_guide, 1)
    render(tmp, chunk, 999990, warm_guide, 1)
    warm_guide.close()
    # reference image
    ref = torch.zeros_like(tmp)
    ref_ms = 0.0
    for c in range(0, args.guide_ref_spp, 64):
        ms, _ = render(ref, min(64, args.guide_ref_spp - c), 10_000_000 + c)
        ref_ms += ms
    ref /= args.guide_ref_spp

    def rmse(acc, spp):
        return float(torch.sqrt(torch.mean((acc / spp - ref) ** 2)))

    # plain: the target
    acc = torch.zeros_like(tmp)
    plain_ms, plain_curve, rays_plain = 0.0, [], 0
    for c in range(0, args.guide_plain_spp, chunk):
        ms, st = render(acc, chunk, 20_000_000 + c)
        plain_ms += ms
        rays_plain += st.extend_rays + st.shadow_rays
        plain_curve.append((c + chunk, round(plain_ms, 1), rmse(acc, c + chunk)))
    target = plain_curve[-1][2]
    # guided, trained online from scratch
    guide = mcpt.Guide(ctx, lo.tolist(), hi.tolist(), seed=7, learning_rate=args.guide_lr,
                       train_steps=args.guide_steps, train_vertices=args.guide_vertices, direction_input=gdir,
                       guided_depth=args.guide_depth, weight_cap=args.guide_weight_cap,
                       fold_below=args.guide_fold, anchor_lobes=None if args.guide_anchor < 0 else bool(args.guide_anchor),
                            batch_capacity=args.guide_batch,
                            nee_records=bool(args.guide_nee))
    # an untimed render without training sizes the new guide's buffers; its
    # weights stay as initialised
    render(tmp, chunk, 999997, guide, 0)
    for c in range(0, args.guide_pretrain_spp, chunk):
        render(tmp, chunk, 50_000_000 + c, guide, 1)
    acc = torch.zeros_like(tmp)
    g_ms, g_curve, reached, rays_g = 0.0, [], None, 0
    spp = 0
    while spp < args.guide_plain_spp * 4:
        ms, st = render(acc, chunk, 30_000_000 + spp, guide, 1)
        prev_ms, prev_err = g_ms, (g_curve[-1][2] if g_curve else None)
        g_ms += ms
        spp += chunk
        rays_g += st.extend_rays + st.shadow_rays
        err = rmse(acc, spp)
        g_curve.append((spp, round(g_ms, 1), err))
        if err <= target:
            # interpolate the crossing inside the last chunk (error ~ 1/sqrt(time))
            if prev_err is not None and prev_err > target:
                f = (1 / prev_err ** 2 - 1 / target ** 2) / (1 / prev_err ** 2 - 1 / err ** 2)
                reached = prev_ms + f * (g_ms - prev_ms)
            else:
                reached = g_ms
            break
    steps = guide.steps()
    # where a guided wave's time goes: one more chunk with every launch timed
    # by phase (instrument bit 1; untimed above), and the same for plain
    split = {}
    for name, g in (("guided", guide), ("plain", None)):
        st = mcpt.RenderStats()
        p = params(chunk, 40_000_000)
        p.instrument = 2
        tmp.zero_()
        torch.cuda.synchronize()
        if g is None:
            mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), tmp.data_ptr(),
                                                   C.byref(st)))
        else:
            mcpt.check(ctx.lib.mc_render_guided(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), g.handle, 1,
                                                tmp.data_ptr(), C.byref(st)))
        per = 1.0 / chunk
        split[name] = {"ms_per_spp": round(st.render_ms * per, 3), "trace": round(st.trace_ms * per, 3),
                       "shade": round(st.shade_ms * per, 3), "guide_inference": round(st.guide_infer_ms * per, 3),
                       "guide_training": round(st.guide_train_ms * per, 3)}
        split[name]["other"] = round(split[name]["ms_per_spp"] - sum(v for k, v in split[name].items()
                                                                     if k != "ms_per_spp"), 3)

    mlp = mlp_throughput(ctx, guide) if mlp else None
    guide.close()
    ratio = reached / plain_ms if reached is not None else None
    out = {"metric": "time to fixed RMSE vs plain wavefront", "value": round(ratio, 4) if ratio is not None else None,
           "unit": "guided time / plain time (lower is better)", "higher_is_better": False, "n_gpus": 1,
           "workload": "guiding_room", "triangles": int(len(tris)), "width": W, "height": H, "max_depth": s.max_depth,
           "target_rmse": round(target, 6), "plain_spp": args.guide_plain_spp, "plain_ms": round(plain_ms, 1),
           "guided_ms_to_target": round(reached, 1) if reached is not None else None,
           "guided_spp": spp, "adam_steps": steps, "learning_rate": args.guide_lr, "reference_spp": args.guide_ref_spp,
           "pretrain_spp": args.guide_pretrain_spp,
           "train_vertices": int(guide.config.train_vertices) or 1, "direction_input": args.guide_dir,
           "guided_depth": int(guide.config.guided_depth) or 2, "weight_cap": args.guide_weight_cap, "fold_below": bool(args.guide_fold),
           "anchor_lobes": args.guide_anchor != 0, "batch_records": int(guide.config.batch_capacity) or 65536,
           "nee_records": bool(args.guide_nee),
           "plain_mrays": round(rays_plain / (plain_ms / 1e3) / 1e6, 1),
           "guided_mrays": round(rays_g / (g_ms / 1e3) / 1e6, 1),
           "plain_curve": plain_curve, "guided_curve": g_curve, "phase_split_ms": split,
           "mlp": mlp,
           "data": "synthetic (seeded procedural room)", "dtype": "bf16 MLP / f32 tracer"}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_server(args):
    """Render server under Poisson load. Scenes: 16 members of the 64-scene
    batch (seeded, 1k-2M triangles) and a level-7 displaced-icosphere scene
    (983k triangles), resident with their BVHs. Requests (seed 5): scene
    uniform, resolution uniform over {256^2, 512^2, 1024^2, 1920x1080}, spp
    log-uniform in [1, 256], guided for half of them. For each arrival rate
    the same request trace runs through the server (shared waves, HBM budget
    150 GB) and through the plain per-request wavefront tracer (one request
    at a time, arrival order). Latency = completion - scheduled arrival."""
    import math
    import random

    import torch

    import mcpt
    ctx = mcpt.Context(0)
    scenes = [mcpt.generate_scene(mcpt.SCENE_BATCH_MEMBER, variant=i, seed=3) for i in range(16)]
    scenes.append(mcpt.generate_scene(mcpt.SCENE_DISPLACED_ICOSPHERES, variant=7, seed=2))
    devs = []
    for s in scenes:
        env = mcpt.host_env(s) if s.env_width > 0 else None
        devs.append(mcpt.DeviceScene(mcpt.host_triangles(s), env_rgba=env, env_intensity=s.env_intensity))
    srv = mcpt.Server(ctx, samples_per_step=args.server_sps, wave_paths=args.server_wave_paths,
                      flags=mcpt.SERVER_SCENE_WAVES if args.server_scene_waves else 0)
    sids = [srv.add_scene(d) for d in devs]
    bvhs = [mcpt.Bvh(ctx, d.view, layout=mcpt.LAYOUT_WIDE4) for d in devs]
    sizes = [(256, 256), (512, 512), (1024, 1024), (1920, 1080)]

    def trace(rate, n, seed):
        rnd = random.Random(seed)
        t, out = 0.0, []
        for _ in range(n):
            t += rnd.expovariate(rate)
            k = rnd.randrange(len(scenes))
            W, H = sizes[rnd.randrange(len(sizes))]
            spp = max(1, min(256, int(math.exp(rnd.uniform(0.0, math.log(256.0))))))
            out.append((t, k, W, H, spp, rnd.random() < 0.5))
        return out

    def params(k, W, H, spp, first=0):
        s = scenes[k]
        cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
        cam.image_width = W
        cam.aspect_ratio = W / float(H)
        mcpt.camera_initialize(cam)
        return mcpt.render_params(cam, W, H, spp, 8, persistent=True, rng=mcpt.RNG_PHILOX, seed=5, first_sample=first)

    def pct(xs, q):
        xs = sorted(xs)
        return xs[min(len(xs) - 1, int(math.ceil(q * len(xs))) - 1)]

    def serve(tr):
        t0 = srv.now()
        base_rays = srv.stats().rays
        pending = list(tr)
        ids = []
        while pending or srv.stats().active or srv.stats().pending:
            now = srv.now() - t0
            while pending and pending[0][0] <= now:
                t, k, W, H, spp, guided = pending.pop(0)
                ids.append((t, srv.submit(sids[k], params(k, W, H, spp), guided=guided)))
            st = srv.stats()
            if st.active or st.pending:
                srv.step()
                for t, rid in ids:
                    r = srv.result(rid)
                    if r.state == mcpt.REQ_DONE:
                        srv.release(rid)
            elif pending:
                time.sleep(max(0.0, min(0.002, pending[0][0] - now)))
        lat, last = [], 0.0
        for t, rid in ids:
            r = srv.result(rid)
            lat.append(r.done_s - t0 - t)
            last = max(last, r.done_s - t0)
        rays = srv.stats().rays - base_rays
        return lat, rays / last / 1e6

    def baseline(tr):
        acc = {}
        t0 = time.perf_counter()
        lat, rays, last = [], 0, 0.0
        for t, k, W, H, spp, guided in tr:
            now = time.perf_counter() - t0
            if now < t:
                time.sleep(t - now)
            a = acc.get((W, H))
            if a is None:
                a = acc[(W, H)] = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
            a.zero_()
            p = params(k, W, H, spp)
            st = mcpt.RenderStats()
            mcpt.check(ctx.lib.mc_render_wavefront(ctx.handle, bvhs[k].handle, C.byref(devs[k].view), C.byref(p),
                                                   a.data_ptr(), C.byref(st)))
            done = time.perf_counter() - t0
            lat.append(done - t)
            rays += st.extend_rays + st.shadow_rays
            last = done
        return lat, rays / last / 1e6

    # warm-up: one small request of each scene through both
    warm = [(0.0, k, 256, 256, 1, k % 2 == 0) for k in range(len(scenes))]
    serve(warm)
    baseline([(0.0, k, 256, 256, 1, False) for k in range(len(scenes))])
    def summary(runs):
        # runs: [(latencies, mrays)] of repeats -> median and range of p50, p99, Mrays/s
        cols = {"p50_s": [pct(l, 0.5) for l, _ in runs], "p99_s": [pct(l, 0.99) for l, _ in runs],
                "mrays": [m for _, m in runs]}
        out = {}
        for k, v in cols.items():
            nd = 1 if k == "mrays" else 4
            out[k] = round(statistics.median(v), nd)
            out[k + "_range"] = [round(min(v), nd), round(max(v), nd)]
        return out

    points = []
    for rate in args.server_rates:
        # the same trace for a rate whatever else is swept; fewer requests at low
        # rates, where the arrivals themselves take wall-clock time
        n_req = max(24, min(args.server_requests, int(16 * rate)))
        tr = trace(rate, n_req, 5 + int(round(rate * 1000)))
        plain_tr = [(t, k, W, H, spp, False) for t, k, W, H, spp, _ in tr]
        mixed, plain, base = [], [], []
        for _ in range(max(1, args.server_repeats)):
            mixed.append(serve(tr))
            plain.append(serve(plain_tr))
            base.append(baseline(tr))
        point = {"lambda_per_s": rate, "requests": len(tr), "guided_requests": sum(1 for x in tr if x[5]),
                 "repeats": len(mixed)}
        point.update(summary(mixed))
        point.update({"plain_only_" + k: v for k, v in summary(plain).items()})
        point.update({"baseline_" + k: v for k, v in summary(base).items()})
        points.append(point)
    st = srv.stats()
    out = {"metric": "served-render p50/p99 latency", "unit": "s", "higher_is_better": False, "n_gpus": 1,
           "workload": "render_server", "scenes": len(scenes),
           "scene_triangles": [int(s.triangle_count) for s in scenes], "budget_gb": st.budget_bytes / 1e9,
           "resident_scene_gb": round(st.scene_bytes / 1e9, 3), "samples_per_step": args.server_sps,
           "wave_paths": args.server_wave_paths or 4194304, "scene_waves": bool(args.server_scene_waves),
           "points": points, "data": "synthetic (seeded scenes and request trace)",
           "baseline": "plain per-request wavefront tracer, one request at a time in arrival order"}
    print(json.dumps(out), flush=True)
    srv.close()
    for s in scenes:
        mcpt.free_scene(s)


def run_reference(args):
    """The unmodified reference (oracle/_ref/libmcref.so: the reference's
    src/path_tracer.cu compiled for sm_100a, curand XORWOW) through its own
    renderWithWavefront with --persistent semantics, on the same scene. This
    process loads only the reference build: the scene comes from the copy of
    the library's seeded generator linked into that harness, not from the
    library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import mcref
    if not mcref.available(False):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmcref.so was not built (needs the reference sources)"}))
        return
    ref = mcref.load(False)
    scene = mcref.SceneHost()
    assert ref.mcref_generate_scene(mcref.SCENE_DISPLACED_ICOSPHERES, args.level, 2, 0, C.byref(scene)) == 0
    assert ref.mcref_scene_upload(scene.triangles, scene.triangle_count, None, 0, scene.env_rgba, scene.env_width,
                                  scene.env_height, scene.env_intensity, 0.0) == 0
    W, H, K, S = scene.width, scene.height, args.steps, args.spp_per_step
    acc = np.zeros(W * H * 3, np.float32)
    stats = np.zeros(3, np.float64)
    cam = C.addressof(scene.camera)
    for _ in range(args.warmup):
        assert ref.mcref_render(cam, W, H, 1, 8, 2, 1234, 0, 1, acc.ctypes.data, stats.ctypes.data) == 0
    clocks = Clocks(0)
    # timed: renderWithWavefront (PT:3757) itself, K steps of S samples, wavefront + persistent
    assert ref.mcref_render(cam, W, H, K * S, 8, 2, 1234, 0, 1, acc.ctypes.data, stats.ctypes.data) == 0
    ck = clocks.stop()
    ms = stats[2]
    # untimed replay of the same launch sequence that also reads the shadow-queue sizes
    assert ref.mcref_render(cam, W, H, K * S, 8, 2, 1234, 0, 0, acc.ctypes.data, stats.ctypes.data) == 0
    rays = stats[0] + stats[1]
    ref.mcref_free_scene(C.byref(scene))
    value = rays / (ms / 1e3) / 1e6
    variant = None
    if not args.no_1m and args.level == 8:
        # the ~1M-triangle reading of the scene (level-7 icospheres), fewer samples
        v = mcref.SceneHost()
        assert ref.mcref_generate_scene(mcref.SCENE_DISPLACED_ICOSPHERES, 7, 2, 0, C.byref(v)) == 0
        assert ref.mcref_scene_upload(v.triangles, v.triangle_count, None, 0, v.env_rgba, v.env_width, v.env_height,
                                      v.env_intensity, 0.0) == 0
        vspp = 4 * S
        vcam = C.addressof(v.camera)
        assert ref.mcref_render(vcam, W, H, 1, 8, 2, 1234, 0, 1, acc.ctypes.data, stats.ctypes.data) == 0
        assert ref.mcref_render(vcam, W, H, vspp, 8, 2, 1234, 0, 1, acc.ctypes.data, stats.ctypes.data) == 0
        vms = stats[2]
        assert ref.mcref_render(vcam, W, H, vspp, 8, 2, 1234, 0, 0, acc.ctypes.data, stats.ctypes.data) == 0
        variant = {"workload": "displaced_icospheres level 7", "triangles": int(v.triangle_count), "spp": vspp,
                   "value": round((stats[0] + stats[1]) / (vms / 1e3) / 1e6, 2), "unit": "Mrays/s"}
        ref.mcref_free_scene(C.byref(v))
    out = {"metric": "Mrays/s", "value": round(value, 2), "unit": "Mrays/s", "n_gpus": 1, "steps": K, "warmup": args.warmup,
           "ms_per_step": round(ms / K, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic (seeded procedural scene)", "impl": "reference",
           "config": dict(WORKLOAD, spp=K * S, spp_per_step=S, rng="curand XORWOW (the reference's own)", parallelism="1 GPU",
                          note="unmodified reference renderWithWavefront --wavefront --persistent on the B200"),
           "reference_run": {"kind": "reference", "device": "GPU (the reference's own CUDA build; it has no CPU "
                                                            "implementation of the path)",
                             "host_threads": 1, "sample": "the full workload, %d samples per pixel" % (K * S),
                             "timing": "CUDA events around renderWithWavefront inside the harness; ray counts from "
                                       "an untimed replay of the same launch sequence"},
           "e2e": {"value": round(value, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "clocks": ck}
    if variant:
        out["workload_1m"] = variant
    print(json.dumps(out), flush=True)


def run_guided_waves(args):
    """Guided waves with online training on the aperture room (1024x1024,
    anchored lobes, first bounce guided and trained, 4 Adam steps per sample):
    --steps calls of --guide-chunk samples each from a fresh guide, CUDA
    events around each call; prints rays per second and the time per sample.
    One untimed call on a separate guide loads the kernels first. A short,
    fixed launch sequence for launch lists of the guided path."""
    import numpy as np
    import torch

    import mcpt
    ctx = mcpt.Context(0)
    s = mcpt.generate_scene(mcpt.SCENE_GUIDING_ROOM)
    tris = mcpt.host_triangles(s)
    ds = mcpt.DeviceScene(tris)
    bvh = mcpt.Bvh(ctx, ds.view, layout=mcpt.LAYOUT_WIDE4)
    v = np.frombuffer(tris, dtype=np.uint8).reshape(len(tris), 224)[:, :36].copy().view(np.float32).reshape(-1, 3)
    g = mcpt.Guide(ctx, v.min(0).tolist(), v.max(0).tolist(), seed=7, train_steps=4, anchor_lobes=True,
                   guided_depth=2, train_vertices=1)
    W, H = s.width, s.height
    acc = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    warm = mcpt.Guide(ctx, v.min(0).tolist(), v.max(0).tolist(), seed=3, train_steps=4, anchor_lobes=True,
                      guided_depth=2, train_vertices=1)
    pw = mcpt.render_params(s.camera, W, H, args.guide_chunk, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX,
                            seed=4, first_sample=999000, disable_clamp=True, refill_threshold=16)
    mcpt.check(ctx.lib.mc_render_guided(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(pw), warm.handle, 1,
                                        acc.data_ptr(), C.byref(mcpt.RenderStats())))
    warm.close()
    acc.zero_()
    ms_total, rays = 0.0, 0
    for c in range(args.steps):
        p = mcpt.render_params(s.camera, W, H, args.guide_chunk, s.max_depth, persistent=True, rng=mcpt.RNG_PHILOX,
                               seed=4, first_sample=c * args.guide_chunk, disable_clamp=True, refill_threshold=16)
        st = mcpt.RenderStats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        mcpt.check(ctx.lib.mc_render_guided(ctx.handle, bvh.handle, C.byref(ds.view), C.byref(p), g.handle, 1,
                                            acc.data_ptr(), C.byref(st)))
        e1.record()
        torch.cuda.synchronize()
        ms_total += e0.elapsed_time(e1)
        rays += st.extend_rays + st.shadow_rays
    spp = args.steps * args.guide_chunk
    print(json.dumps({"metric": "Mrays/s", "value": round(rays / (ms_total / 1e3) / 1e6, 1), "unit": "Mrays/s",
                      "workload": "guided_waves (aperture room, 1024x1024)", "spp": spp,
                      "ms_per_spp": round(ms_total / spp, 3), "adam_steps": g.steps(), "n_gpus": 1,
                      "data": "synthetic (seeded procedural room)"}), flush=True)
    g.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "guiding":
        run_guiding(args)
    elif args.workload == "guided_waves":
        run_guided_waves(args)
    elif args.workload == "mlp":
        run_mlp(args)
    elif args.workload == "server":
        run_server(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
