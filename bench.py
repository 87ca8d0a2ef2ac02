"""Benchmark: Mrays/s of the cloud march at 1920x1080 (three layers, 128
primary + 6 light steps), one primary ray per pixel, march + composite.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--storage f16|u8|f32|bf16|fp8] [--schedule plain|fast]
                  [--filter exact|hybrid|texture]

Default: FP16 noise storage, FAST schedule, hybrid filtering (exact FP32
weights for the primary density, texture-unit taps for the light march) —
the form that meets the 1e-3 bar against the FP64 oracle.  The same run also
times the plain FP32-storage drop-in kernel and reports the ratio.

One process per GPU (torchrun for N > 1).  The forward march has no exchange
step, so each rank renders its own full frame of the sequence (weak scaling);
time is the max over ranks of the device-timed step.  `--impl reference`
times the CPU restatement of the reference's FP32 march on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s at 1080p, FP16-stored vs FP32 march at <=1e-3 rel err; % L2/tex roofline"
UNIT = "Mrays/s"
WORKLOAD = "precision_1080p"
# Frame workloads: name -> (default size, frames per step, description).
FRAME_WORKLOADS = {
    "precision_1080p": ((1920, 1080), 1, {"layers": "Cu 1500-2300 cov 0.5; As 4000-5000 cov 0.7; "
                                                    "Ci 8000-9000 cov 0.3", "primary_steps": 128,
                                          "light_steps": 6}),
    "plain_320x180": ((320, 180), 1, {"layers": "Cu 1500-2300 cov 0.5", "primary_steps": 64,
                                      "light_steps": 6, "phase": "dual-lobe HG 0.8/-0.2 w 0.5",
                                      "octaves": 3}),
    "stress_2160p": ((3840, 2160), 8, {"layers": "Cb 600-12000 cov 0.8 x 2048^2 f32 coverage grid",
                                       "primary_steps": 256, "light_steps": 8,
                                       "frames": "8, simulated_seconds 0..7, 15 m/s wind"}),
}


def frame_scenes(workload, W, H, **kw):
    """The scenes of one step of a frame workload."""
    from pedalsky_b200 import scenes
    if workload == "stress_2160p":
        return [scenes.stress_2160p(W, H, frame_index=k, **kw) for k in range(8)]
    if workload == "plain_320x180":
        return [scenes.plain_320x180(W, H, **kw)]
    return [scenes.precision_1080p(W, H, **kw)]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f16")
    ap.add_argument("--schedule", default="fast", choices=["plain", "fast"])
    ap.add_argument("--filter", default="hybrid", choices=["exact", "texture", "hybrid"])
    ap.add_argument("--no-plain-reference", action="store_true",
                    help="skip timing the plain FP32-storage drop-in kernel for the speed-up ratio")
    ap.add_argument("--width", type=int, default=None, help="default: the workload's size")
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="precision_1080p",
                    choices=["precision_1080p", "plain_320x180", "stress_2160p", "batch_64",
                             "grid_512"],
                    help="stress_2160p: eight 4K frames of a Cumulonimbus over a 2048^2 coverage "
                         "grid; batch_64: the 64-view uneven batch in one persistent kernel")
    ap.add_argument("--batch-views", type=int, default=64)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


class _NullCtx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in self.samples for n, v in zip(names, s[5:9]) if v == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def bytes_per_ray(storage: str, schedule: str = "fast", workload: str = WORKLOAD) -> dict:
    """Algorithmic texel bytes per primary ray of this workload: executed
    fetches counted by the instrumented CPU restatement on the same scene
    (tests/golden/fetch_counts.json) times texels per fetch (bilinear 4,
    trilinear 8, load 1) times the bytes per texel of the form the kernel
    reads.  The FAST schedule with FP16 storage reads channel-folded volumes:
    base (R, fbm) 4 B and detail (fbm) 2 B per texel, the curl tile as (R, G)
    half pairs 4 B per texel; other forms read RGBA texels (4 B for RGBA8
    and FP8, 8 B for FP16/BF16, 16 B for FP32).  LUT texels are RGBA32F.
    Outputs: L and T written, the HDR target read and written (64 B)."""
    p = ROOT / "tests" / "golden" / "fetch_counts.json"
    if not p.exists():
        return {}
    d = json.loads(p.read_text()).get(workload)
    if not d:
        return {}
    c = d["counts"]
    if schedule == "fast" and storage == "f16":
        base_b, detail_b, curl_b = 4, 2, 4
    else:
        base_b = detail_b = {"u8": 4, "fp8": 4, "f16": 8, "bf16": 8, "f32": 16}[storage]
        curl_b = 2
    per_kind = {
        "weather": 4 * 4, "base": 8 * base_b, "curl": 4 * curl_b, "detail": 8 * detail_b,
        "light": 8 * base_b, "trans": 4 * 16, "sky": 4 * 16, "ap": 8 * 16, "blue": 4, "depth": 4,
    }
    total = sum(c[k] * v for k, v in per_kind.items()) + c["pixels"] * 64
    return {"bytes_per_ray": total / c["pixels"], "pixels": c["pixels"],
            "dense_per_ray": c["dense"] / c["pixels"], "steps_per_ray": c["steps"] / c["pixels"],
            "light_fetches_per_ray": c["light"] / c["pixels"]}


# DRAM bytes (read + write) per launch of the timed kernel, from one ncu
# capture of the benchmark command (profiles/k_march_fast_f16_hybrid_1080p.md).
DRAM_TRAFFIC_PER_LAUNCH = {("precision_1080p", "fast", "f16", "hybrid", 1920, 1080): 132546048}


def fetch_peaks(device: int) -> dict:
    """L2 / L1 read bandwidth and trilinear texture fetch rate of this GPU,
    measured by the library's calibration kernels (psc_measure_fetch_peaks)."""
    from pedalsky_b200 import capi
    fp = capi.FetchPeaks()
    capi.call("psc_measure_fetch_peaks", device, C.byref(fp), None)
    return {"l2_read_gbs": fp.l2_read_gbs, "l1_read_gbs": fp.l1_read_gbs,
            "tex_trilinear_gfetch_s": fp.tex_trilinear_gfetch_s}


def cpu_baseline(scene, sample_rows: int, reps: int = 1):
    """The FP32 CPU restatement on a bounded row sample; returns (rays/s, rays, threads)."""
    from oracle import pyoracle
    noise = pyoracle.bake_noise()
    luts = pyoracle.bake_luts(scene.frame, scene.world)
    h = scene.height
    step = max(1, h // sample_rows)
    rows = list(range(0, h, step))[:sample_rows]
    threads = os.cpu_count() or 1
    # bands of consecutive rows spread over the image: `rows` start rows
    band = max(1, sample_rows // 8)
    starts = np.linspace(0, h - band, 8).astype(int)
    times = []
    rays = 0
    for _ in range(reps):
        t0 = time.perf_counter()
        rays = 0
        for r0 in starts:
            pyoracle.render(scene, noise, luts, precision=pyoracle.FP32, threads=threads,
                            rows=(int(r0), int(r0) + band))
            rays += band * scene.width
        times.append(time.perf_counter() - t0)
    del rows
    return rays / float(np.median(times)), rays, threads, float(np.median(times))


def run_reference_grid(args):
    """CPU reference arm of the grid workload: the FP64 restatement's forward +
    reverse sweep on a bounded row sample per step, all host threads."""
    from oracle import pyoracle
    from pedalsky_b200 import scenes
    sc = scenes.grid_512()
    noise = pyoracle.bake_noise()
    luts = pyoracle.bake_luts(sc.frame, sc.world)
    for _ in range(args.warmup):
        grid_cpu_baseline(sc, noise, luts, 32)
    vals = []
    for _ in range(args.steps):
        v, rays, threads, secs = grid_cpu_baseline(sc, noise, luts, 64)
        vals.append(v)
    value = float(np.median(vals)) / 1e6
    line = {
        "metric": GRID_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sc.width * sc.height / (value * 1e6), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Worley grid)", "impl": "reference",
        "config": {"workload": "grid_512", "grid": [256, 256, 64], "view": [sc.width, sc.height],
                   "primary_steps": 96, "light_steps": 6,
                   "note": "the reference has no voxel-grid form or adjoint; this is the CPU "
                           "restatement (FP64 reverse sweep) on a row sample"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{rays} rays per step (4 row bands)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    if args.workload == "grid_512":
        return run_reference_grid(args)
    wl = args.workload if args.workload in FRAME_WORKLOADS else WORKLOAD
    (dw, dh), n_frames, desc = FRAME_WORKLOADS[wl]
    W, H = args.width or dw, args.height or dh
    s = frame_scenes(wl, W, H)[0]
    sample = 64 if wl == WORKLOAD else 32  # rows per step
    for _ in range(args.warmup):
        cpu_baseline(s, sample)
    vals = []
    for _ in range(args.steps):
        v, rays, threads, secs = cpu_baseline(s, sample)
        vals.append(v)
    value = float(np.median(vals)) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * n_frames * W * H / (value * 1e6),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded reference noise hash, reference synthesis)",
        "impl": "reference",
        "config": {"workload": f"{wl} {W}x{H}", **desc,
                   "note": "CPU restatement of the reference FP32 march (the reference's WGSL "
                           "cannot run here: no graphics stack)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{rays} rays per step (8 row bands of the first frame)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    from pedalsky_b200 import capi, scenes
    from pedalsky_b200.capi import call
    from pedalsky_b200.subsystem import subsystem_for_scene

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    storage = capi.STORAGE_NAMES[args.storage]
    schedule = capi.SCHED_FAST if args.schedule == "fast" else capi.SCHED_PLAIN
    filt = capi.FILTER_NAMES[args.filter]
    wl = args.workload
    (dw, dh), n_frames, desc = FRAME_WORKLOADS[wl]
    W, H = args.width or dw, args.height or dh
    # each rank renders its own frame(s) of the sequence (weak scaling)
    frames = frame_scenes(wl, W, H, storage=storage, schedule=schedule, filt=filt)
    for f in frames:
        f.frame.frame_index += rank * n_frames
    s = frames[0]
    sub = subsystem_for_scene(s, device=local, luts=None)  # noise + LUTs baked on the device
    stream = torch.cuda.Stream(device=dev)
    sh = C.c_void_p(stream.cuda_stream)

    L = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    T = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    bg = torch.from_numpy(s.background).to(dev)
    hdr = torch.empty_like(bg)
    depth = torch.from_numpy(s.depth).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    o = capi.MarchOptions.from_buffer_copy(sub.options)
    o.composite = 1
    sub.set_options(o)
    view = capi.View(W, H, depth.data_ptr(), L.data_ptr(), T.data_ptr(), hdr.data_ptr())

    def render_step():
        """One step: every frame of the workload (the frames differ only in
        simulated time, so the sky-view and AP LUTs stay valid)."""
        for f in frames:
            if n_frames > 1:
                call("psc_set_frame", sub.handle, C.byref(f.frame), C.byref(f.world))
            hdr.copy_(bg, non_blocking=True)
            call("psc_render", sub.handle, C.byref(view), 1, sh)

    timed_launches = {}

    def timed_steps(clk=None):
        """W untimed steps, then K device-timed steps (L2 flushed before each);
        the library's kernel launches inside the timed loop go to
        timed_launches["n"]."""
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                render_step()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = sub.launch_count()
        with (clk if clk is not None else _NullCtx()):
            with torch.cuda.stream(stream):
                for i in range(args.steps):
                    flush.zero_()                      # evict L2 between timed steps
                    evs[i][0].record(stream)
                    render_step()
                    evs[i][1].record(stream)
            torch.cuda.synchronize()
        timed_launches["n"] = sub.launch_count() - l0
        ms_list = [a.elapsed_time(b) for a, b in evs]
        t = torch.tensor([float(np.mean(ms_list))], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return ms_list, float(t.item())

    peaks_fetch = None
    try:
        peaks_fetch = fetch_peaks(local)
    except Exception as e:  # the calibration is reported, never required
        print(f"fetch-peak calibration failed: {e}", file=sys.stderr)
    clk = ClockSampler(local)
    step_ms, ms_max = timed_steps(clk)
    kernel_launches = timed_launches["n"]
    rays_step = n_frames * W * H
    value = world * rays_step / (ms_max * 1e-3) / 1e6

    # the plain FP32-storage drop-in kernel on the same frame, for the ratio
    plain = None
    if not args.no_plain_reference:
        o_plain = capi.MarchOptions.from_buffer_copy(o)
        o_plain.schedule, o_plain.storage, o_plain.filter = (capi.SCHED_PLAIN, capi.STORAGE_F32,
                                                             capi.FILTER_EXACT)
        sub.set_options(o_plain)
        _, ms_plain = timed_steps()
        sub.set_options(o)
        plain = {"value": world * rays_step / (ms_plain * 1e-3) / 1e6, "ms_per_step": ms_plain,
                 "config": "plain schedule, f32 storage, exact filtering"}

    # the same frames through the persistent batched kernel (psc_render_batch,
    # one launch per step replayed from a CUDA graph, per-view LUT bakes
    # included): its rate against the plain FP32 drop-in and its fraction of
    # the L2 read ceiling are reported beside the single-view kernel's
    batched = None
    if not args.no_plain_reference and schedule == capi.SCHED_FAST:
        from pedalsky_b200 import batch as B
        bt = B.Batch(frames, dev)
        with torch.cuda.stream(stream):
            btune = B.autotune(sub.handle, bt, reps=1, stream=stream)
        B.set_tuning(sub.handle, btune["threads"], btune["tile_w"], use_graph=1)
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                bt.reset_hdr()
                bt.render(sub.handle, stream)
        torch.cuda.synchronize()
        bevs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(args.steps)]
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                bt.reset_hdr()
                bevs[i][0].record(stream)
                bt.render(sub.handle, stream)
                bevs[i][1].record(stream)
        torch.cuda.synchronize()
        ms_b = float(np.mean([a.elapsed_time(b) for a, b in bevs]))
        if world > 1:
            tb = torch.tensor([ms_b], dtype=torch.float64, device=dev)
            dist.all_reduce(tb, op=dist.ReduceOp.MAX)
            ms_b = float(tb.item())
        batched = {"value": world * rays_step / (ms_b * 1e-3) / 1e6, "ms_per_step": ms_b,
                   "config": "psc_render_batch: persistent kernel from a captured CUDA graph, "
                             "per-view LUT bakes included", "autotuned": btune}
        del bt

    # End to end through the C ABI with host buffers, as a frame stream would
    # run it: every frame copies its own depth and background from pinned host
    # memory (input copy stream), is marched and composited (compute stream),
    # and its composited frame is read back into pinned host memory (output
    # copy stream).  Two device slots alternate, so a frame's copies overlap
    # its neighbours' marches; the time is from the first input copy to the
    # last read-back, per step.
    h_bg = torch.from_numpy(s.background).pin_memory()
    h_depth = torch.from_numpy(s.depth).pin_memory()
    in_s, out_s = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    slots = []
    for _ in range(2):
        d_hdr, d_dep = torch.empty_like(hdr), torch.empty_like(depth)
        slots.append({"hdr": d_hdr, "depth": d_dep, "out": torch.empty_like(h_bg).pin_memory(),
                      "view": capi.View(W, H, d_dep.data_ptr(), L.data_ptr(), T.data_ptr(),
                                        d_hdr.data_ptr())})

    def e2e_pass(n_steps):
        if n_steps <= 0:
            return 0.0
        n = n_steps * n_frames
        freed = []  # read-back of frame i done: its slot is free for frame i + 2
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(in_s)
        for i in range(n):
            f, sl = frames[i % n_frames], slots[i % 2]
            if i >= 2:
                in_s.wait_event(freed[i - 2])
            with torch.cuda.stream(in_s):
                sl["hdr"].copy_(h_bg, non_blocking=True)
                sl["depth"].copy_(h_depth, non_blocking=True)
            got = torch.cuda.Event()
            got.record(in_s)
            stream.wait_event(got)
            with torch.cuda.stream(stream):
                if i % n_frames == 0:
                    flush.zero_()  # L2 evicted once per step, as in the device-timed run
                if n_frames > 1:
                    call("psc_set_frame", sub.handle, C.byref(f.frame), C.byref(f.world))
                call("psc_render", sub.handle, C.byref(sl["view"]), 1, sh)
            done = torch.cuda.Event()
            done.record(stream)
            out_s.wait_event(done)
            with torch.cuda.stream(out_s):
                sl["out"].copy_(sl["hdr"], non_blocking=True)
            freed.append(torch.cuda.Event())
            freed[-1].record(out_s)
        end.record(out_s)
        end.synchronize()
        return start.elapsed_time(end) / n_steps

    e2e_pass(args.warmup)
    te = torch.tensor([e2e_pass(args.steps)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * rays_step / (float(te.item()) * 1e-3) / 1e6
    h_out = slots[0]["out"]
    h2d = n_frames * (h_bg.numel() * 4 + h_depth.numel() * 4)
    d2h = n_frames * h_out.numel() * 4

    if rank == 0:
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        hbm = peaks.get("hbm_gbs")
        bpr = bytes_per_ray(args.storage, args.schedule, wl)
        roof = None
        if bpr:
            achieved = bpr["bytes_per_ray"] * rays_step / (ms_max * 1e-3) / 1e9
            peak = hbm if hbm else 6650.0
            traffic = DRAM_TRAFFIC_PER_LAUNCH.get((wl, args.schedule, args.storage, args.filter, W, H))
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "peak_source": "measured" if hbm else "fallback",
                    "bytes_per_ray": bpr["bytes_per_ray"], "kernel": "k_march_fast",
                    "note": "achieved = algorithmic texel bytes of the executed fetches per launch / "
                            "kernel time.  The noise/LUT working set is L2-resident, so these bytes "
                            "are served by L1/TEX and L2, not HBM (DRAM traffic per launch is "
                            "`traffic`); `fetch` relates them to the on-chip ceilings measured on "
                            "this GPU"}
            if peaks_fetch and batched:
                b_ach = bpr["bytes_per_ray"] * rays_step / (batched["ms_per_step"] * 1e-3) / 1e9
                batched["fetch_gbs"] = b_ach
                batched["frac_of_l2_read"] = b_ach / peaks_fetch["l2_read_gbs"]
            if peaks_fetch:
                light_rate = bpr["light_fetches_per_ray"] * rays_step / (ms_max * 1e-3) / 1e9
                roof["fetch"] = {
                    "l2_read_peak_gbs": peaks_fetch["l2_read_gbs"],
                    "frac_of_l2_read": achieved / peaks_fetch["l2_read_gbs"],
                    "l1_read_peak_gbs": peaks_fetch["l1_read_gbs"],
                    "frac_of_l1_read": achieved / peaks_fetch["l1_read_gbs"],
                    "tex_trilinear_peak_gfetch_s": peaks_fetch["tex_trilinear_gfetch_s"],
                    "light_march_gfetch_s": light_rate,
                    "frac_of_tex_trilinear": light_rate / peaks_fetch["tex_trilinear_gfetch_s"],
                    "source": "psc_measure_fetch_peaks, this run"}
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                v, rays, threads, secs = cpu_baseline(s, 64 if wl == WORKLOAD else 32)
                cpu = {"value": v / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
                       "sample": f"{rays} rays (8 row bands of the first {W}x{H} frame), {secs:.1f} s"}
            except Exception as e:  # the baseline is reported, never the product
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                       "sample": f"failed: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded reference noise hash, reference synthesis)",
            "config": {"workload": f"{wl} {W}x{H}", **desc, "storage": args.storage,
                       "schedule": args.schedule,
                       "filter": args.filter, "composite": "fused",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"views{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "pipeline": "per frame: pinned H2D, march + composite, D2H on three "
                                "streams, two device slots"},
            "gpu_launches": kernel_launches,
            "roofline": roof,
            "plain_fp32_dropin": plain,
            "speedup_vs_plain_fp32": (value / plain["value"]) if plain else None,
            "batched_fp16": batched,
            "batched_speedup_vs_plain_fp32": (batched["value"] / plain["value"])
            if (batched and plain) else None,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "step_ms": [round(x, 4) for x in step_ms],
        }
        print(json.dumps(line), flush=True)
    sub.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """64 uneven views with their own scenes, one persistent kernel per step,
    relaunched from a captured CUDA graph; launch shape chosen by the autotuner."""
    import torch

    from pedalsky_b200 import batch as B
    from pedalsky_b200 import capi, scenes
    from pedalsky_b200.subsystem import subsystem_for_scene

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    storage = capi.STORAGE_NAMES[args.storage]
    filt = capi.FILTER_NAMES[args.filter]
    views = scenes.batch_views(args.batch_views, seed=rank, host_inputs=False, storage=storage,
                               filt=filt, composite=1)
    sub = subsystem_for_scene(views[0], device=local, luts=None)
    b = B.Batch(views, dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    with torch.cuda.stream(stream):
        tune = B.autotune(sub.handle, b, reps=1, stream=stream)
    B.set_tuning(sub.handle, tune["threads"], tune["tile_w"], use_graph=1)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            b.reset_hdr()
            b.render(sub.handle, stream)
    torch.cuda.synchronize()
    launches0 = sub.launch_count()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.zero_()
                b.reset_hdr()
                evs[i][0].record(stream)
                b.render(sub.handle, stream)
                evs[i][1].record(stream)
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(c) for a, c in evs]
    ms = float(np.mean(step_ms))
    value = world * b.rays / (ms * 1e-3) / 1e6
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random scenes per view, reference synthesis)",
            "config": {"workload": f"batch_{args.batch_views} uneven views", "rays_per_step": b.rays,
                       "storage": args.storage, "filter": args.filter, "schedule": "fast",
                       "launch": "one persistent kernel per step from a captured CUDA graph",
                       "autotuned": tune, "l2": "flushed between timed steps (256 MiB write)"},
            "e2e": None, "gpu_launches": sub.launch_count() - launches0,
            "clocks": clk.summary(), "step_ms": [round(x, 3) for x in step_ms],
        }
        print(json.dumps(line), flush=True)
    sub.close()
    return 0


GRID_METRIC = ("Mrays/s of the adjoint (forward + checkpointed reverse + gradient all-reduce), "
               "512^2 view of a 256x256x64 voxel grid, 96+6 steps")


def grid_bytes_per_ray() -> dict:
    """Algorithmic bytes per ray of the grid forward and adjoint kernels from
    the executed work counted by the CPU restatement (fetch_counts.json):
    FP32 texels read by primary and light taps, two bilinear RGBA32F LUT taps
    (sun transmittance, sky view) per step, the blue-noise load and the L/T
    writes; the adjoint adds the segment recompute (texels again), the
    reverse sweep's LUT taps, one 4-byte atomic add per texel and the
    background/target reads."""
    p = ROOT / "tests" / "golden" / "fetch_counts.json"
    if not p.exists():
        return {}
    d = json.loads(p.read_text()).get("grid_512")
    if not d:
        return {}
    c = d["counts"]
    px = c["pixels"]
    tex = 4 * (c["primary_texels"] + c["light_texels"])
    lut = c["steps"] * 2 * 4 * 16
    fwd = (tex + lut) / px + 4 + 32
    adj = (3 * tex + 2 * lut) / px + 4 + 32 + 32
    return {"forward": fwd, "adjoint": adj, "steps_per_ray": c["steps"] / px}


def grid_cpu_baseline(sc, noise, luts, rows: int):
    """FP64 CPU restatement of forward + reverse sweep on `rows` rows spread
    over the view; returns (rays/s, rays, threads, seconds)."""
    from oracle import pyoracle
    G = sc.extra["grid"]
    spec = sc.extra["grid_spec"]
    bg = sc.background
    tgt = np.ascontiguousarray(bg, np.float32)  # the timing does not depend on the target values
    threads = os.cpu_count() or 1
    band = max(1, rows // 4)
    starts = np.linspace(0, sc.height - band, 4).astype(int)
    t0 = time.perf_counter()
    for r0 in starts:
        pyoracle.grid_adjoint(sc, noise, luts, G, spec, bg, tgt, threads=threads,
                              rows=(int(r0), int(r0) + band))
    secs = time.perf_counter() - t0
    rays = 4 * band * sc.width
    return rays / secs, rays, threads, secs


def run_grid(args):
    """The differentiable form: one 512^2 view's loss gradient per step.  Pixels
    are sharded in row bands over the ranks (strong scaling); each rank runs
    its band's adjoint and one sum all-reduce (NCCL) of the 16 MiB gradient
    grid gives every rank the whole image's gradient."""
    import datetime

    import torch
    import torch.distributed as dist

    from pedalsky_b200 import grid as GR
    from pedalsky_b200 import scenes, sharding
    from pedalsky_b200.subsystem import subsystem_for_scene

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sc = scenes.grid_512()
    W, H = sc.width, sc.height
    G = sc.extra["grid"]
    sub = subsystem_for_scene(sc, device=local, luts=None)
    stream = torch.cuda.Stream(device=dev)
    sh = stream
    P = GR.GridProblem(sc, G, device=dev)
    Pt = GR.GridProblem(sc, scenes.grid_target_values(G), device=dev)
    with torch.cuda.stream(stream):
        Pt.render(sub.handle, stream=sh)
        P.set_target(Pt.composite_image())
    torch.cuda.synchronize()
    del Pt
    band = sharding.row_bands(H, world)[rank]
    rows = (band.y0, band.y1) if world > 1 else None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        P.zero_grad()
        P.adjoint(sub.handle, rows=rows, stream=sh)
        sharding.allreduce_gradient(P.grad, P.acc)

    def timed(fn, n):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(n)]
        with torch.cuda.stream(stream):
            for i in range(n):
                flush.zero_()
                evs[i][0].record(stream)
                fn()
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        ms = [a.elapsed_time(b) for a, b in evs]
        return ms, sharding.max_over_ranks(float(np.mean(ms)), device=dev)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = sub.launch_count()
    with ClockSampler(local) as clk:
        step_ms, ms = timed(step, args.steps)
    launches = sub.launch_count() - launches0
    value = W * H / (ms * 1e-3) / 1e6
    fwd_ms_list, fwd_ms = timed(lambda: P.render(sub.handle, rows=rows, stream=sh), args.steps)
    adj_only_ms_list, adj_ms = timed(lambda: (P.zero_grad(), P.adjoint(sub.handle, rows=rows, stream=sh)),
                                     args.steps)

    # end to end: the grid values go up from pinned host memory, the loss
    # and the gradient come back
    h_vals = torch.from_numpy(np.ascontiguousarray(G)).pin_memory()
    h_grad = torch.empty_like(h_vals).pin_memory()
    h_acc = torch.empty(2, dtype=torch.float64).pin_memory()

    def e2e():
        P.values.copy_(h_vals, non_blocking=True)
        step()
        h_grad.copy_(P.grad, non_blocking=True)
        h_acc.copy_(P.acc, non_blocking=True)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            e2e()
    _, e2e_ms = timed(e2e, args.steps)
    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = peaks.get("hbm_gbs")
        peak = hbm if hbm else 6650.0
        bpr = grid_bytes_per_ray()
        roof = None
        if bpr:
            rays_rank = W * (band.y1 - band.y0)
            ach = bpr["adjoint"] * rays_rank / (adj_ms * 1e-3) / 1e9
            roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "traffic": None, "peak_source": "measured" if hbm else "fallback",
                    "bytes_per_ray": bpr["adjoint"], "kernel": "k_grid_march<adjoint>",
                    "note": "algorithmic bytes (texels, LUT taps, atomic adds); the grid and "
                            "gradient (16 MiB each) are L2-resident"}
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            from oracle import pyoracle
            noise = pyoracle.bake_noise()
            luts = pyoracle.bake_luts(sc.frame, sc.world)
            v, rays, threads, secs = grid_cpu_baseline(sc, noise, luts, 128)
            cpu = {"value": v / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{rays} rays (4 row bands), FP64 forward + reverse sweep, {secs:.1f} s"}
        line = {
            "metric": GRID_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Worley grid; target = render of the grid with 5% noise)",
            "config": {"workload": "grid_512", "grid": [256, 256, 64], "view": [W, H],
                       "primary_steps": 96, "light_steps": 6, "checkpoint_every": 16,
                       "exit_transmittance": 0.01,
                       "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": f"rowbands{world} + all-reduce"},
            "forward_only": {"value": W * H / (fwd_ms * 1e-3) / 1e6, "ms_per_step": fwd_ms},
            "adjoint_kernel_ms": adj_ms,
            "e2e": {"value": W * H / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": h_vals.numel() * 4,
                    "d2h_bytes_per_step": h_grad.numel() * 4 + 16},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "step_ms": [round(x, 4) for x in step_ms],
        }
        print(json.dumps(line), flush=True)
    sub.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch_64":
        return run_batch(args)
    if args.workload == "grid_512":
        return run_grid(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
