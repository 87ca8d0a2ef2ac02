"""Benchmark: Mrays/s of the cloud march at 1920x1080 (three layers, 128
primary + 6 light steps), one primary ray per pixel, march + composite.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload precision_1080p|plain_320x180|stress_2160p|batch_64|grid_512]
                  [--storage f16|u8|f32|bf16|fp8] [--schedule plain|fast]
                  [--filter exact|hybrid|texture] [--no-legs]

Default: FP16 noise storage, FAST schedule, hybrid filtering (exact FP32
weights for the primary density, texture-unit taps for the light march) —
the form that meets the 1e-3 bar against the FP64 oracle.  The default run
prints ONE JSON line: the headline (the 1080p frame), the plain FP32-storage
drop-in on the same frame, the same frame through the batched kernel, the
frame split into row bands over the ranks, and three legs with their own
timing and clock record: the 64-view uneven batch, the eight 4K Cumulonimbus
frames and the grid adjoint.

One process per GPU.  `--gpus N` without a torchrun environment re-launches
itself under torch.distributed.run with N ranks.  The forward march has no
exchange step: for the headline each rank renders its own frame of the
sequence (weak scaling); the 64 views and the eight 4K frames are partitioned
over the ranks by estimated cost, and the row-band leg splits one frame (both
strong scaling, the fixed total work divided); the grid adjoint shards rows
and sums its gradient with one NCCL all-reduce.  Times are device-timed
(CUDA events on the launching stream) and the max over ranks.

`--impl reference` times the CPU restatement of the reference's FP32 march
on the host cores (the reference's own WGSL cannot run on this box), each
step a bounded row sample of the same frame; only rank 0 works.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import socket
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
L2_NOTE = ("GPU arm: L2 flushed between timed steps (256 MiB write); CPU arm: no flush, its "
           "working set stays in the host caches")
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
# Which GPU tests hold each workload's parity against the FP64 oracle.
PARITY = {
    "precision_1080p": "tests/test_gpu_fullsize.py::test_precision_1080p_benchmark_pipeline "
                       "(full frame, GPU-baked noise and LUTs, this exact form)",
    "plain_320x180": "tests/test_gpu_march.py (c1, every storage and filter form)",
    "stress_2160p": "tests/test_gpu_fullsize.py::test_stress_2160p_frame_benchmark_pipeline "
                    "(a full 3840x2160 frame) and tests/test_gpu_march.py (frames 0 and 7)",
    "batch_64": "tests/test_gpu_batch.py (batched views against single-view renders and the "
                "FP64 oracle)",
    "grid_512": "tests/test_gpu_grid.py (gradients against the FP64 reverse sweep and central "
                "differences)",
}
# ncu figures of the timed kernel on the benchmark command: DRAM bytes read +
# written per launch and the fraction of issue slots busy (the binding limit).
NCU_KERNEL = {("precision_1080p", "fast", "f16", "hybrid", 1920, 1080):
              {"traffic": 132197120, "issue_active": 0.837}}


def workload_config(wl, W, H):
    """The workload as both arms state it (the reference arm uses the same dict)."""
    _, _, desc = FRAME_WORKLOADS[wl]
    return {"workload": f"{wl} {W}x{H}", **desc, "l2": L2_NOTE}


def frame_scenes(workload, W, H, **kw):
    """The scenes of one step of a frame workload."""
    from pedalsky_b200 import scenes
    if workload == "stress_2160p":
        return [scenes.stress_2160p(W, H, frame_index=k, **kw) for k in range(8)]
    if workload == "plain_320x180":
        return [scenes.plain_320x180(W, H, **kw)]
    return [scenes.precision_1080p(W, H, **kw)]


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f16")
    ap.add_argument("--schedule", default="fast", choices=["plain", "fast"])
    ap.add_argument("--filter", default="hybrid", choices=["exact", "texture", "hybrid"])
    ap.add_argument("--no-plain-reference", action="store_true",
                    help="skip the plain FP32-storage drop-in and the batched form of the frame")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the 64-view, 8x4K and grid-adjoint legs of the default run")
    ap.add_argument("--legs", default="all",
                    help="comma-separated legs of the default run (batch_64, stress_2160p, "
                         "grid_512, layer_params_480x270, passes_1080p) or all")
    ap.add_argument("--width", type=int, default=None, help="default: the workload's size")
    ap.add_argument("--height", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="precision_1080p",
                    choices=["precision_1080p", "plain_320x180", "stress_2160p", "batch_64",
                             "grid_512"],
                    help="stress_2160p: eight 4K frames of a Cumulonimbus over a 2048^2 coverage "
                         "grid; batch_64: the 64-view uneven batch in one persistent kernel")
    ap.add_argument("--batch-views", type=int, default=64)
    return ap.parse_args(argv)


# ---------------------------------------------------------------- ranks

class Ranks:
    """This process's place in the job (torchrun environment) and the
    collectives the benchmark uses: a barrier and the max of a scalar."""

    def __init__(self, backend="nccl"):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.dist = None
        self.backend = backend

    def init(self, device):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(self.backend, init_method="env://",
                                    timeout=datetime.timedelta(seconds=180), device_id=device)
            self.dist = dist
            assert dist.get_world_size() == self.world
        return self

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, value: float, device) -> float:
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def relaunch(args) -> int:
    """`--gpus N` outside torchrun: run this script under torch.distributed.run
    with N ranks on this node and return its exit status."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve()), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


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


# ------------------------------------------------------------- roofline

# Bytes per fetch of the FAST schedule's forms, by kind: a bilinear or
# trilinear tap is its texels times the bytes of the form read.  F16
# storage reads the channel-folded volumes (base 4 B and detail 2 B per
# texel, the curl tile as (R, G) half pairs); other storages read RGBA
# texels (4 B for RGBA8 and FP8, 8 B for FP16/BF16, 16 B for FP32).  LUT
# texels are RGBA32F.  Outputs: L and T written, the HDR target read and
# written (64 B per ray).
def fetch_sizes(storage: str, schedule: str = "fast") -> dict:
    if schedule == "fast" and storage == "f16":
        base_b, detail_b, curl_b = 4, 2, 4
    else:
        base_b = detail_b = {"u8": 4, "fp8": 4, "f16": 8, "bf16": 8, "f32": 16}[storage]
        curl_b = 2
    return {"weather": 4 * 4, "type": 1, "base": 8 * base_b, "curl": 4 * curl_b,
            "detail": 8 * detail_b, "light": 8 * base_b, "trans": 4 * 16, "sky": 4 * 16,
            "ap": 8 * 16, "blue": 4, "depth": 4, "output": 64}


def bytes_per_ray(storage: str, schedule: str = "fast", workload: str = WORKLOAD) -> dict:
    """Algorithmic texel bytes per primary ray of this workload: the fetches
    the reference algorithm executes on the same scene, counted by the
    instrumented CPU restatement (tests/golden/fetch_counts.json), times the
    bytes per fetch of the form the kernel reads (fetch_sizes)."""
    p = ROOT / "tests" / "golden" / "fetch_counts.json"
    if not p.exists():
        return {}
    d = json.loads(p.read_text()).get(workload)
    if not d:
        return {}
    c = d["counts"]
    sz = fetch_sizes(storage, schedule)
    total = sum(c[k] * sz[k] for k in ("weather", "base", "curl", "detail", "light", "trans",
                                       "sky", "ap", "blue", "depth")) + c["pixels"] * sz["output"]
    return {"bytes_per_ray": total / c["pixels"], "pixels": c["pixels"],
            "dense_per_ray": c["dense"] / c["pixels"], "steps_per_ray": c["steps"] / c["pixels"],
            "light_fetches_per_ray": c["light"] / c["pixels"]}


def fetched_bytes_per_ray(counts: dict, storage: str, schedule: str = "fast") -> dict:
    """Bytes per ray the FAST kernel actually requested, from the counts of
    its instrumented build (psc_count_fetches) on the benchmark frame."""
    sz = fetch_sizes(storage, schedule)
    n = max(counts["rays"], 1)
    total = (counts["weather_taps"] * sz["weather"] + counts["type_loads"] * sz["type"]
             + counts["live_steps"] * (sz["base"] + sz["curl"])
             + counts["detail_taps"] * sz["detail"] + counts["light_taps"] * sz["light"]
             + counts["transmittance_taps"] * sz["trans"] + counts["skyview_taps"] * sz["sky"]
             + counts["ap_taps"] * sz["ap"] + counts["depth_loads"] * sz["depth"]
             + counts["rays"] * (sz["blue"] + sz["output"]))
    passes = max(counts.get("dense_warp_passes", 0), 1)
    return {"bytes_per_ray": total / n, "steps_per_ray": counts["primary_steps"] / n,
            "live_steps_per_ray": counts["live_steps"] / n,
            "dense_per_ray": counts["dense_samples"] / n,
            "light_fetches_per_ray": counts["light_taps"] / n,
            "dense_body_simt_efficiency": counts.get("dense_warp_lanes", 0) / (32.0 * passes)}


def fetch_peaks(device: int) -> dict:
    """L2 / L1 read bandwidth and trilinear texture fetch rate of this GPU,
    measured by the library's calibration kernels (psc_measure_fetch_peaks)."""
    from pedalsky_b200 import capi
    fp = capi.FetchPeaks()
    capi.call("psc_measure_fetch_peaks", device, C.byref(fp), None)
    return {"l2_read_gbs": fp.l2_read_gbs, "l1_read_gbs": fp.l1_read_gbs,
            "tex_trilinear_gfetch_s": fp.tex_trilinear_gfetch_s}


def measured_peaks() -> dict:
    pk = ROOT / "MEASURED_PEAKS.json"
    return json.loads(pk.read_text()) if pk.exists() else {}


# ---------------------------------------------------------- CPU baseline

def cpu_sample(scene, noise, luts, rows: int, bands: int = 8):
    """One bounded sample of the FP32 CPU restatement: `bands` bands of
    rows // bands consecutive rows spread over the frame, all host threads.
    Returns (rays, seconds, threads)."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    band = max(1, rows // bands)
    starts = np.linspace(0, scene.height - band, bands).astype(int)
    t0 = time.perf_counter()
    for r0 in starts:
        pyoracle.render(scene, noise, luts, precision=pyoracle.FP32, threads=threads,
                        rows=(int(r0), int(r0) + band))
    return bands * band * scene.width, time.perf_counter() - t0, threads


def cpu_baseline(scene, rows: int, reps: int = 5):
    """Median over `reps` repeats (after one warm-up) of the FP32 CPU
    restatement on a bounded row sample of `scene`."""
    from oracle import pyoracle
    noise = pyoracle.bake_noise()
    luts = pyoracle.bake_luts(scene.frame, scene.world)
    cpu_sample(scene, noise, luts, rows)
    runs = [cpu_sample(scene, noise, luts, rows) for _ in range(reps)]
    rays, threads = runs[0][0], runs[0][2]
    secs = float(np.median([r[1] for r in runs]))
    return {"value": rays / secs / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{rays} rays (8 row bands of the {scene.width}x{scene.height} frame) per "
                      f"repeat, median of {reps} repeats after one warm-up: {secs:.2f} s"}


# ------------------------------------------------------- reference arm

def run_reference(args):
    """The CPU restatement of the reference's FP32 march, timed on the host
    cores: each step is one bounded row sample of the frame, timed whole.
    The scene is assembled by the oracle's own restatements of the
    reference's input producers, so this process maps no product library."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    from oracle import pyoracle
    from pedalsky_b200 import scenes
    if args.workload == "grid_512":
        return run_reference_grid(args)
    wl = args.workload if args.workload in FRAME_WORKLOADS else WORKLOAD
    (dw, dh), n_frames, desc = FRAME_WORKLOADS[wl]
    W, H = args.width or dw, args.height or dh
    with scenes.host_helpers(pyoracle.OracleHost()):
        if wl == "stress_2160p":
            s = scenes.stress_2160p(W, H, frame_index=0)
        else:
            s = frame_scenes(wl, W, H)[0]
    noise = pyoracle.bake_noise()
    luts = pyoracle.bake_luts(s.frame, s.world)
    rows = 64 if wl == WORKLOAD else 32
    for _ in range(args.warmup):
        cpu_sample(s, noise, luts, rows)
    runs = [cpu_sample(s, noise, luts, rows) for _ in range(args.steps)]
    rays, threads = runs[0][0], runs[0][2]
    secs = [r[1] for r in runs]
    value = float(np.median([rays / t for t in secs])) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded reference noise hash, reference synthesis)",
        "impl": "reference",
        "config": workload_config(wl, W, H),
        "arm": "CPU restatement of the reference's FP32 march (RGBA8 noise, RGBA16F LUTs and "
               "weather, FP32 arithmetic), all host threads; the reference's own WGSL path "
               "needs a graphics stack, which this box does not have",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step marches {rays} rays (8 row bands of the {W}x{H} "
                                   f"frame) and is timed whole; ms_per_step is that sample's "
                                   f"time, value the median rate over the steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "rays_per_step": rays,
    }
    print(json.dumps(line), flush=True)
    return 0


def grid_cpu_sample(sc, noise, luts, rows: int):
    """FP64 CPU restatement of the grid forward + reverse sweep on `rows`
    rows (4 bands) spread over the view; returns (rays, seconds, threads)."""
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
    return 4 * band * sc.width, time.perf_counter() - t0, threads


GRID_METRIC = ("Mrays/s of the adjoint (forward + checkpointed reverse + gradient all-reduce), "
               "512^2 view of a 256x256x64 voxel grid, 96+6 steps")


def grid_config(world=1):
    return {"workload": "grid_512", "grid": [256, 256, 64], "view": [512, 512],
            "primary_steps": 96, "light_steps": 6, "checkpoint_every": 16,
            "exit_transmittance": 0.01, "l2": L2_NOTE}


def run_reference_grid(args):
    """CPU reference arm of the grid workload: the FP64 restatement's forward +
    reverse sweep on a bounded row sample per step, all host threads."""
    from oracle import pyoracle
    from pedalsky_b200 import scenes
    with scenes.host_helpers(pyoracle.OracleHost()):
        sc = scenes.grid_512()
    noise = pyoracle.bake_noise()
    luts = pyoracle.bake_luts(sc.frame, sc.world)
    for _ in range(args.warmup):
        grid_cpu_sample(sc, noise, luts, 32)
    runs = [grid_cpu_sample(sc, noise, luts, 64) for _ in range(args.steps)]
    rays, threads = runs[0][0], runs[0][2]
    secs = [r[1] for r in runs]
    value = float(np.median([rays / t for t in secs])) / 1e6
    line = {
        "metric": GRID_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Worley grid)", "impl": "reference",
        "config": grid_config(),
        "arm": "the reference has no voxel-grid form or adjoint; this is the CPU restatement "
               "(FP64 reverse sweep)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step runs {rays} rays (4 row bands) and is timed whole"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "rays_per_step": rays,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ our arm

class Bench:
    """Per-process GPU state shared by the legs: device, stream, L2 flush
    buffer, ranks."""

    def __init__(self, args, ranks: Ranks):
        import torch
        self.torch = torch
        self.args = args
        self.ranks = ranks
        torch.cuda.set_device(ranks.local)
        self.dev = torch.device("cuda", ranks.local)
        ranks.init(self.dev)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=self.dev)

    def timed(self, step, pre=None, clk=None, kernel_events=None, steps=None, warmup=None,
              counter=None):
        """W untimed steps, then K device-timed steps with the L2 flushed (and
        `pre` run) before each, outside the events.  Returns (per-step ms of
        this rank, the max over ranks of their mean).  `kernel_events`, when
        given, is a list that `step` appends (start, end) event pairs to;
        `counter`, when given, returns the library's launch count, and the
        launches of the K timed steps go to self.timed_launches."""
        torch = self.torch
        steps = self.args.steps if steps is None else steps
        warmup = self.args.warmup if warmup is None else warmup
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):
                if pre:
                    pre()
                step()
        torch.cuda.synchronize()
        if kernel_events is not None:
            kernel_events.clear()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        self.ranks.barrier()
        torch.cuda.synchronize()
        c0 = counter() if counter else 0
        with (clk if clk is not None else _NullCtx()):
            with torch.cuda.stream(self.stream):
                for i in range(steps):
                    self.flush.zero_()
                    if pre:
                        pre()
                    evs[i][0].record(self.stream)
                    step()
                    evs[i][1].record(self.stream)
            torch.cuda.synchronize()
        self.timed_launches = (counter() - c0) if counter else None
        ms = [a.elapsed_time(b) for a, b in evs]
        mean = float(np.mean(ms)) if ms else 0.0
        return ms, self.ranks.max(mean, self.dev)

    def sh(self):
        return C.c_void_p(self.stream.cuda_stream)


def leg_row_bands(B: Bench, sub, s, depth, bg):
    """One frame split into contiguous row bands, one per rank (weighted by
    the rows' sky fraction: ground pixels stop at the depth buffer), each
    band marched through psc_render with its viewport offset, then the
    composited bands all-gathered so every rank holds the whole frame."""
    from pedalsky_b200 import capi, sharding
    from pedalsky_b200.capi import call
    torch = B.torch
    W, H = s.width, s.height
    sky_rows = (s.depth == 0).mean(axis=1) + 0.25
    bands = sharding.row_bands(H, B.ranks.world, sky_rows)
    band = bands[B.ranks.rank]
    rows = band.y1 - band.y0
    L = torch.empty((max(rows, 1), W, 4), dtype=torch.float32, device=B.dev)
    T = torch.empty_like(L)
    hdr = torch.empty_like(L)
    bg_band = bg[band.y0:band.y1].contiguous() if rows else None
    dep_band = depth[band.y0:band.y1].contiguous() if rows else None
    view = capi.View(W, rows, dep_band.data_ptr() if rows else None, L.data_ptr(), T.data_ptr(),
                     hdr.data_ptr(), W, H, 0, band.y0)
    full = {}

    def pre():
        if rows:
            hdr[:rows].copy_(bg_band, non_blocking=True)

    def step():
        if rows:
            call("psc_render", sub.handle, C.byref(view), 1, B.sh())
        if B.ranks.world > 1:
            full["img"] = sharding.gather_rows(hdr[:rows], band, bands)

    ms, ms_max = B.timed(step, pre=pre)
    return {"value": W * H / (ms_max * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_max,
            "scaling": "strong", "ranks": B.ranks.world,
            "bands": [[b.y0, b.y1] for b in bands],
            "config": "the headline frame split into one row band per rank (psc_render with a "
                      "viewport offset), then all-gathered (NCCL) into the whole frame on every "
                      "rank; the gather is inside the timed step"}


def leg_batch64(B: Bench, storage, filt, n_views=64):
    """c3: 64 seeded views of uneven size and scene, partitioned over the
    ranks by estimated cost (largest first onto the lightest rank); each
    rank marches its views in one persistent kernel per step, replayed from
    a captured CUDA graph, launch shape from the autotuner."""
    from pedalsky_b200 import batch as Bt
    from pedalsky_b200 import scenes, sharding
    from pedalsky_b200.subsystem import subsystem_for_scene
    views = scenes.batch_views(n_views, seed=0, host_inputs=False, storage=storage, filt=filt,
                               composite=1)
    costs = [sharding.view_cost(v.width, v.height, v.params.cloud_steps, v.n_layers) for v in views]
    parts = sharding.partition_views(costs, B.ranks.world)
    mine = [views[i] for i in parts[B.ranks.rank]]
    total_rays = sum(v.width * v.height for v in views)
    sub = b = None
    tune = None
    launches = 0
    if mine:
        sub = subsystem_for_scene(mine[0], device=B.ranks.local, luts=None)
        b = Bt.Batch(mine, B.dev)
        with B.torch.cuda.stream(B.stream):
            tune = Bt.autotune(sub.handle, b, reps=1, stream=B.stream)
        Bt.set_tuning(sub.handle, tune["threads"], tune["tile_w"], use_graph=1,
                      form=tune["form_id"])
    clk = ClockSampler(B.ranks.local)
    ms, ms_max = B.timed((lambda: b.render(sub.handle, B.stream)) if mine else (lambda: None),
                         pre=(b.reset_hdr if mine else None), clk=clk,
                         counter=(sub.launch_count if mine else None))
    if mine:
        launches = B.timed_launches
        sub.close()
    return {"metric": f"Mrays/s, {n_views} uneven views (c3)", "value":
            total_rays / (ms_max * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_max,
            "scaling": "strong", "rays_per_step": total_rays, "views": n_views,
            "views_this_rank": len(mine), "autotuned": tune, "gpu_launches": launches,
            "config": "the autotuned form (persistent kernel or one kernel per view) per rank "
                      "per step from a captured CUDA graph; a view's sky-view / aerial-perspective "
                      "LUTs are re-baked in the step whenever its camera or sun changed (the 64 "
                      "views are static, so the timed steps bake none); views split over ranks "
                      "by estimated cost",
            "parity": PARITY["batch_64"], "clocks": clk.summary(),
            "step_ms": [round(x, 3) for x in ms]}


def leg_stress(B: Bench, storage, schedule, filt, W=3840, H=2160):
    """c5: eight 4K Cumulonimbus frames (simulated_seconds 0..7 at 15 m/s)
    over a 2048^2 coverage grid, partitioned over the ranks; each frame is
    one march + fused composite."""
    from pedalsky_b200 import capi, scenes, sharding
    from pedalsky_b200.capi import call
    from pedalsky_b200.subsystem import subsystem_for_scene
    torch = B.torch
    frames = [scenes.stress_2160p(W, H, frame_index=k, host_inputs=False, storage=storage,
                                  schedule=schedule, filt=filt) for k in range(8)]
    parts = sharding.partition_views([1.0] * 8, B.ranks.world)
    mine = [frames[i] for i in parts[B.ranks.rank]]
    launches = 0
    sub = None
    if mine:
        sub = subsystem_for_scene(mine[0], device=B.ranks.local, luts=None)
        o = capi.MarchOptions.from_buffer_copy(sub.options)
        o.composite = 1
        sub.set_options(o)
        depth, bg = scenes.device_inputs(mine[0].frame, mine[0].world, W, H, B.dev)
        hdr = torch.empty_like(bg)
        L = torch.empty_like(bg)
        T = torch.empty_like(bg)
        view = capi.View(W, H, depth.data_ptr(), L.data_ptr(), T.data_ptr(), hdr.data_ptr())

    def step():
        for f in mine:
            call("psc_set_frame", sub.handle, C.byref(f.frame), C.byref(f.world))
            hdr.copy_(bg, non_blocking=True)
            call("psc_render", sub.handle, C.byref(view), 1, B.sh())

    clk = ClockSampler(B.ranks.local)
    ms, ms_max = B.timed(step, clk=clk, counter=(sub.launch_count if mine else None))
    if mine:
        launches = B.timed_launches
        sub.close()
    rays = 8 * W * H
    return {"metric": "Mrays/s, eight 3840x2160 Cumulonimbus frames (c5)",
            "value": rays / (ms_max * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_max,
            "scaling": "strong", "rays_per_step": rays, "frames_this_rank": len(mine),
            "gpu_launches": launches,
            "config": f"{storage} storage, {schedule} schedule, {filt} filtering, fused "
                      "composite; 256 + 8 steps; frames split over ranks",
            "parity": PARITY["stress_2160p"], "clocks": clk.summary(),
            "step_ms": [round(x, 3) for x in ms]}


def leg_grid(B: Bench, with_e2e=False):
    """c4: one 512^2 view's loss gradient with respect to the 256x256x64
    voxel grid per step.  Pixels are sharded in row bands over the ranks;
    each rank runs its band's adjoint and one sum all-reduce (NCCL) of the
    16 MiB gradient grid gives every rank the whole image's gradient."""
    from pedalsky_b200 import grid as GR
    from pedalsky_b200 import scenes, sharding
    from pedalsky_b200.subsystem import subsystem_for_scene
    torch = B.torch
    sc = scenes.grid_512()
    W, H = sc.width, sc.height
    G = sc.extra["grid"]
    sub = subsystem_for_scene(sc, device=B.ranks.local, luts=None)
    P = GR.GridProblem(sc, G, device=B.dev)
    Pt = GR.GridProblem(sc, scenes.grid_target_values(G), device=B.dev)
    with torch.cuda.stream(B.stream):
        Pt.render(sub.handle, stream=B.stream)
        P.set_target(Pt.composite_image())
    torch.cuda.synchronize()
    del Pt
    band = sharding.row_bands(H, B.ranks.world)[B.ranks.rank]
    rows = (band.y0, band.y1) if B.ranks.world > 1 else None

    def step():
        P.zero_grad()
        if band.y1 > band.y0:
            P.adjoint(sub.handle, rows=rows, stream=B.stream)
        sharding.allreduce_gradient(P.grad, P.acc)

    clk = ClockSampler(B.ranks.local)
    ms, ms_max = B.timed(step, clk=clk, counter=sub.launch_count)
    launches = B.timed_launches
    _, fwd_ms = B.timed(lambda: P.render(sub.handle, rows=rows, stream=B.stream))
    _, adj_ms = B.timed(lambda: (P.zero_grad(), P.adjoint(sub.handle, rows=rows, stream=B.stream)))
    out = {"metric": GRID_METRIC, "value": W * H / (ms_max * 1e-3) / 1e6, "unit": UNIT,
           "ms_per_step": ms_max, "scaling": "strong", "gpu_launches": launches,
           "forward_only": {"value": W * H / (fwd_ms * 1e-3) / 1e6, "ms_per_step": fwd_ms},
           "adjoint_kernel_ms": adj_ms, "rows_this_rank": [band.y0, band.y1],
           "config": grid_config(), "parity": PARITY["grid_512"], "clocks": clk.summary(),
           "step_ms": [round(x, 4) for x in ms]}
    bpr = grid_bytes_per_ray()
    if bpr:
        rays_rank = W * (band.y1 - band.y0)
        peak, src = _hbm_peak()
        ach = bpr["adjoint"] * rays_rank / (adj_ms * 1e-3) / 1e9
        out["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                           "frac": ach / peak, "traffic": None, "peak_source": src,
                           "bytes_per_ray": bpr["adjoint"], "kernel": "k_grid_march<adjoint>",
                           "note": "algorithmic bytes (texels, LUT taps, atomic adds); the grid "
                                   "and gradient (16 MiB each) are L2-resident"}
    if with_e2e:
        h_vals = torch.from_numpy(np.ascontiguousarray(G)).pin_memory()
        h_grad = torch.empty_like(h_vals).pin_memory()
        h_acc = torch.empty(2, dtype=torch.float64).pin_memory()

        def e2e():
            P.values.copy_(h_vals, non_blocking=True)
            step()
            h_grad.copy_(P.grad, non_blocking=True)
            h_acc.copy_(P.acc, non_blocking=True)

        _, e2e_ms = B.timed(e2e)
        out["e2e"] = {"value": W * H / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
                      "h2d_bytes_per_step": h_vals.numel() * 4,
                      "d2h_bytes_per_step": h_grad.numel() * 4 + 16}
        out["_scene"] = sc
    sub.close()
    return out


def leg_layer_params(B: Bench, W=480, H=270):
    """d loss / d (coverage, shape_bias, detail_bias, density_scale, base_m,
    top_m) of the cumulus layer of the three-layer frame at W x H
    (psc_layer_param_gradient: the PLAIN march in forward mode with six
    tangents), the loss against the frame rendered with the layer's coverage
    0.04 higher.  Each rank computes the whole view (replicas)."""
    from pedalsky_b200 import capi, scenes
    from pedalsky_b200.capi import call
    from pedalsky_b200.layer_grad import layer_param_gradient
    from pedalsky_b200.subsystem import subsystem_for_scene
    torch = B.torch
    sc = scenes.precision_1080p(W, H, storage=capi.STORAGE_F32, schedule=capi.SCHED_PLAIN,
                                filt=capi.FILTER_EXACT)
    sc.params.diurnal_strength = 1.0
    sub = subsystem_for_scene(sc, device=B.ranks.local, luts=None)
    dev = B.dev
    bg = torch.from_numpy(np.ascontiguousarray(sc.background, np.float32)).to(dev)
    depth = torch.from_numpy(np.ascontiguousarray(sc.depth, np.float32)).to(dev)
    L = torch.zeros((H, W, 4), device=dev)
    T = torch.zeros_like(L)
    layers = (capi.CloudLayerGpu * 8).from_buffer_copy(sc.layers)
    layers[0].coverage += 0.04
    call("psc_set_layers", sub.handle, layers, sc.n_layers)
    view = capi.View(W, H, depth.data_ptr(), L.data_ptr(), T.data_ptr(), None)
    with torch.cuda.stream(B.stream):
        call("psc_render", sub.handle, C.byref(view), 1, B.sh())
    torch.cuda.synchronize()
    target = (L + bg * T).contiguous()
    call("psc_set_layers", sub.handle, sc.layers, sc.n_layers)
    grad = torch.zeros(6, dtype=torch.float64, device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    gview = capi.View(W, H, depth.data_ptr(), None, None, None)

    def step():
        grad.zero_()
        loss.zero_()
        layer_param_gradient(sub.handle, gview, 0, bg, target, grad, loss, stream=B.stream)

    clk = ClockSampler(B.ranks.local)
    ms, ms_max = B.timed(step, clk=clk, counter=sub.launch_count)
    out = {"value": W * H / (ms_max * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms_max,
           "gpu_launches": B.timed_launches, "scaling": "replicas",
           "config": {"workload": f"precision_1080p {W}x{H}, layer 0 (Cu), six parameters",
                      "schedule": "plain", "storage": "f32", "filter": "exact"},
           "gradient": [float(x) for x in grad.cpu().numpy()], "loss": float(loss.cpu().numpy()[0]),
           "parity": "tests/test_gpu_layer_params.py (FP64 branch-held central differences)",
           "clocks": clk.summary(), "step_ms": [round(x, 4) for x in ms]}
    sub.close()
    return out


def leg_passes(B: Bench, storage, schedule, filt, full_ms=None, W=1920, H=1080):
    """The passes around the march on the headline frame (W x H): the
    half-res frame (march into the floor(W/2) x floor(H/2) cloud RT, depth
    downsample, Catmull-Rom composite into the W x H target), the same with
    the TAA resolve, and alone the HBM-bound kernels (bytes per pixel over
    the device time against the HBM peak, the L2 flushed before each step):
    the Catmull-Rom composite (k_composite_halfres: the RT's L and T once, 8
    B per output pixel at 2x2, and the target read and written, 32 B), the
    TAA resolve of a W x H cloud RT (k_taa_resolve: current and history L/T
    read, resolve written, 96 B per pixel) and the full-res two-pass
    composite (k_composite: 64 B per pixel); then the per-frame atmosphere
    LUT bake (transmittance, multi-scatter, sky-view, aerial perspective) and
    the once-per-context noise bake by wall clock.  Each rank runs the same
    frame (replicas)."""
    import time
    from pedalsky_b200 import capi, scenes
    from pedalsky_b200.capi import call
    from pedalsky_b200.subsystem import subsystem_for_scene
    torch, dev, sh = B.torch, B.dev, B.sh()
    sc = scenes.precision_1080p(W, H, storage=storage, schedule=schedule, filt=filt)
    sub = subsystem_for_scene(sc, device=B.ranks.local, luts=None)
    bg = torch.from_numpy(np.ascontiguousarray(sc.background, np.float32)).to(dev)
    depth = torch.from_numpy(np.ascontiguousarray(sc.depth, np.float32)).to(dev)
    hdr = torch.empty_like(bg)
    rw, rh = C.c_uint32(), C.c_uint32()
    call("psc_cloud_rt_size", W, H, 1, C.byref(rw), C.byref(rh))
    rw, rh = rw.value, rh.value
    peak, src = _hbm_peak()
    out = {"config": {"workload": f"precision_1080p {W}x{H}, cloud RT {rw}x{rh} at half res",
                      "storage": B.args.storage, "schedule": B.args.schedule, "filter": B.args.filter,
                      "l2": "flushed before every step"},
           "parity": "tests/test_gpu_post.py, tests/test_gpu_march.py (half-res and TAA against the "
                     "FP64 restatements of the composite and the resolve)"}
    o0 = capi.MarchOptions.from_buffer_copy(sub.options)
    view = capi.View(W, H, depth.data_ptr(), None, None, hdr.data_ptr())

    def frame_leg(half_res, taa):
        o = capi.MarchOptions.from_buffer_copy(o0)
        o.composite, o.half_res, o.taa = 1, half_res, taa
        sub.set_options(o)
        call("psc_invalidate_taa_history", sub.handle)
        clk = ClockSampler(B.ranks.local)
        ms, ms_max = B.timed(lambda: (hdr.copy_(bg, non_blocking=True),
                                      call("psc_render", sub.handle, C.byref(view), 1, sh)),
                             clk=clk, counter=sub.launch_count)
        r = {"ms_per_step": ms_max, "Mpixels_per_s": W * H / (ms_max * 1e-3) / 1e6,
             "march_rays_per_step": rw * rh if half_res else W * H,
             "gpu_launches": B.timed_launches, "clocks": clk.summary(),
             "step_ms": [round(x, 4) for x in ms]}
        if full_ms:
            r["speedup_vs_full_res_frame"] = full_ms / ms_max
        return r

    out["half_res_frame"] = frame_leg(1, 0)
    out["half_res_taa_frame"] = frame_leg(1, 1)
    sub.set_options(o0)

    def hbm_leg(kernel, step, bytes_per_step, launches):
        clk = ClockSampler(B.ranks.local)
        ms, ms_max = B.timed(step, clk=clk)
        ach = bytes_per_step / (ms_max * 1e-3) / 1e9
        return {"kernel": kernel, "ms_per_step": ms_max, "gpu_launches": launches * B.args.steps,
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                             "frac": ach / peak, "traffic": None, "peak_source": src,
                             "bytes_per_step": bytes_per_step},
                "clocks": clk.summary(), "step_ms": [round(x, 4) for x in ms]}

    rl = torch.rand((rh, rw, 4), device=dev)
    rt = torch.rand((rh, rw, 4), device=dev)
    out["composite_halfres"] = hbm_leg(
        "k_composite_halfres",
        lambda: call("psc_composite_halfres", C.c_void_p(rl.data_ptr()), C.c_void_p(rt.data_ptr()),
                     rw, rh, C.c_void_p(hdr.data_ptr()), W, H, sh),
        rw * rh * 32 + W * H * 32, 1)
    del rl, rt
    cl = torch.rand((H, W, 4), device=dev)
    ct = torch.rand((H, W, 4), device=dev)
    call("psc_invalidate_taa_history", sub.handle)
    with torch.cuda.stream(B.stream):  # the first resolve after an invalidate bootstraps
        call("psc_taa_resolve", sub.handle, C.c_void_p(cl.data_ptr()), C.c_void_p(ct.data_ptr()), W, H,
             None, None, sh)
    torch.cuda.synchronize()
    out["taa_resolve"] = hbm_leg(
        "k_taa_resolve",
        lambda: call("psc_taa_resolve", sub.handle, C.c_void_p(cl.data_ptr()), C.c_void_p(ct.data_ptr()),
                     W, H, None, None, sh),
        W * H * 96, 1)
    out["composite"] = hbm_leg(
        "k_composite",
        lambda: call("psc_composite", C.c_void_p(cl.data_ptr()), C.c_void_p(ct.data_ptr()),
                     C.c_void_p(hdr.data_ptr()), W, H, sh),
        W * H * 64, 1)
    del cl, ct

    clk = ClockSampler(B.ranks.local)
    ms, ms_max = B.timed(lambda: call("psc_bake_luts", sub.handle, sh), clk=clk, counter=sub.launch_count)
    out["lut_bake"] = {"ms_per_step": ms_max, "gpu_launches": B.timed_launches, "bound": "ALU, once per frame",
                       "luts": "transmittance 256x64, multi-scatter 32x32, sky-view 192x108, "
                               "aerial perspective 32x32x64",
                       "clocks": clk.summary(), "step_ms": [round(x, 4) for x in ms]}
    walls = []
    for i in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call("psc_bake_noise", sub.handle)
        torch.cuda.synchronize()
        if i:
            walls.append(1e3 * (time.perf_counter() - t0))
    out["noise_bake"] = {"wall_ms": float(np.median(walls)), "bound": "ALU, once per context",
                         "note": "base 128^3 RGBA8, detail 32^3, curl 128^2, their storage forms and "
                                 "folds, and the host blue-noise tile; median of 3 after one"}
    sub.close()
    return out


def _hbm_peak():
    hbm = measured_peaks().get("hbm_gbs")
    return (hbm, "measured (MEASURED_PEAKS.json)") if hbm else (6650.0, "fallback")


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


def run_frames(args, ranks: Ranks):
    """Frame workloads (the default): the headline frame and the extras."""
    from pedalsky_b200 import capi, scenes
    from pedalsky_b200.capi import call
    from pedalsky_b200.subsystem import subsystem_for_scene

    B = Bench(args, ranks)
    torch, dev = B.torch, B.dev
    storage = capi.STORAGE_NAMES[args.storage]
    schedule = capi.SCHED_FAST if args.schedule == "fast" else capi.SCHED_PLAIN
    filt = capi.FILTER_NAMES[args.filter]
    wl = args.workload
    (dw, dh), n_frames, desc = FRAME_WORKLOADS[wl]
    W, H = args.width or dw, args.height or dh
    # each rank renders its own frame(s) of the sequence (weak scaling)
    frames = frame_scenes(wl, W, H, storage=storage, schedule=schedule, filt=filt)
    for f in frames:
        f.frame.frame_index += ranks.rank * n_frames
    s = frames[0]
    sub = subsystem_for_scene(s, device=ranks.local, luts=None)  # noise + LUTs baked on the device
    sh = B.sh()
    stream = B.stream

    L = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    T = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    bg = torch.from_numpy(s.background).to(dev)
    hdr = torch.empty_like(bg)
    depth = torch.from_numpy(s.depth).to(dev)
    o = capi.MarchOptions.from_buffer_copy(sub.options)
    o.composite = 1
    sub.set_options(o)
    view = capi.View(W, H, depth.data_ptr(), L.data_ptr(), T.data_ptr(), hdr.data_ptr())
    kev = []

    def render_step():
        """One step: every frame of the workload (the frames differ only in
        simulated time, so the sky-view and AP LUTs stay valid); the march
        launch itself is bracketed by its own events for the roofline."""
        for f in frames:
            if n_frames > 1:
                call("psc_set_frame", sub.handle, C.byref(f.frame), C.byref(f.world))
            hdr.copy_(bg, non_blocking=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call("psc_render", sub.handle, C.byref(view), 1, sh)
            e1.record(stream)
            kev.append((e0, e1))

    peaks_fetch = None
    try:
        peaks_fetch = fetch_peaks(ranks.local)
    except Exception as e:  # reported with the roofline, never required
        print(f"fetch-peak calibration failed: {e}", file=sys.stderr)
    clk = ClockSampler(ranks.local)
    step_ms, ms_max = B.timed(render_step, clk=clk, kernel_events=kev, counter=sub.launch_count)
    kernel_launches = B.timed_launches
    kernel_ms = float(np.mean([a.elapsed_time(b) for a, b in kev])) if kev else None
    rays_step = n_frames * W * H
    value = ranks.world * rays_step / (ms_max * 1e-3) / 1e6

    # the fetches the timed kernel issues on this frame (instrumented build)
    counts = None
    if schedule == capi.SCHED_FAST and args.storage in ("f16", "u8") and args.filter != "texture":
        fc = capi.FetchCounts()
        with torch.cuda.stream(stream):
            hdr.copy_(bg)
            call("psc_count_fetches", sub.handle, C.byref(view), C.byref(fc), sh)
        counts = fc.as_dict()

    # the plain FP32-storage drop-in kernel on the same frame, for the ratio
    plain = None
    if not args.no_plain_reference:
        o_plain = capi.MarchOptions.from_buffer_copy(o)
        o_plain.schedule, o_plain.storage, o_plain.filter = (capi.SCHED_PLAIN, capi.STORAGE_F32,
                                                             capi.FILTER_EXACT)
        sub.set_options(o_plain)
        _, ms_plain = B.timed(render_step)
        sub.set_options(o)
        plain = {"value": ranks.world * rays_step / (ms_plain * 1e-3) / 1e6,
                 "ms_per_step": ms_plain, "config": "plain schedule, f32 storage, exact filtering"}

    # the same frames through psc_render_batch (the autotuner's form,
    # replayed from a CUDA graph; the frame is static, so its sky-view / AP
    # LUTs are baked once, before the timed steps)
    batched = None
    if not args.no_plain_reference and schedule == capi.SCHED_FAST:
        from pedalsky_b200 import batch as Bt
        bt = Bt.Batch(frames, dev)
        with torch.cuda.stream(stream):
            btune = Bt.autotune(sub.handle, bt, reps=1, stream=stream)
        Bt.set_tuning(sub.handle, btune["threads"], btune["tile_w"], use_graph=1,
                      form=btune["form_id"])
        _, ms_b = B.timed(lambda: bt.render(sub.handle, stream), pre=bt.reset_hdr)
        batched = {"value": ranks.world * rays_step / (ms_b * 1e-3) / 1e6, "ms_per_step": ms_b,
                   "config": "psc_render_batch in the autotuner's form and light-march batch, "
                             "replayed from a captured CUDA graph; per-view LUT bakes only when "
                             "a view's camera or sun changed (none in the timed steps)",
                   "autotuned": btune}
        del bt
        sub.set_options(o)  # the autotuner keeps its light-march batch in the options

    row_bands = None
    if n_frames == 1 and not args.no_legs:
        row_bands = leg_row_bands(B, sub, s, depth, bg)

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
                    B.flush.zero_()  # L2 evicted once per step, as in the device-timed run
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
    ranks.barrier()
    e2e_ms = ranks.max(e2e_pass(args.steps), dev)
    e2e_value = ranks.world * rays_step / (e2e_ms * 1e-3) / 1e6
    h2d = n_frames * (h_bg.numel() * 4 + h_depth.numel() * 4)
    d2h = n_frames * slots[0]["out"].numel() * 4
    sub.close()

    legs = {}
    if wl == WORKLOAD and not args.no_legs and schedule == capi.SCHED_FAST:
        want = set(args.legs.split(",")) if args.legs != "all" else None
        for name, run in (("batch_64", lambda: leg_batch64(B, storage, filt)),
                          ("stress_2160p", lambda: leg_stress(B, storage, schedule, filt)),
                          ("grid_512", lambda: leg_grid(B)),
                          ("layer_params_480x270", lambda: leg_layer_params(B)),
                          ("passes_1080p", lambda: leg_passes(B, storage, schedule, filt, full_ms=ms_max))):
            if want is None or name in want:
                legs[name] = run()

    if ranks.rank == 0:
        roof = roofline(args, wl, W, H, W * H, kernel_ms, peaks_fetch, counts, batched, rays_step)
        cpu = None
        if not args.no_cpu_baseline and ranks.world == 1:
            try:
                cpu = cpu_baseline(s, 64 if wl == WORKLOAD else 32)
            except Exception as e:  # the baseline is reported, never the product
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                       "sample": f"failed: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ranks.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded reference noise hash, reference synthesis)",
            "config": workload_config(wl, W, H),
            "form": {"storage": args.storage, "schedule": args.schedule, "filter": args.filter,
                     "composite": "fused", "parallelism": f"frames{ranks.world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "pipeline": "per frame: pinned H2D, march + composite, D2H on three "
                                "streams, two device slots"},
            "gpu_launches": kernel_launches,
            "library": {"path": capi.LIB_PATH.name, "build_id": capi.lib().psc_build_id().decode()},
            "kernel_ms": kernel_ms,
            "roofline": roof,
            "fetch_counts": counts,
            "parity": PARITY.get(wl),
            "plain_fp32_dropin": plain,
            "speedup_vs_plain_fp32": (value / plain["value"]) if plain else None,
            "batched_fp16": batched,
            "batched_speedup_vs_plain_fp32": (batched["value"] / plain["value"])
            if (batched and plain) else None,
            "row_bands": row_bands,
            "legs": legs or None,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "step_ms": [round(x, 4) for x in step_ms],
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def roofline(args, wl, W, H, rays, kernel_ms, peaks_fetch, counts, batched, rays_step):
    """The timed kernel against the ceiling that bounds it (`rays` per launch
    of it; `rays_step` per step, for the batched form's whole-step rate).  The march's
    working set (folded volumes, LUTs, weather) is L2-resident, so its
    fetches are served on chip: the ceiling is the L2 read bandwidth
    measured on this GPU in this run.  `achieved` counts the algorithmic
    bytes (the reference algorithm's executed fetches); `fetched_*` counts
    what the kernel requests (its instrumented build's tally); `hbm` is the
    DRAM traffic from the ncu capture of the same command against the
    measured copy bandwidth."""
    if not kernel_ms:
        return None
    alg = bytes_per_ray(args.storage, args.schedule, wl)
    ncu = NCU_KERNEL.get((wl, args.schedule, args.storage, args.filter, W, H), {})
    out = {"kernel": "k_march_fast" if args.schedule == "fast" else "k_march_plain",
           "kernel_ms": kernel_ms, "unit": "GB/s"}
    if peaks_fetch:
        l2 = peaks_fetch["l2_read_gbs"]
        out.update({"bound": "l2_fetch", "peak": l2,
                    "peak_source": "psc_measure_fetch_peaks: L2 read bandwidth of this GPU, "
                                   "this run"})
    else:
        hbm, src = _hbm_peak()
        out.update({"bound": "hbm", "peak": hbm, "peak_source": src,
                    "note": "the on-chip calibration failed; HBM copy peak as the ceiling"})
    if alg:
        out["bytes_per_ray"] = alg["bytes_per_ray"]
        out["achieved"] = alg["bytes_per_ray"] * rays / (kernel_ms * 1e-3) / 1e9
        out["frac"] = out["achieved"] / out["peak"]
    if counts:
        fb = fetched_bytes_per_ray(counts, args.storage, args.schedule)
        out["fetched_bytes_per_ray"] = fb["bytes_per_ray"]
        out["fetched_achieved"] = fb["bytes_per_ray"] * rays / (kernel_ms * 1e-3) / 1e9
        out["fetched_frac"] = out["fetched_achieved"] / out["peak"]
        out["fetched"] = fb
    out["traffic"] = ncu.get("traffic")
    out["issue_active"] = ncu.get("issue_active")
    if ncu:
        out["binding_limit"] = "SM issue slots (ncu smsp__issue_active of this kernel)"
    hbm, src = _hbm_peak()
    if ncu.get("traffic"):
        dram = ncu["traffic"] / (kernel_ms * 1e-3) / 1e9
        out["hbm"] = {"dram_gbs": dram, "peak": hbm, "peak_source": src, "frac": dram / hbm}
    if peaks_fetch:
        out["fetch"] = {
            "l1_read_peak_gbs": peaks_fetch["l1_read_gbs"],
            "tex_trilinear_peak_gfetch_s": peaks_fetch["tex_trilinear_gfetch_s"]}
        if alg:
            out["fetch"]["frac_of_l1_read"] = out["achieved"] / peaks_fetch["l1_read_gbs"]
            light = alg["light_fetches_per_ray"] * rays / (kernel_ms * 1e-3) / 1e9
            out["fetch"]["light_march_gfetch_s"] = light
            out["fetch"]["frac_of_tex_trilinear"] = light / peaks_fetch["tex_trilinear_gfetch_s"]
        if alg and batched:
            b_ach = alg["bytes_per_ray"] * rays_step / (batched["ms_per_step"] * 1e-3) / 1e9
            batched["fetch_gbs"] = b_ach
            batched["frac_of_l2_read"] = b_ach / peaks_fetch["l2_read_gbs"]
    return out


def run_batch(args, ranks: Ranks):
    """64 uneven views with their own scenes: the c3 leg as the headline."""
    from pedalsky_b200 import capi
    B = Bench(args, ranks)
    leg = leg_batch64(B, capi.STORAGE_NAMES[args.storage], capi.FILTER_NAMES[args.filter],
                      args.batch_views)
    if ranks.rank == 0:
        line = {
            "metric": METRIC, "value": leg["value"], "unit": UNIT, "n_gpus": ranks.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random scenes per view, reference synthesis)",
            "config": {"workload": f"batch_{args.batch_views} uneven views",
                       "rays_per_step": leg["rays_per_step"], "l2": L2_NOTE},
            "form": {"storage": args.storage, "filter": args.filter, "schedule": "fast",
                     "launch": leg["config"], "autotuned": leg["autotuned"]},
            "e2e": None, "gpu_launches": leg["gpu_launches"], "parity": leg["parity"],
            "clocks": leg["clocks"], "step_ms": leg["step_ms"],
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def run_grid(args, ranks: Ranks):
    """The differentiable form as the headline (c4)."""
    B = Bench(args, ranks)
    leg = leg_grid(B, with_e2e=True)
    sc = leg.pop("_scene")
    if ranks.rank == 0:
        cpu = None
        if not args.no_cpu_baseline and ranks.world == 1:
            from oracle import pyoracle
            noise = pyoracle.bake_noise()
            luts = pyoracle.bake_luts(sc.frame, sc.world)
            runs = [grid_cpu_sample(sc, noise, luts, 128) for _ in range(5)]
            secs = float(np.median([r[1] for r in runs]))
            cpu = {"value": runs[0][0] / secs / 1e6, "unit": UNIT, "cores": runs[0][2],
                   "kind": "port", "sample": f"{runs[0][0]} rays (4 row bands), FP64 forward + "
                                             f"reverse sweep, median of 5: {secs:.2f} s"}
        line = {
            "metric": GRID_METRIC, "value": leg["value"], "unit": UNIT, "n_gpus": ranks.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Worley grid; target = render of the grid with 5% noise)",
            "config": grid_config(),
            "form": {"parallelism": f"rowbands{ranks.world} + all-reduce"},
            "forward_only": leg["forward_only"], "adjoint_kernel_ms": leg["adjoint_kernel_ms"],
            "e2e": leg["e2e"], "gpu_launches": leg["gpu_launches"],
            "roofline": leg.get("roofline"), "cpu_baseline": cpu, "parity": leg["parity"],
            "clocks": leg["clocks"], "step_ms": leg["step_ms"],
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def run_stress(args, ranks: Ranks):
    """Eight 4K frames as the headline (c5), frames split over the ranks."""
    from pedalsky_b200 import capi
    B = Bench(args, ranks)
    leg = leg_stress(B, capi.STORAGE_NAMES[args.storage],
                     capi.SCHED_FAST if args.schedule == "fast" else capi.SCHED_PLAIN,
                     capi.FILTER_NAMES[args.filter])
    if ranks.rank == 0:
        line = {
            "metric": METRIC, "value": leg["value"], "unit": UNIT, "n_gpus": ranks.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded coverage grid, reference synthesis)",
            "config": workload_config("stress_2160p", 3840, 2160),
            "form": {"storage": args.storage, "schedule": args.schedule, "filter": args.filter,
                     "composite": "fused", "parallelism": f"frames split over {ranks.world}"},
            "e2e": None, "gpu_launches": leg["gpu_launches"], "parity": leg["parity"],
            "clocks": leg["clocks"], "step_ms": leg["step_ms"],
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args)
    ranks = Ranks()
    if ranks.world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but the launch has WORLD_SIZE={ranks.world} ranks")
    if args.workload == "batch_64":
        return run_batch(args, ranks)
    if args.workload == "grid_512":
        return run_grid(args, ranks)
    if args.workload == "stress_2160p" and args.width is None:
        return run_stress(args, ranks)
    return run_frames(args, ranks)


if __name__ == "__main__":
    sys.exit(main())
