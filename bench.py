#!/usr/bin/env python3
"""Benchmark of the B200 analysis path.

Workload: one 4032x3024 8-bit sRGB image from the seeded synthetic generator
(1/f^alpha colour noise, gradients, blobs, 0-40 hard-edged polygons, random
saturation, Gaussian sensor noise sigma in [0.5, 3] DN), distance 1.0,
effort 7. A step is one pass of the whole analysis half over that image:
sRGB -> XYB, quantization-matrix statistics, initial quant field, inverse
Gaborish, initial CfL, AC-strategy costs and greedy merge, forward
transforms, and the adaptive-quantization loop (three evaluations, each with
quantizer, final CfL, AC/DC quantization, decoder-equivalent
reconstruction, Gaborish + EPF, Butteraugli and per-transform reduction, and
two field updates), then the coefficient-order populations and scans and the
AC tokens with their histogram. The metric is megapixels per second (source
pixels).

`value` is measured with the input already in device memory, in each
session's own input buffer (CUDA events around K steps). `e2e` runs the same steps through
gjxl_b200_session_analyze_host: host->device copy of the packed pixels from
pinned memory, the analysis, and device->host copies of the results, all
inside the timed region.

Each GPU runs `--sessions` analysis sessions (default 3) on their own
streams, as a serving process with several images in flight would: step i
goes to session i mod S, so one image's latency-bound phases and host
copies overlap another image's compute. For `e2e` every session is driven by
its own host thread (the host-input call waits for its results). K steps
are K images in total; the events bracket all of them.

`--impl reference` times the reference's own CPU implementation of the same
analysis (compiled from its sources into oracle/_ref) on the host cores: the
reference analyses one image on one thread (its Butteraugli and AC search are
serial), so every host core analyses its own 512x512 crop of the workload
image in parallel and the metric is the crops' megapixels per wall second.

`--launch-list` runs only the warm-up and K device-resident steps (no e2e,
no stage profile, no CPU leg, no clock sampling) for an ncu launch list.

Multi-GPU: images are independent, so N GPUs run N independent replicas (one
image each per step, no collective); value = N images' megapixels / max-rank
time.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT = 4032, 3024
SEED = 2_000_000  # configuration 2, image 0
METRIC = "Megapixels/s analysis stage (e7, d1.0)"
WORKLOAD = ("analysis half of one 4032x3024 synthetic sRGB image at d1.0 e7: sRGB->XYB, "
            "matrix stats, initial AQ field, inverse Gaborish, initial CfL, AC-strategy costs "
            "+ greedy merge, forward transforms, 3 AQ evaluations (quantizer, final CfL, AC/DC "
            "quantization, reconstruction, Gaborish+EPF, Butteraugli, block reduction) with 2 "
            "field updates, then coefficient-order populations/scans and AC tokens")


def load_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return {**json.loads(path.read_text()), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        query = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={query}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def wait_ready(self, timeout_s: float = 5.0) -> None:
        """Blocks until nvidia-smi has written its first sample, so that the
        timed region that follows is sampled from its start."""
        deadline = time.monotonic() + timeout_s
        while self.proc is not None and time.monotonic() < deadline:
            self.file.flush()
            if Path(self.file.name).stat().st_size > 0:
                return
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.flush()
        rows = [line.split(",") for line in Path(self.file.name).read_text().splitlines()
                if line.strip()]
        os.unlink(self.file.name)
        clocks = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().isdigit()]
        maxes = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(clocks) if clocks else None,
                "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(clocks)}


def make_image() -> np.ndarray:
    from gjxl_b200.synthetic import generate_srgb8
    return generate_srgb8(WIDTH, HEIGHT, SEED, sensor_noise=True)


def dist_setup(gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    # NCCL reduces device tensors; the gloo group of the CPU tests host ones.
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# Families searched per 64x64 tile (ac_strategy_search_policy.h:21-29): pixel
# extent (W, H), covered blocks and anchor step.
FAMILIES = [(8, 8, 1, 1, 1), (8, 16, 1, 2, 1), (16, 8, 2, 1, 1), (16, 16, 2, 2, 1),
            (16, 32, 2, 4, 2), (32, 16, 4, 2, 2), (32, 32, 4, 4, 2)]


def candidate_cost_fp64_ops(blocks_x: int, blocks_y: int) -> int:
    """Algorithmic FP64 operations of the candidate-cost kernels for one
    image: every candidate transforms 3 channels forward and back, each
    separable DCT costs (W + H) multiply-adds per coefficient, and the
    bit-exact restatement rounds every multiply and every add separately
    (2 FP64 operations per multiply-add)."""
    total = 0
    for w, h, cw, ch, step in FAMILIES:
        anchors = 0
        for ty in range(0, blocks_y, 8):
            for tx in range(0, blocks_x, 8):
                tw, th = min(8, blocks_x - tx), min(8, blocks_y - ty)
                nx = len([x for x in range(0, 8 - cw + 1, step) if x + cw <= tw])
                ny = len([y for y in range(0, 8 - ch + 1, step) if y + ch <= th])
                anchors += nx * ny
        total += anchors * 3 * 2 * (w * h) * (w + h) * 2
    return total


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the seven
# candidate-cost launches of one analysis: 354.57 MB measured by ncu on the
# 2048x1536 image of the same generator, scaled by the pixel ratio to
# 4032x3024 (each launch reads the three XYB planes and the pixel mask once,
# 16 B per pixel, so traffic grows with the image area).
COST_KERNEL_DRAM_BYTES = round(354_570_240 * (4032 * 3024) / (2048 * 1536))


def fp64_peak_tflops(stream: int) -> float:
    """FP64 multiply/add throughput of this GPU (TFLOP/s, one DMUL or DADD =
    one operation), measured by the library's calibration kernel."""
    import ctypes
    import torch
    from gjxl_b200 import _lib
    sink = torch.zeros(1, dtype=torch.float64, device="cuda")
    ops = ctypes.c_double()
    _lib.call("gjxl_b200_fp64_throughput", sink.data_ptr(), ctypes.byref(ops), stream)
    return ops.value / 1e12


def d2h_bytes(session) -> int:
    """Bytes the host-input entry point copies back per analysis: block maps
    (strategy cells, initial and final quant fields, raw quant field, DC), CfL
    maps, statistics, error words, score history, quantizer, group offsets and
    the AC tokens (4-byte values, 2-byte contexts)."""
    o = session.outputs
    blocks, tiles = o.blocks_x * o.blocks_y, o.tiles_x * o.tiles_y
    return (blocks * (1 + 4 + 4 + 4 + 12) + 2 * tiles + 12 + 12 + 8 * (o.iterations + 1) + 40
            + 4 * (o.groups + 1) + 6 * o.host_token_count)


def run_gpu(args) -> dict:
    import torch
    from gjxl_b200.session import AnalysisSession

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    img = make_image()
    count = 1 if args.launch_list else max(1, args.sessions)
    precision = 1 if args.precision == "fast" else 0
    sessions = [AnalysisSession(WIDTH, HEIGHT, butteraugli_target=1.0, effort=7,
                                precision=precision) for _ in range(count)]
    session = sessions[0]
    main_stream = torch.cuda.current_stream()
    stream = main_stream.cuda_stream
    side = [torch.cuda.Stream() for _ in range(count)]
    d_img = torch.from_numpy(img.reshape(HEIGHT, -1)).cuda()
    pinned = torch.from_numpy(img).pin_memory()
    pinned_np = pinned.numpy()
    row = WIDTH * 3

    # The image resident in each session's own input buffer (packed rows).
    import ctypes
    for sess in sessions:
        ctypes.CDLL("libcudart.so.12").cudaMemcpy(
            ctypes.c_void_p(sess.outputs.input_pixels), ctypes.c_void_p(d_img.data_ptr()),
            ctypes.c_size_t(row * HEIGHT), 3)  # device to device
    torch.cuda.synchronize()
    resident = [sess.outputs.input_pixels for sess in sessions]

    if args.launch_list:
        for _ in range(args.warmup):
            session.analyze(resident[0], row, 3, stream)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            session.analyze(resident[0], row, 3, stream)
        torch.cuda.synchronize()
        session.close()
        return {}
    # Warm-up (and each session's graph capture) one session at a time.
    for i, sess in enumerate(sessions):
        for _ in range(args.warmup):
            sess.analyze(resident[i], row, 3, side[i].cuda_stream)
        torch.cuda.synchronize()

    def fork(start_event):
        for st in side:
            st.wait_event(start_event)

    def join(stop_event):
        for st in side:
            done = torch.cuda.Event()
            done.record(st)
            main_stream.wait_event(done)
        stop_event.record(main_stream)

    # Device-resident throughput: step i on session i mod S.
    barrier(world)
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler is not None:
        sampler.wait_ready()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(main_stream)
    fork(start)
    for i in range(args.steps):
        sessions[i % count].analyze(resident[i % count], row, 3, side[i % count].cuda_stream)
    join(stop)
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop), world) / args.steps
    mp = WIDTH * HEIGHT / 1e6
    value = world * mp / (ms / 1e3)

    # End to end through the host-input entry point, one host thread per
    # session (each call returns once its results are on the host).
    import threading
    for i, sess in enumerate(sessions):
        for _ in range(max(1, args.warmup // 2)):
            sess.analyze_host(pinned_np, side[i].cuda_stream)
    torch.cuda.synchronize()
    barrier(world)
    start.record(main_stream)
    fork(start)
    shares = [args.steps // count + (1 if i < args.steps % count else 0) for i in range(count)]
    failures = []

    def drive(i):
        try:
            for _ in range(shares[i]):
                sessions[i].analyze_host(pinned_np, side[i].cuda_stream)
        except Exception as exc:  # reported after the join
            failures.append(exc)

    threads = [threading.Thread(target=drive, args=(i,)) for i in range(count)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if failures:
        raise failures[0]
    join(stop)
    torch.cuda.synchronize()
    # The clock samples span both timed regions (device-resident and end to
    # end) and the untimed host-input warm-up between them.
    clocks = sampler.stop() if sampler else None
    e2e_ms = max_over_ranks(start.elapsed_time(stop), world) / args.steps
    for sess in sessions:
        assert sess.host_error() == 0, "device error word set"

    # Per-stage times and the dominant kernel's roofline (separate session so
    # the timed region above carries no event records).
    prof = AnalysisSession(WIDTH, HEIGHT, butteraugli_target=1.0, effort=7, profile_stages=True,
                           precision=precision)
    stage_ms = {}
    reps = max(3, min(args.steps, 10))
    for _ in range(reps):
        prof.analyze(d_img.data_ptr(), row, 3, stream)
        torch.cuda.synchronize()
        for k, v in prof.stage_times().items():
            stage_ms[k] = stage_ms.get(k, 0.0) + v / reps
    prof.close()

    o = prof.outputs
    cost_ms = stage_ms.get("ac_strategy_costs", float("nan"))
    fp64_ops = candidate_cost_fp64_ops(o.blocks_x, o.blocks_y)
    achieved = fp64_ops / (cost_ms / 1e3) / 1e12
    peak = fp64_peak_tflops(stream)
    launches = session.kernel_count(d_img.data_ptr(), row, 3)
    result = {
        "metric": METRIC, "value": round(value, 3), "unit": "MP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": WORKLOAD, "width": WIDTH, "height": HEIGHT, "distance": 1.0,
                   "effort": 7, "seed": SEED, "precision": args.precision,
                   "parallelism": f"replicas x{world}, {count} concurrent sessions per GPU",
                   "l2": "working set (~0.6 GB of planes) exceeds the 126 MB L2"},
        "e2e": {"value": round(world * mp / (e2e_ms / 1e3), 3), "unit": "MP/s",
                "ms_per_step": round(e2e_ms, 4),
                "h2d_bytes_per_step": WIDTH * HEIGHT * 3,
                "d2h_bytes_per_step": d2h_bytes(session)},
        "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "gpu_launches": args.steps * launches,
        "roofline": {
            "kernel": "CandidateCostKernel<W,H> (7 transform families, one launch each)",
            "bound": "fp64",
            "achieved": round(achieved, 3),
            "peak": round(peak, 3),
            "unit": "TFLOP/s (FP64, multiply and add rounded and counted separately)",
            "frac": round(achieved / peak, 4),
            "traffic": COST_KERNEL_DRAM_BYTES,
            "algorithmic_ops": fp64_ops,
            "peak_source": ("measured live: gjxl_b200_fp64_throughput (independent DMUL/DADD "
                            "chains on every SM); MEASURED_PEAKS.json has no FP64 figure"),
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum summed over "
                               "the 7 family launches, captured at 2048x1536 and scaled by "
                               "the pixel ratio; algorithmic bytes are 16 B/px per launch "
                               "(1.366 GB)"),
        },
        "clocks": clocks,
    }
    for sess in sessions:
        sess.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return result if rank == 0 else {}


CROP_W, CROP_H = 512, 512


def reference_crops(count: int) -> list[tuple[int, int]]:
    """Top-left corners of `count` 512x512 crops tiling the workload image."""
    cols, rows = WIDTH // CROP_W, HEIGHT // CROP_H
    return [((i % (cols * rows)) % cols * CROP_W, (i % (cols * rows)) // cols * CROP_H)
            for i in range(count)]


_worker_image = None


def _reference_worker(corner: tuple[int, int]) -> float:
    """One crop through the reference's CPU analysis half, as its workflow
    runs it for d1.0 e7 (RunCpuQuantizationPipeline). Returns seconds."""
    global _worker_image
    from oracle import ref
    if _worker_image is None:
        _worker_image = make_image()
    x, y = corner
    crop = np.ascontiguousarray(_worker_image[y:y + CROP_H, x:x + CROP_W])
    t0 = time.perf_counter()
    lin = ref.srgb8_to_linear(crop)
    opsin = ref.linear_to_padded_opsin(lin)
    stats = ref.matrix_scale_stats(opsin, CROP_W, CROP_H)
    xs, bs = ref.select_matrix_scales(stats, 1.0)
    ref.quantization_pipeline(lin, opsin, 1.0, 7, xs, bs)
    return time.perf_counter() - t0


class ReferencePool:
    """One process per host core (spawned before any GPU work), each running
    the reference on its own crop."""

    def __init__(self, workers: int | None = None):
        import multiprocessing as mp
        self.workers = workers or min(os.cpu_count() or 1, 64)
        self.pool = mp.get_context("spawn").Pool(self.workers)

    def step(self) -> float:
        """All workers analyse one crop each; returns wall seconds."""
        t0 = time.perf_counter()
        self.pool.map(_reference_worker, reference_crops(self.workers), chunksize=1)
        return time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def run_reference(args) -> dict:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return {}
    pool = ReferencePool()
    for _ in range(args.warmup):
        pool.step()
    times = [pool.step() for _ in range(args.steps)]
    pool.close()
    mp = pool.workers * CROP_W * CROP_H / 1e6
    value = mp / statistics.mean(times)
    sample = f"{pool.workers} parallel 512x512 crops of the workload image per step"
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "MP/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.mean(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": WORKLOAD, "width": WIDTH, "height": HEIGHT, "distance": 1.0,
                   "effort": 7, "seed": SEED, "parallelism": "host CPU processes",
                   "sample": (f"bounded sample of the workload: each step analyses "
                              f"{pool.workers} different {CROP_W}x{CROP_H} crops of the "
                              f"{WIDTH}x{HEIGHT} image, one per host core (one 12 MP "
                              f"image takes the reference minutes); MP/s counts the crops' "
                              f"pixels")},
        "cpu_baseline": {"value": round(value, 4), "unit": "MP/s", "cores": pool.workers,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "MP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def reference_gpu_leg(samples: int = 5, warmup: int = 2) -> dict:
    """The reference's own CUDA path on this GPU (its gjxl_cuda sources built
    for sm_100a into oracle/_ref/libgjxl_ref_cuda.so), as its
    cuda_encoding_benchmark runs it: fully-resident adaptive quantization,
    d1.0 e7, the same image. MP/s of the workflow's analysis phase
    (quantization_pipeline), median of `samples` encodes, one image at a
    time (the reference runs one encode per CUDA backend)."""
    from oracle import ref
    if not ref.cuda_available():
        return {"unavailable": "oracle/_ref/libgjxl_ref_cuda.so not built"}
    linear = ref.srgb8_to_linear(make_image())
    for _ in range(warmup):
        ref.cuda_encode(linear, 1.0, 7)
    runs = [ref.cuda_encode(linear, 1.0, 7) for _ in range(samples)]
    analysis = statistics.median(r["analysis_ms"] for r in runs)
    total = statistics.median(r["total_ms"] for r in runs)
    mp = WIDTH * HEIGHT / 1e6
    return {"value": round(mp / (analysis / 1e3), 3), "unit": "MP/s",
            "analysis_ms": round(analysis, 3), "encode_ms": round(total, 3),
            "codestream_bytes": len(runs[-1]["codestream"]), "score": runs[-1]["score"],
            "kind": "reference CUDA path (sm_100a build of its gjxl_cuda sources), "
                    "fully-resident AQ, quantization_pipeline phase, one image at a time",
            "samples": samples}


def cpu_baseline_leg(pool: "ReferencePool") -> dict:
    """About 15 s of reference CPU work on all host cores (one step)."""
    pool.step()  # first step loads the library in every worker
    seconds = pool.step()
    mp = pool.workers * CROP_W * CROP_H / 1e6
    return {"value": round(mp / seconds, 4), "unit": "MP/s", "cores": pool.workers,
            "kind": "reference",
            "sample": f"{pool.workers} parallel 512x512 crops of the workload image, one step"}


# Batched form: 64 images of the seeded generator, width and height
# log-uniform in [256, 4096] with aspect ratio in [0.5, 2], distance uniform in
# [0.5, 3.0], effort 7 (the batched configuration, seeds workload_seed(4, i)).
BATCH_IMAGES = 64


def batch_specs(count: int = BATCH_IMAGES) -> list[tuple[int, int, float, int]]:
    """(width, height, distance, seed) of each image of the batch."""
    from gjxl_b200.synthetic import workload_seed
    rng = np.random.default_rng(workload_seed(4, 999_999))
    specs = []
    for i in range(count):
        w = int(round(np.exp(rng.uniform(np.log(256), np.log(4096)))))
        lo, hi = max(256, w / 2), min(4096, 2 * w)
        h = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        specs.append((w, h, float(rng.uniform(0.5, 3.0)), workload_seed(4, i)))
    return specs


def _batch_image(spec) -> np.ndarray:
    from gjxl_b200.synthetic import generate_srgb8
    w, h, _, seed = spec
    return generate_srgb8(w, h, seed)


class BatchImages:
    """Generates the batch's images in host processes (spawned before any GPU
    work) while the GPU legs run."""

    def __init__(self):
        import multiprocessing as mp
        self.specs = batch_specs()
        self.pool = mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1))
        self.result = self.pool.map_async(_batch_image, self.specs, chunksize=1)

    def get(self) -> list[np.ndarray]:
        images = self.result.get()
        self.pool.close()
        self.pool.join()
        return images


def batched_leg(images: "BatchImages", precision: int) -> dict:
    """Aggregate MP/s of the whole batch through gjxl_b200_batch_analyze
    (device-resident inputs, autotuned lanes and order), and per-image
    latency percentiles, against the same images one after another on one
    lane (the plain form's sequential analyses)."""
    import torch
    from gjxl_b200.batch import BatchAnalyzer
    imgs = images.get()
    specs = images.specs
    dev = [torch.from_numpy(img.reshape(img.shape[0], -1)).cuda() for img in imgs]
    mp = sum(w * h for w, h, _, _ in specs) / 1e6
    b = BatchAnalyzer(precision=precision)
    reqs = b.requests([(d.data_ptr(), w, h, t) for d, (w, h, t, _) in zip(dev, specs)])

    def timed(reps: int = 3):
        runs = [b.analyze(reqs) for _ in range(reps)]
        results, ms = min(runs, key=lambda r: r[1])
        assert all(r["status"] == 0 for r in results), "batch image failed"
        service = [r["service_ms"] for r in results]
        ready = [r["ready_ms"] for r in results]
        return {"value": round(mp / (ms / 1e3), 3), "unit": "MP/s", "batch_ms": round(ms, 3),
                "service_ms_p50": round(float(np.percentile(service, 50)), 3),
                "service_ms_p99": round(float(np.percentile(service, 99)), 3),
                "ready_ms_p50": round(float(np.percentile(ready, 50)), 3),
                "ready_ms_p99": round(float(np.percentile(ready, 99)), 3)}

    b.set_schedule(1, False)
    b.analyze(reqs)  # plans the sequential lane (sessions, graphs)
    sequential = timed()
    lanes, largest_first = b.autotune(reqs, lane_counts=(2, 4, 8))
    batched = timed()
    device_gb = b.device_bytes() / 1e9
    b.close()
    del dev
    torch.cuda.empty_cache()
    return {"images": len(specs), "megapixels": round(mp, 3),
            "sizes": "width, height log-uniform in [256, 4096], aspect 0.5-2, "
                     "distance uniform in [0.5, 3.0], effort 7, seeds 4000000 + i",
            "batched": batched | {"lanes": lanes, "largest_first": largest_first},
            "sequential": sequential | {"lanes": 1},
            "speedup": round(batched["value"] / sequential["value"], 3),
            "device_gb": round(device_gb, 2),
            "timing": "device clock (CUDA events), min of 3 runs after planning; "
                      "service = an image's own analysis, ready = batch arrival to its end"}


def learned_leg(images: "BatchImages | None", precision: int, steps: int, warmup: int) -> dict:
    """The learned form (the committed proposal network, one field update):
    the 12 MP workload's MP/s with 3 sessions in flight, as the plain line
    is timed; the 64-image batch through the batched analysis; and the
    BD-rate against the plain method on 4 held-out 2048x2048 images of the
    proposal network's configuration (seeds 5001000 + i, never trained on)
    at distances 0.5, 1, 2, 3, through the reference's unchanged serializer,
    for the default form and for the form with the plain method's two field
    updates."""
    import torch
    from gjxl_b200 import learned
    from gjxl_b200.session import AnalysisSession
    net = learned.ProposalNetwork.load()
    w = net.params.data_ptr()
    img = make_image()
    d_img = torch.from_numpy(img.reshape(HEIGHT, -1)).cuda()
    row = WIDTH * 3
    sessions = [AnalysisSession(WIDTH, HEIGHT, butteraugli_target=1.0, effort=7,
                                precision=precision, proposal_weights=w, learned_iterations=1)
                for _ in range(3)]
    side = [torch.cuda.Stream() for _ in sessions]
    main = torch.cuda.current_stream()
    for s, st in zip(sessions, side):
        for _ in range(warmup):
            s.analyze(d_img.data_ptr(), row, 3, st.cuda_stream)
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(main)
    for st in side:
        st.wait_event(start)
    for i in range(steps):
        sessions[i % 3].analyze(d_img.data_ptr(), row, 3, side[i % 3].cuda_stream)
    for st in side:
        done = torch.cuda.Event()
        done.record(st)
        main.wait_event(done)
    stop.record(main)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop) / steps
    o = sessions[0].outputs
    masks = learned.device_array(o.tile_family_masks, (o.tiles_y, o.tiles_x), np.uint8)
    masks = masks.cpu().numpy()
    kept = float(np.unpackbits(masks[..., None], axis=-1)[..., 1:].sum(-1).mean() / 7.0)
    for s in sessions:
        s.close()
    out = {"iterations": 1, "value_12mp": round(WIDTH * HEIGHT / 1e6 / (ms / 1e3), 3),
           "ms_per_step_12mp": round(ms, 4), "families_kept": round(kept, 4),
           "fallback_tiles": round(float((masks == 0x7F).mean()), 4)}
    if images is not None:
        from gjxl_b200.batch import BatchAnalyzer
        imgs = images.get() if not hasattr(images, "cached") else images.cached
        images.cached = imgs
        dev = [torch.from_numpy(a.reshape(a.shape[0], -1)).cuda() for a in imgs]
        mp = sum(wd * ht for wd, ht, _, _ in images.specs) / 1e6
        b = BatchAnalyzer(precision=precision, proposal_weights=w, learned_iterations=1)
        reqs = b.requests([(d.data_ptr(), wd, ht, t)
                           for d, (wd, ht, t, _) in zip(dev, images.specs)])
        lanes, _ = b.autotune(reqs, lane_counts=(2, 4, 8))
        runs = [b.analyze(reqs) for _ in range(3)]
        results, bms = min(runs, key=lambda r: r[1])
        assert all(r["status"] == 0 for r in results)
        out["batched"] = {"value": round(mp / (bms / 1e3), 3), "batch_ms": round(bms, 3),
                          "lanes": lanes}
        b.close()
        del dev
    from gjxl_b200.synthetic import generate_srgb8, workload_seed
    held = [generate_srgb8(2048, 2048, workload_seed(5, 1000 + i)) for i in range(4)]
    ev = learned.evaluate(learned.WEIGHTS_PATH, held, learned_iterations=1)
    out["bd_rate_max"] = round(ev["bd_rate_mean"], 5)
    out["bd_rate_pnorm"] = round(ev["bd_rate_pnorm_mean"], 5)
    out["bd_rate_max_per_image"] = [round(p["bd_rate"], 4) for p in ev["per_image"]]
    out["bd_rate_images"] = ("4 held-out 2048x2048 images, distances 0.5/1/2/3, plain vs "
                             "learned; max = BD-rate on the maximum Butteraugli score, "
                             "pnorm = on the 3-norm")
    out["analysis_speedup_4mp"] = round(ev["speedup_mean"], 3)
    ev2 = learned.evaluate(learned.WEIGHTS_PATH, held, learned_iterations=2)
    out["two_updates"] = {"bd_rate_max": round(ev2["bd_rate_mean"], 5),
                          "bd_rate_pnorm": round(ev2["bd_rate_pnorm_mean"], 5),
                          "analysis_speedup_4mp": round(ev2["speedup_mean"], 3)}
    torch.cuda.empty_cache()
    return out


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", default="b200", choices=["b200", "reference"])
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--launch-list", action="store_true")
    parser.add_argument("--sessions", type=int, default=3,
                        help="analysis sessions (images in flight) per GPU")
    parser.add_argument("--size", default=None,
                        help="WxH of a smaller image of the same generator (profiling only)")
    parser.add_argument("--no-reference-gpu", action="store_true",
                        help="skip timing the reference's own CUDA path")
    parser.add_argument("--no-learned", action="store_true",
                        help="skip the learned-form leg")
    parser.add_argument("--no-batched", action="store_true",
                        help="skip the batched-form leg (64 images of uneven sizes)")
    parser.add_argument("--precision", default="exact", choices=["exact", "fast"],
                        help="candidate-cost precision: exact (FP64, the reference's CPU "
                             "results bit for bit) or fast (tcgen05 tensor cores)")
    args = parser.parse_args()
    if args.size:
        global WIDTH, HEIGHT
        WIDTH, HEIGHT = (int(v) for v in args.size.lower().split("x"))
    if args.impl == "reference":
        out = run_reference(args)
        if out:
            print(json.dumps(out))
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    # The CPU leg's worker processes start before any CUDA work (spawn).
    pool = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.launch_list:
        pool = ReferencePool()
    batch_images = None
    if rank == 0 and world == 1 and not args.no_batched and not args.launch_list:
        batch_images = BatchImages()
    out = run_gpu(args)
    if out:
        precision = 1 if args.precision == "fast" else 0
        if batch_images is not None:
            imgs = batch_images.get()
            batch_images.cached = imgs
            batch_images.get = lambda: imgs
            out["batched_form"] = batched_leg(batch_images, precision)
        if world == 1 and not args.no_learned and not args.launch_list:
            out["learned_form"] = learned_leg(batch_images, precision, args.steps, args.warmup)
            base = out["batched_form"]["sequential"]["value"] if batch_images else None
            if base and "batched" in out["learned_form"]:
                out["learned_form"]["batched_vs_plain_sequential"] = round(
                    out["learned_form"]["batched"]["value"] / base, 3)
            out["learned_form"]["vs_plain_12mp"] = round(
                out["learned_form"]["value_12mp"] / out["value"], 3)
        if pool is not None:
            out["cpu_baseline"] = cpu_baseline_leg(pool)
        if world == 1 and not args.launch_list and not args.no_reference_gpu:
            try:
                out["reference_gpu"] = reference_gpu_leg()
            except Exception as exc:  # reported, never fatal to our own line
                out["reference_gpu"] = {"unavailable": str(exc)[:200]}
        print(json.dumps(out))
    if pool is not None:
        pool.close()


if __name__ == "__main__":
    main()
