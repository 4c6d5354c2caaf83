"""Benchmark: bilateral filtering throughput and latency of the B200 permutohedral lattice.

Headline workload (one "step"): a batch of four 3840x2160 RGB frames through the batched
lattice (FP32 values by default, --payload to change), d=5 positions (r/0.1, g/0.1, b/0.1,
x/16, y/16), values RGB + homogeneous 1, on seeded synthetic frames (gradients, 64
rectangles, Gaussian noise sigma 0.05).  `value` is Mpix/s with the frames already resident
in HBM; `e2e` is the same step through the C ABI with pinned host frames, host->device and
device->host copies inside the timed region.  Beside it, the same line reports the plain
GPU lattice (one FP32 frame per call), the same batch with the FP16 payload, the
mixed-size batch (256 images, sides log-uniform 128..1024, per-image sigmas, FP16, CUDA
graph), a served request stream (Poisson arrivals ramped 50 -> 2000 req/s, bilateral RGB
and grey joint-bilateral requests, sides 64..2048) with p50/p99 latency, and each
payload's error against the FP64 lattice.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); frames are independent, so ranks run replicas
with no data-path collective ("weak" scaling); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, SIGMA_S, SIGMA_R, RECTS, SEED = 3840, 2160, 16.0, 0.1, 64, 2
FRAMES_PER_STEP = 4
METRIC = "bilateral Mpix/s (d=5 4K, batched) vs plain GPU; p50/p99 latency @ err<=1e-3"
PAYLOAD_NAMES = {"fp32": "FP32 values", "fp16": "FP16 payload / FP32 accumulation",
                 "bf16": "BF16 payload / FP32 accumulation", "fp64": "FP64 values"}


def workload(payload):
    return ("bilateral RGB 3840x2160 x%d frames per batch, d=5 (sigma_s 16, sigma_r 0.1), %s"
            % (FRAMES_PER_STEP, PAYLOAD_NAMES[payload]))


L2_BYTES = 126 * 1024 * 1024
# launches of one lattice besides the blur's: tile splat, neighbours, replay slice, and the
# list-ordered compaction where rows stay in slot space


def kernels_per_lattice(vertex_rows):
    return 3 if vertex_rows else 4
TUNE_MAX_CALLS = 24       # at most this many calls for the autotuner to finish a shape


def tune(fn, prepare=None):
    """Call fn until the batch autotuner reports its choice for the shape (stats "tuned"
    2: its trials, each setting timed twice, are over); returns the calls made."""
    for k in range(TUNE_MAX_CALLS):
        if prepare:
            prepare()
        fn()
        if fn.stats()["tuned"] != 1:
            return k + 1
    return TUNE_MAX_CALLS
D = 5


def blur_launches(d, pairs=True):
    return (d + 2) // 2 if pairs else d + 1   # axes blurred in fused pairs, or one by one


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def stage_bytes(N, M, d=D, C=3, p=4, vdp=4, vertex_rows=False, nbr_half=False):
    """Algorithmic bytes of each lattice stage for N points and M vertices: what each stage's
    kernels must move as they are built, every input read once and every output written
    once (a row is vdp values of p bytes; the splat's sums and the slice's rows are FP32).
      splat       image N*C*4 read; replay record N*(d+1)*(4 index + 4 weight) written;
                  table M*(16 key + 4*vdp row) written once; with vertex-ordered rows the
                  creator also writes the key in vertex order M*16, the vertex's slot M*4
                  and its index in the key word M*4 (and, for the one-lookup neighbour
                  search, the vertex's absent-neighbour pairs M*8*(d+1))
      compaction  (slot-space rows only) vertex list M*4, key M*16 and row M*4*vdp read;
                  key M*16, row M*p*vdp, both index maps M*8 and the index in the key word
                  M*16 written (and the absent pairs M*8*(d+1) for the one-lookup search)
      neighbours  key M*16 read, one table slot M*16 per lookup (2(d+1) lookups, or d+1
                  with one lookup per axis plus a 4-byte pair entry written per lookup), the
                  pairs M*8*(d+1) written
      blur        per axis (the separable [1 2 1] passes of the algorithm, however many
                  axes a launch fuses): rows M*p*vdp read and written and the axis's
                  neighbour pairs M*8 read; the last axis writes FP32 rows M*4*vdp
                  (slot-space rows: through the vertex->slot map M*4)
      slice       replay record N*(d+1)*8 and the FP32 rows M*4*vdp read, N*C*4 written"""
    axes = d + 1
    splat = N * C * 4 + N * axes * 8 + M * (16 + 4 * vdp)
    if vertex_rows:
        splat += M * (16 + 4 + 4) + (M * 8 * axes if nbr_half else 0)
        compact = 0
    else:
        compact = M * (4 + 16 + 4 * vdp) + M * (16 + p * vdp + 8 + 16) + (M * 8 * axes if nbr_half else 0)
    lookups = axes if nbr_half else 2 * axes
    neighbours = M * 16 + lookups * M * 16 + axes * M * 8 + (lookups * M * 4 if nbr_half else 0)
    blur = axes * (2 * M * p * vdp + M * 8) + M * (4 * vdp - p * vdp) + (0 if vertex_rows else M * 4)
    slice_ = N * axes * 8 + M * 4 * vdp + N * C * 4
    return {"splat": int(splat), "compact": int(compact), "neighbours": int(neighbours),
            "blur": int(blur), "slice": int(slice_)}


def ncu_traffic():
    """DRAM bytes of each stage for one 3840x2160 frame, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_bilateral_4k_frame.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            line = line.strip()
            if line and not line.startswith("#") and "=" in line:
                k, v = line.split("=", 1)
                try:
                    out[k.strip()] = float(v)
                except ValueError:
                    pass
    return out


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML while the timed region runs."""

    NAMES = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
             "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._ready.set()
            while not self._stop.is_set():
                self.samples.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                for n, bit in self.NAMES.items():
                    if r & bit:
                        self.reasons.add(n)
                time.sleep(0.005)
        except Exception:
            pass
        finally:
            self._ready.set()

    def __enter__(self):
        # NVML is initialised before the timed region opens, so that the region (about
        # 0.1 s for 20 steps) is sampled from its start
        self._ready = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        self._ready.wait(timeout=10)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=5)

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def dist_init():
    from imagestack_b200.replicas import rank_env
    return rank_env()


def rel_err(a, b, floor_frac=1e-2):
    import numpy as np
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(np.abs(b).max() * floor_frac, 1e-30)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max())


# --------------------------------------------------------------------------------------
# CPU baselines: the reference's own code (oracle/_ref), or the C restatement if absent
# --------------------------------------------------------------------------------------

_FRAMES = {}


def headline_config(payload, world):
    """The `config` of the headline line; the reference arm reports exactly this dict."""
    return {"workload": workload(payload), "frame": [W, H], "frames_per_step": FRAMES_PER_STEP,
            "seed": SEED, "payload": payload, "path": "batched",
            "l2": "flushed between steps (512 MiB write), outside the timed window",
            "parallelism": "replicas x%d" % world}


def _cpu_worker(args):
    """One reference Bilateral::apply on a full frame of the headline workload (frame
    seed `seed`); returns (apply seconds, kind).  The frame is generated once per process
    and is not timed."""
    seed = args[0] if isinstance(args, (tuple, list)) else args
    os.environ["OMP_NUM_THREADS"] = "1"
    import oracle
    from imagestack_b200 import synth
    if seed not in _FRAMES:
        _FRAMES[seed] = synth.image(W, H, 3, rects=RECTS, seed=seed)
    img = _FRAMES[seed]
    if oracle.reference_available():
        _, t = oracle.reference_bilateral(img, SIGMA_S, SIGMA_R)
        return t, "reference"
    pos, val = oracle.bilateral_points(img, img, SIGMA_S, SIGMA_R)
    t0 = time.perf_counter()
    oracle.oracle_lattice(pos, val)
    return time.perf_counter() - t0, "port"


def _cpu_fresh_process(seed, build):
    """_cpu_worker in a process of its own (the reference's timing drifts with reuse)."""
    code = ("import sys,json; sys.path.insert(0,%r); import bench; "
            "print(json.dumps(bench._cpu_worker(%d)))" % (ROOT, seed))
    env = dict(os.environ, OMP_NUM_THREADS="1", PGPU_REFERENCE_BUILD=build)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=900)
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_baseline_single(build="strict", runs=3):
    """Reference Bilateral::apply on one full frame (the headline's first frame), one
    thread, the median of `runs` fresh processes.  build "strict": the reference compiled
    with IEEE-exact flags (the parity oracle); "shipped": its shipped -ffast-math flags."""
    from imagestack_b200.replicas import frame_seeds
    seed = frame_seeds(0, FRAMES_PER_STEP, SEED)[0]
    res = [_cpu_fresh_process(seed, build) for _ in range(runs)]
    times = sorted(t for t, _ in res)
    t = statistics.median(times)
    flags = ("-O3 -ffp-contract=off (strict IEEE)" if build == "strict"
             else "-O3 -ffast-math (the reference's shipped flags)")
    return {"value": round(W * H / t / 1e6, 4), "unit": "Mpix/s", "cores": 1, "kind": res[0][1],
            "sample": "one full 3840x2160 frame (seed %d), Bilateral::apply(permutohedral), "
                      "1 thread, median of %d fresh processes (%s s), reference built %s"
                      % (seed, runs, ", ".join("%.2f" % x for x in times), flags)}


def _cpu_mixed_worker(spec):
    """The reference's Bilateral::apply on one image of the mixed batch (regenerated here
    from its seed, not timed); returns (pixels, apply seconds)."""
    os.environ["OMP_NUM_THREADS"] = "1"
    import oracle
    from imagestack_b200 import synth
    w, h, ss, sr, seed = spec
    img = synth.image(w, h, 3, rects=16, seed=seed)
    _, t = oracle.reference_bilateral(img, ss, sr)
    return w * h, t


def cpu_baseline_mixed():
    """The mixed batch (256 uneven RGB images, their own sigmas) through the reference on
    all host cores, one single-threaded process per core over disjoint images."""
    import multiprocessing as mp
    from imagestack_b200 import synth
    specs = synth.batch_specs(256, 128, 1024, seed=SEED)
    procs = max(1, min(os.cpu_count() or 1, 64))
    with mp.get_context("spawn").Pool(procs) as pool:
        pool.map(_cpu_mixed_worker, [(64, 64, 8.0, 0.1, 1)] * procs)   # start the workers
        t0 = time.perf_counter()
        res = pool.map(_cpu_mixed_worker, specs, chunksize=1)
        wall = time.perf_counter() - t0
    px = sum(r[0] for r in res)
    return {"value": round(px / wall / 1e6, 2), "unit": "Mpix/s", "cores": procs,
            "kind": "reference", "sample": "the 256-image mixed batch, FP32, one Bilateral::apply "
            "per image, %d single-threaded processes (%.2f s wall)" % (procs, wall)}


def run_reference_arm(args):
    """The reference's own CPU path on the headline workload: full 3840x2160 frames of the
    headline batch (the same seeds), one Bilateral::apply per frame, one single-threaded
    process per host core (the lattice is serial), each step every process filtering one
    frame; throughput over the whole host."""
    world, rank, _ = dist_init()
    if rank != 0:
        return
    import multiprocessing as mp

    from imagestack_b200.replicas import frame_seeds
    try:
        import psutil
        mem = psutil.virtual_memory().available
    except Exception:
        mem = 64 << 30
    cores = os.cpu_count() or 1
    # a full 4K frame through the reference takes about 1.5 GB of host memory
    procs = max(1, min(cores, int(mem // (2 << 30)) - 1, 64))
    seeds = frame_seeds(0, FRAMES_PER_STEP, SEED)
    ctx = mp.get_context("spawn")
    times = []
    kind = "reference"
    with ctx.Pool(procs) as pool:
        for step in range(args.warmup + args.steps):
            # every process filters one frame of the headline batch; a step lasts as long
            # as the slowest apply
            res = pool.map(_cpu_worker, [seeds[(step * procs + i) % len(seeds)] for i in range(procs)],
                           chunksize=1)
            kind = res[0][1]
            if step >= args.warmup:
                times.append(max(r[0] for r in res))
    ms = 1e3 * statistics.median(times)
    value = procs * W * H / (ms / 1e3) / 1e6
    sample = ("%d single-threaded processes, each Bilateral::apply on one full 3840x2160 frame "
              "of the headline batch per step (median step)" % procs)
    line = {"metric": METRIC, "value": round(value, 4), "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": headline_config(args.payload, world),
            "cpu_baseline": {"value": round(value, 4), "unit": "Mpix/s", "cores": procs,
                             "kind": kind, "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------

def timed_steps(stream, steps, fn, prepare):
    """Per-step CUDA events on `stream`, `prepare` (restore inputs, flush L2) outside."""
    import torch
    events, stats = [], []
    for _ in range(steps):
        prepare()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        events.append((e0, e1))
        stats.append(fn.stats() if hasattr(fn, "stats") else None)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in events), stats


def exact_error(ib, torch, frame, filtered, samples=4096, seed=7):
    """Error of a filtered frame against the exact Gauss transform it approximates: the
    FP64 brute-force transform (every pixel a source) at `samples` seeded pixels, with the
    positions and values JointBilateral::apply builds.  The permutohedral lattice is an
    approximation of that Gaussian, so this is reported, not held to a tolerance."""
    c, h, w = frame.shape
    one = torch.tensor(1.0, dtype=torch.float32)
    inv_r = (one / torch.tensor(SIGMA_R, dtype=torch.float32)).item()
    inv_s = (one / torch.tensor(SIGMA_S, dtype=torch.float32)).item()
    ys, xs = torch.meshgrid(torch.arange(h, device=frame.device, dtype=torch.float32),
                            torch.arange(w, device=frame.device, dtype=torch.float32), indexing="ij")
    pos = torch.stack([frame[k] * inv_r for k in range(c)] + [xs * inv_s, ys * inv_s], -1).reshape(-1, c + 2)
    val = torch.cat([frame.reshape(c, -1).t(), torch.ones(h * w, 1, device=frame.device)], 1)
    g = torch.Generator().manual_seed(seed)
    idx = torch.randperm(h * w, generator=g)[:samples].to(frame.device)
    t0 = time.perf_counter()
    ex = ib.exact_gauss_transform_f64(pos[idx].contiguous(), pos.contiguous(), val.contiguous())
    secs = time.perf_counter() - t0
    exact = (ex[:, :c] / ex[:, c:]).cpu().numpy()
    lat = filtered.reshape(c, -1)[:, idx].t().double().cpu().numpy()
    import numpy as np
    floor = 1e-2 * np.abs(exact).max()
    rel = np.abs(lat - exact) / np.maximum(np.abs(exact), floor)
    return {"samples": samples, "max_rel_err": float(rel.max()), "mean_rel_err": float(rel.mean()),
            "oracle": "FP64 brute force over all %d pixels on the GPU (%.2f s)" % (h * w, secs)}


def grey_4k(ib, synth, torch, frame, steps=10):
    """The 4K config's grey variant: joint bilateral of the frame's luminance with itself
    (d=3: luminance/0.1, x/16, y/16), by the permutohedral lattice and by the bilateral
    grid (the method JointBilateral::apply's AUTO picks for three position channels)."""
    lum = (0.299 * frame[0] + 0.587 * frame[1] + 0.114 * frame[2])[None].contiguous()
    work = torch.empty_like(lum)
    stream = torch.cuda.current_stream(lum.device)
    out = {}
    for method in ("permutohedral_gpu", "grid_gpu"):
        def fn():
            ib.Bilateral.apply(work, SIGMA_S, SIGMA_S, 0.0, SIGMA_R, method=method)
        for _ in range(3):
            work.copy_(lum)
            fn()
        ms, _ = timed_steps(stream, steps, fn, lambda: work.copy_(lum))
        out[method] = {"ms_per_frame": round(ms / steps, 4),
                       "mpix_s": round(W * H * steps / (ms / 1e3) / 1e6, 1)}
    return out


def gauss_transform_d16(ib, synth, torch, dev, reps=3):
    """GaussTransform::apply on 2M points of a 16-D Gaussian mixture (4 value channels +
    the homogeneous one, unit sigmas), the high-dimensional case where keys take three
    words.  Two untimed calls first: the first learns the vertices-per-point ratio of this
    shape, the second grows the hash table to the capacity that ratio asks for."""
    import numpy as np
    n, d = 2_000_000, 16
    pos, vals = synth.gauss_mixture(n, d=d, seed=SEED)
    P = torch.from_numpy(np.ascontiguousarray(pos.T.reshape(d, 1, -1))).to(dev)
    V = torch.from_numpy(np.ascontiguousarray(vals.T.reshape(vals.shape[1], 1, -1))).to(dev)
    stream = torch.cuda.current_stream(dev)

    def fn():
        ib.GaussTransform.apply(None, P, V, [1.0] * d)
    fn.stats = ib.last_stats
    for _ in range(2):
        fn()
    ms, st = timed_steps(stream, reps, fn, lambda: None)
    return {"points": n, "d": d, "ms_per_call": round(ms / reps, 3),
            "device_ms": round(sum(s["ms_total"] for s in st) / reps, 3),
            "vertices": st[-1]["vertices"],
            "mpoints_s": round(n * reps / (ms / 1e3) / 1e6, 1)}


def mixed_batch(ib, synth, torch, dev, steps):
    """The mixed-size batch: 256 uneven RGB images, per-image sigmas, one batched launch
    sequence (FP16 payload, CUDA graph) against the plain per-image FP32 path."""
    specs = synth.batch_specs(256, 128, 1024, seed=SEED)
    imgs = [torch.from_numpy(synth.image(w, h, 3, rects=16, seed=s)).to(dev)
            for (w, h, ss, sr, s) in specs]
    ss = [s[2] for s in specs]
    sr = [s[3] for s in specs]
    px = sum(im.shape[1] * im.shape[2] for im in imgs)
    work = [torch.empty_like(im) for im in imgs]
    stream = torch.cuda.current_stream(dev)

    def restore():
        for wk, im in zip(work, imgs):
            wk.copy_(im)

    def batched():
        ib.bilateral_batch(work, ss, sr, payload="fp16", graph=True, autotune=True)

    def plain():
        for wk, s, r in zip(work, ss, sr):
            ib.Bilateral.apply(wk, s, s, 0.0, r)

    batched.stats = ib.last_stats
    tune(batched, restore)   # the autotuner's trials of this batch shape
    for _ in range(2):
        restore()
        batched()
        restore()
        plain()
    torch.cuda.synchronize()
    tb, _ = timed_steps(stream, steps, batched, restore)
    tp, _ = timed_steps(stream, max(1, steps // 2), plain, restore)
    # error of the batched FP16 results against the FP64 lattice on a sample of images
    restore()
    batched()
    torch.cuda.synchronize()
    err = 0.0
    for k in range(0, 256, 32):
        ref = imgs[k].clone()
        ib.Bilateral.apply(ref, ss[k], ss[k], 0.0, sr[k], payload="fp64")
        torch.cuda.synchronize()
        err = max(err, rel_err(work[k].cpu().numpy(), ref.cpu().numpy()))
    return {"images": 256, "pixels": px,
            "batched_fp16_graph_mpix_s": round(px * steps / (tb / 1e3) / 1e6, 2),
            "plain_fp32_per_image_mpix_s": round(px * max(1, steps // 2) / (tp / 1e3) / 1e6, 2),
            "max_rel_err_fp16_vs_fp64": err}


def served_saturation(ib, synth, torch, count=4000, workers=2, max_batch=32):
    """The server at saturation: `count` requests of the served stream's mix (24 pooled
    images, bilateral RGB and grey joint bilateral, sides 64..2048) submitted at once."""
    import numpy as np
    sides = synth.log_uniform_int(SEED, 31, 48, 64, 2048)
    rng = np.random.default_rng(SEED + 1)
    pool = []
    for k in range(24):
        w, h = int(sides[2 * k]), int(sides[2 * k + 1])
        rgb = synth.image(w, h, 3, rects=8, seed=700 + k)
        if k % 2 == 0:
            img, ref, kind = torch.from_numpy(rgb).pin_memory(), None, ib.REQ_BILATERAL
        else:
            img = torch.from_numpy(synth.luminance(rgb)).pin_memory()
            ref = torch.from_numpy(synth.luminance(synth.image(w, h, 3, rects=8, seed=900 + k))).pin_memory()
            kind = ib.REQ_JOINT_BILATERAL
        pool.append((kind, img.numpy(), None if ref is None else ref.numpy(),
                     torch.empty_like(img).pin_memory().numpy(),
                     float(4 + 28 * rng.random()), float(0.05 + 0.25 * rng.random())))
    with ib.Server(workers=workers, max_batch=max_batch, payload="fp16", memory_budget=40 << 30) as srv:
        for kind, img, ref, out, ss, sr in pool:   # warm-up: every shape once
            srv.wait(srv.submit(kind, img, out, ref=ref, filter_width=ss, color_sigma=sr))
        srv.reset_stats()
        tickets = []
        for j in range(count):
            kind, img, ref, out, ss, sr = pool[j % 24]
            tickets.append(srv.submit(kind, img, out, ref=ref, filter_width=ss, color_sigma=sr))
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
    return {"requests": int(st["completed"]), "failed": int(st["failed"]),
            "throughput_req_s": round(st["req_per_s"], 1), "throughput_mpix_s": round(st["mpix_per_s"], 1),
            "p50_ms": round(st["p50_ms"], 2), "p99_ms": round(st["p99_ms"], 2), "workers": workers,
            "note": "every request of the same pooled image writes the same output buffer"}


def served_stream(ib, synth, torch, seconds=60.0, rate0=50.0, rate1=2000.0, workers=2, max_batch=32):
    """The served stream: Poisson arrivals ramped rate0 -> rate1 req/s over `seconds`;
    half bilateral RGB (d=5), half joint bilateral of a grey image on a grey guide (d=3);
    sides log-uniform 64..2048, sigmas as the mixed batch; FP16 payload, 40 GB budget.
    Requests reuse a pool of pinned host images; each has its own pinned output."""
    import numpy as np
    rng = np.random.default_rng(SEED)
    P = 24
    sides = synth.log_uniform_int(SEED, 31, 2 * P, 64, 2048)
    pool = []
    for k in range(P):
        w, h = int(sides[2 * k]), int(sides[2 * k + 1])
        rgb = synth.image(w, h, 3, rects=8, seed=700 + k)
        kind = k % 2
        if kind == 0:
            img = torch.from_numpy(rgb).pin_memory()
            ref = None
        else:
            img = torch.from_numpy(synth.luminance(rgb)).pin_memory()
            ref = torch.from_numpy(synth.luminance(synth.image(w, h, 3, rects=8, seed=900 + k))).pin_memory()
        outs = [torch.empty_like(img).pin_memory() for _ in range(4)]
        pool.append(dict(kind=ib.REQ_BILATERAL if kind == 0 else ib.REQ_JOINT_BILATERAL,
                         img=img, ref=ref, outs=outs, busy=[None] * 4,
                         ss=float(4 + 28 * rng.random()), sr=float(0.05 + 0.25 * rng.random())))
    srv = ib.Server(workers=workers, max_batch=max_batch, payload="fp16", memory_budget=40 << 30)
    # warm each worker's workspace on the pool
    tickets = []
    for q in pool:
        t = srv.submit(q["kind"], q["img"].numpy(), q["outs"][0].numpy(),
                       ref=None if q["ref"] is None else q["ref"].numpy(),
                       filter_width=q["ss"], color_sigma=q["sr"])
        tickets.append(t)
    for t in tickets:
        srv.wait(t)
    srv.reset_stats()
    pending = []
    lock = threading.Lock()
    t_start = time.perf_counter()
    t = 0.0
    j = 0
    while t < seconds:
        rate = rate0 + (rate1 - rate0) * t / seconds
        t += rng.exponential(1.0 / rate)
        delay = t_start + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        q = pool[j % P]
        slot = (j // P) % 4
        if q["busy"][slot] is not None:      # the output slot is still owned by an older request
            srv.wait(q["busy"][slot])
        tk = srv.submit(q["kind"], q["img"].numpy(), q["outs"][slot].numpy(),
                        ref=None if q["ref"] is None else q["ref"].numpy(),
                        filter_width=q["ss"], color_sigma=q["sr"])
        q["busy"][slot] = tk
        pending.append(tk)
        j += 1
    for q in pool:
        for s, tk in enumerate(q["busy"]):
            if tk is not None:
                srv.wait(tk)
    st = srv.stats()
    srv.close()
    return {"requests": int(st["completed"]), "failed": int(st["failed"]),
            "window_s": round(seconds, 2), "rate_req_s": [rate0, rate1],
            "p50_ms": round(st["p50_ms"], 3), "p99_ms": round(st["p99_ms"], 3),
            "max_ms": round(st["max_ms"], 3), "throughput_mpix_s": round(st["mpix_per_s"], 2),
            "throughput_req_s": round(st["req_per_s"], 1), "batches": int(st["batches"]),
            "payload": "fp16", "workers": workers, "max_batch": max_batch, "memory_budget_gib": 40}


def run_ours(args):
    import numpy as np
    import torch

    import imagestack_b200 as ib
    from imagestack_b200 import synth

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    from imagestack_b200.replicas import frame_seeds, max_over_ranks
    frames = [synth.image(W, H, 3, rects=RECTS, seed=s)
              for s in frame_seeds(rank, FRAMES_PER_STEP, SEED)]
    pristine = [torch.from_numpy(f).to(dev) for f in frames]
    work = [torch.empty_like(p) for p in pristine]
    flush = torch.empty(4 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ss = [SIGMA_S] * FRAMES_PER_STEP
    sr = [SIGMA_R] * FRAMES_PER_STEP

    def prepare():
        for wk, p in zip(work, pristine):
            wk.copy_(p)      # the filter is in place: restore the frames
        flush.fill_(1.0)     # evict L2 between steps; both outside the timed window

    def headline():
        ib.bilateral_batch(work, ss, sr, payload=args.payload, autotune=not args.no_autotune)
    headline.stats = ib.last_stats

    def plain():
        ib.Bilateral.apply(work[0], SIGMA_S, SIGMA_S, 0.0, SIGMA_R, payload="fp32")
    plain.stats = ib.last_stats

    # the same batch with the 16-bit payload (FP16 rows, FP32 accumulation), beside it
    alt_payload = "fp16" if args.payload != "fp16" else "fp32"

    def alt():
        ib.bilateral_batch(work, ss, sr, payload=alt_payload, autotune=not args.no_autotune)
    alt.stats = ib.last_stats

    tune_calls = {}
    if not args.no_autotune:   # the autotuner's trials
        tune_calls[args.payload] = tune(headline, prepare)
        if not args.quick:
            tune_calls[alt_payload] = tune(alt, prepare)
    for _ in range(args.warmup):
        prepare()
        headline()
        prepare()
        plain()
        if not args.quick:
            prepare()
            alt()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms, stage = timed_steps(stream, args.steps, headline, prepare)
    plain_ms, plain_stage = timed_steps(stream, args.steps, plain, prepare)
    if not args.quick:
        alt_ms, alt_stage = timed_steps(stream, args.steps, alt, prepare)
    total_ms = max_over_ranks(total_ms, dev)
    ms_per_step = total_ms / args.steps
    px_step = W * H * FRAMES_PER_STEP
    value = world * px_step * args.steps / (total_ms / 1e3) / 1e6
    plain_mpix = W * H * args.steps / (plain_ms / 1e3) / 1e6

    # End to end through the C ABI, pinned host frames in and filtered frames out, every
    # step's uploads and downloads inside the timed region.  A step is one queued batch of
    # the four frames (pgpu_bilateral_batch_submit, out of place, so the inputs stay as
    # they are); two steps are in flight, so one step's uploads overlap the previous
    # step's lattices and downloads.  Timed by the host clock from the first submission to
    # the last wait.
    host_in = [torch.from_numpy(f.copy()).pin_memory() for f in frames]
    host_out = [[torch.empty_like(h).pin_memory() for h in host_in] for _ in range(2)]
    in_np = [h.numpy() for h in host_in]
    out_np = [[h.numpy() for h in row] for row in host_out]
    autotune = not args.no_autotune

    def submit(i):
        return ib.bilateral_batch_submit(in_np, ss, sr, outputs=out_np[i % 2], payload=args.payload,
                                         autotune=autotune)
    e2e_steps = max(args.steps, 10)
    e2e_tune = 0
    for i in range(TUNE_MAX_CALLS):   # the autotuner's trials of the one-frame chunk shape
        submit(i).wait()
        e2e_tune += 1
        if not autotune or ib.last_stats()["tuned"] != 1:
            break
    for i in range(args.warmup):
        submit(i).wait()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    from collections import deque
    t0 = time.perf_counter()
    inflight = deque()
    for i in range(e2e_steps):
        if len(inflight) == 2:
            inflight.popleft().wait()
        inflight.append(submit(i))
    while inflight:
        inflight.popleft().wait()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dev)
    e2e = world * px_step * e2e_steps / e2e_s / 1e6
    e2e_out = out_np[(e2e_steps - 1) % 2][0].copy()

    # the same step as one synchronous call (in place: the frames are restored outside the
    # timed region), which cannot overlap one step's copies with the next step's
    host_np = out_np[0]
    sync_times = []
    for i in range(args.warmup + 10):
        for hn, f in zip(host_np, frames):
            hn[...] = f
        t1 = time.perf_counter()
        ib.bilateral_batch(host_np, ss, sr, payload=args.payload, autotune=autotune)
        if i >= args.warmup:
            sync_times.append(time.perf_counter() - t1)
    e2e_sync = px_step * len(sync_times) / sum(sync_times) / 1e6

    # the copies alone: the four frames up, down, and both at once on two streams
    def copy_ms(up, down, reps=5):
        s_up, s_dn = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        best = 1e30
        for _ in range(reps):
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            if up:
                with torch.cuda.stream(s_up):
                    for wk, h in zip(work, host_in):
                        wk.copy_(h, non_blocking=True)
            if down:
                with torch.cuda.stream(s_dn):
                    for p_, h in zip(pristine, host_out[1]):
                        h.copy_(p_, non_blocking=True)
            torch.cuda.synchronize()
            best = min(best, (time.perf_counter() - t2) * 1e3)
        return best
    copies = {"h2d_ms": round(copy_ms(True, False), 3), "d2h_ms": round(copy_ms(False, True), 3),
              "both_ms": round(copy_ms(True, True), 3)}
    copies["bound_mpix_s"] = round(px_step / (copies["both_ms"] / 1e3) / 1e6, 1)

    if rank == 0:
        hbm, peak_kind = peaks()
        n = W * H
        M = stage[-1]["vertices"]
        splat_ms = statistics.mean(s["ms_splat"] for s in stage)
        stages = {k: round(statistics.mean(s[k] for s in stage), 4)
                  for k in ("ms_splat", "ms_compact", "ms_neighbours", "ms_blur", "ms_slice",
                            "ms_total")}
        plain_stages = {k: round(statistics.mean(s[k] for s in plain_stage), 4)
                        for k in ("ms_splat", "ms_compact", "ms_neighbours", "ms_blur",
                                  "ms_slice", "ms_total")}
        # Algorithmic bytes of each stage (stage_bytes: formulas that follow the kernels),
        # for all frames of the batch and M = the measured vertices of the batch
        p = {"fp32": 4, "fp16": 2, "bf16": 2, "fp64": 8}[args.payload]
        N = FRAMES_PER_STEP * n
        passes = blur_launches(D, bool(stage[-1]["blur_pairs"]))
        sb = stage_bytes(N, M, p=p, vertex_rows=bool(stage[-1]["vertex_rows"]),
                         nbr_half=bool(stage[-1]["nbr_half"]))
        splat_bytes = sb["splat"]
        achieved = splat_bytes / (splat_ms / 1e3) / 1e9
        total_bytes = sum(sb.values())
        lattice_ms = statistics.mean(s["ms_total"] for s in stage)
        traffic = ncu_traffic()
        stage_ms_key = {"splat": "ms_splat", "compact": "ms_compact", "neighbours": "ms_neighbours",
                        "blur": "ms_blur", "slice": "ms_slice"}
        roofline_stages = {}
        for k, b in sb.items():
            ms = stages[stage_ms_key[k]]
            ach = b / (ms / 1e3) / 1e9 if (ms > 0 and b > 0) else None
            roofline_stages[k] = {"bytes": b, "ms": ms, "achieved_gbs": round(ach, 1) if ach else None,
                                  "frac": round(ach / hbm, 4) if ach else None,
                                  "traffic_per_frame": traffic.get(k + "_dram_bytes")}
        # the splat's atomic roofline: one float4 RED per (point, remainder) against the
        # measured RED rate at scattered rows of an L2-resident table (16 MB: the L2 atomic
        # units' ceiling), and, for reference, of a table as large as the batch's
        red_peak = ib.probe_red_rate(1 << 20)
        red_table = ib.probe_red_rate(int(stage[-1]["capacity"]))
        red_splat = N * (D + 1) / (splat_ms / 1e3)
        atomics = {"kernel": "splat", "bound": "l2_atomics", "unit": "1e9 float4 RED/s",
                   "achieved": round(red_splat / 1e9, 2), "peak": round(red_peak / 1e9, 2),
                   "frac": round(red_splat / red_peak, 4),
                   "uniform_random_rows_of_the_batch_table": round(red_table / 1e9, 2),
                   "peak_kind": "measured by pgpu_probe_red_rate in this run (16 MB table)"}
        # the payload's error on the 4K frame against the FP64 lattice
        a = pristine[0].clone()
        ib.Bilateral.apply(a, SIGMA_S, SIGMA_S, 0.0, SIGMA_R, payload=args.payload)
        b = pristine[0].clone()
        ib.Bilateral.apply(b, SIGMA_S, SIGMA_S, 0.0, SIGMA_R, payload="fp64")
        torch.cuda.synchronize()
        err4k = rel_err(a.cpu().numpy(), b.cpu().numpy())
        if not args.quick:
            c = pristine[0].clone()
            ib.Bilateral.apply(c, SIGMA_S, SIGMA_S, 0.0, SIGMA_R, payload=alt_payload)
            torch.cuda.synchronize()
            alt_line = {
                "payload": alt_payload, "path": "batched",
                "mpix_s": round(px_step * args.steps / (alt_ms / 1e3) / 1e6, 2),
                "max_rel_err_vs_fp64": rel_err(c.cpu().numpy(), b.cpu().numpy()),
                "stages_ms": {k: round(statistics.mean(s_[k] for s_ in alt_stage), 4)
                              for k in ("ms_splat", "ms_compact", "ms_neighbours", "ms_blur",
                                        "ms_slice", "ms_total")}}
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp16": "f16-payload/f32-accum",
                      "bf16": "bf16-payload/f32-accum", "fp64": "f64"}[args.payload],
            "data": "synthetic",
            "config": headline_config(args.payload, world),
            "plain_gpu": {"mpix_s": round(plain_mpix, 2), "payload": "fp32",
                          "path": "one frame per call", "stages_ms": plain_stages},
            "max_rel_err_vs_fp64": {"4k_frame": err4k, "tolerance": 1e-3,
                                    "denominator": "max(|fp64|, 1e-2 x max|fp64|)"},
            "roofline": {"kernel": "splat", "bound": "hbm", "achieved": round(achieved, 2),
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4),
                         "traffic": (traffic["splat_dram_bytes"] * FRAMES_PER_STEP
                                     if "splat_dram_bytes" in traffic else None),
                         "algorithmic_bytes": splat_bytes,
                         "note": "issue bound: the per-point simplex, keys and hashes, plus one "
                                 "float4 L2 reduction per (point, vertex); see profiles/"},
            "roofline_atomics": atomics,
            "roofline_blur": dict(roofline_stages["blur"], peak=hbm, unit="GB/s"),
            "roofline_slice": dict(roofline_stages["slice"], peak=hbm, unit="GB/s"),
            "roofline_stages": roofline_stages,
            "roofline_pipeline": {"bytes": sb, "ms": round(lattice_ms, 4),
                                  "achieved": round(total_bytes / (lattice_ms / 1e3) / 1e9, 2),
                                  "peak": hbm, "unit": "GB/s",
                                  "frac": round(total_bytes / (lattice_ms / 1e3) / 1e9 / hbm, 4)},
            "e2e": {"value": round(e2e, 2), "unit": "Mpix/s",
                    "h2d_bytes_per_step": px_step * 3 * 4, "d2h_bytes_per_step": px_step * 3 * 4,
                    "steps": e2e_steps, "ms_per_step": round(e2e_s * 1e3 / e2e_steps, 3),
                    "path": "pgpu_bilateral_batch_submit / pgpu_batch_wait, pinned host frames, "
                            "out of place, two steps in flight",
                    "max_rel_err_vs_device_path": rel_err(e2e_out, a.cpu().numpy()),
                    "copies_alone": copies,
                    "one_call_per_step_mpix_s": round(e2e_sync, 2),
                    "autotuner_calls": e2e_tune},
            "gpu_launches": args.steps * (kernels_per_lattice(stage[-1]["vertex_rows"]) + passes),
            "autotuned": {"load_factor": round(stage[-1]["load_factor"], 3),
                          "blur_pairs": bool(stage[-1]["blur_pairs"]),
                          "blur_grid": "one vertex per thread" if stage[-1]["blur_grid"]
                                       else "16 blocks per SM, striding",
                          "splat": "tile" if stage[-1]["tiled"] else "direct",
                          "rows": "vertex-ordered by the splat" if stage[-1]["vertex_rows"]
                                  else "slot space + compaction",
                          "neighbour_lookups_per_axis": 1 if stage[-1]["nbr_half"] else 2,
                          "tiles": "%dx%d" % (stage[-1]["tile_w"], 256 // max(1, stage[-1]["tile_w"])),
                          "calls": tune_calls,
                          "knobs": "coordinate descent, each option timed twice: load factor "
                                   "0.5/0.35/0.7, blur axes in pairs or one per pass (FP32/FP64), "
                                   "blur grid, tile or direct splat, slot-space or vertex-ordered "
                                   "rows, one or two neighbour lookups per axis, 16x16 or 32x8 "
                                   "tiles"},
            "stages_ms": stages, "vertices": M, "capacity": stage[-1]["capacity"],
            "clocks": clk.summary(),
        }
        if not args.quick:
            line["batched_" + alt_payload] = alt_line
            line["exact_gt_err"] = exact_error(ib, torch, pristine[0], a)
            line["grey_4k_d3"] = grey_4k(ib, synth, torch, pristine[0])
            line["gauss_transform_d16"] = gauss_transform_d16(ib, synth, torch, dev)
        if world == 1 and not args.quick:
            line["mixed_batch"] = mixed_batch(ib, synth, torch, dev, steps=6)
            line["served"] = served_stream(ib, synth, torch)
            line["served_saturation"] = served_saturation(ib, synth, torch)
            line["p50_ms"] = line["served"]["p50_ms"]
            line["p99_ms"] = line["served"]["p99_ms"]
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline_single("strict")
                line["cpu_baseline_shipped_flags"] = cpu_baseline_single("shipped")
                if not args.quick:
                    line["cpu_baseline_mixed_batch"] = cpu_baseline_mixed()
            except Exception as e:   # report, never fail the GPU line
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_profile_case(args):
    """A small, fixed case for profiler captures: one seeded RGB frame (4K or 1080p, the
    headline's generator and sigmas) through the plain single-frame path three times, so
    that a capture can skip the first two calls (the first learns the vertex ratio, the
    second sizes the table); nothing is timed."""
    import torch

    import imagestack_b200 as ib
    from imagestack_b200 import synth
    w, h = {"frame4k": (W, H), "frame1080p": (W // 2, H // 2)}[args.profile]
    frame = torch.from_numpy(synth.image(w, h, 3, rects=RECTS if w == W else RECTS // 2, seed=SEED)).cuda()
    work = torch.empty_like(frame)
    for _ in range(3):
        work.copy_(frame)
        ib.Bilateral.apply(work, SIGMA_S, SIGMA_S, 0.0, SIGMA_R, payload=args.payload)
        torch.cuda.synchronize()
    st = ib.last_stats()
    print(json.dumps({"profile": args.profile, "vertices": st["vertices"],
                      "stages_ms": {k: round(v, 4) for k, v in st.items() if k.startswith("ms_")}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--payload", default="fp32", choices=["fp32", "fp16", "bf16", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="headline and plain path only")
    ap.add_argument("--no-autotune", action="store_true",
                    help="fixed batch settings (load factor 0.5, blur axes in pairs): a launch "
                         "sequence that does not depend on the tuner, for profiler captures")
    ap.add_argument("--profile", choices=["frame4k", "frame1080p"],
                    help="run one frame through the plain path three times for a profiler "
                         "capture, and exit (nothing timed)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
