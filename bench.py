"""Benchmark: Mattes MI value+derivative evaluations per second on one B200.

Workload (one "step" = one value+derivative evaluation through the C ABI): the finest
level of the 256³ rigid registration — fixed/moving 256³ f32 blob phantoms (60 blobs,
rotation ±15°, translation ±12 mm, seeded synthetic data), VersorRigid3DTransform,
32 histogram bins, 10 % random sampling (SplitMix64, 1,677,721 samples). L2 is
flushed (a 256 MiB write) before every evaluation, outside the timed events.

  value  device time of the evaluations (CUDA events on the library's stream, first
         kernel to the result copy), inputs resident in HBM; the flush is queued on
         the same stream, so the launches of an evaluation wait behind it
  e2e    the same call timed end to end through the public C ABI from the host,
         starting from an idle stream (parameters in from host memory, value and
         derivative back to host memory, launch latency and host wait included)

Beside them, in the same line: the histogram pass's roofline, the serial CPU baseline
(median of 6 after a 2 s warm-up), the same pair with every voxel a sample (full_grid),
mean squares and correlation, a B-spline transform, one full three-level registration,
the 64-pair batched registration (device-timed per-pair completion), and the batched +
learned-initialiser form against the plain single-pair driver on held-out 128³ pairs
(the committed weights). `--storage-study`, `--initnet` and `--gemm-study` run the
512³ storage study, the initialiser's training study and its GEMM timings instead.
`--corners tiles` times the histogram pass with TMA-staged moving tiles (the opt-in
corner source) instead of the moving volume's texture.

--impl reference times the reference algorithm's CPU implementation on this host's
cores (the C++ restatement under oracle/, all threads), since the Rust reference
cannot be built here. Multi-GPU runs are independent replicas (one registration pair
per rank): weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sitk-rs_b200"))

import numpy as np  # noqa: E402

METRIC = "MI value+derivative evals/sec"
UNIT = "evals/s"
WORKLOAD = ("256^3 f32 VersorRigid3D, 32 bins, 10% random sampling (finest pyramid level of the "
            "256^3 rigid registration), value+derivative")
N = 256
BINS = 32
PCT = 0.10
SEED = 20261203
# a pose near the generating transform's inverse (versor right part, translation)
POSE = [0.021, -0.034, 0.047, 3.1, -4.2, 2.6]
# what the evaluation computes in: each sample's value, gradient and Parzen taps in
# FP32 (an exact FP64 chain wherever a decision could differ from the reference's),
# the joint histogram in u32/u64 fixed point (exact integer sums), the tail, the
# moments' cross-warp sums and the contraction in FP64
DTYPE = "f32 samples, u32/u64 fixed-point histogram, f64 reductions"


def workload_config(samples: int, world: int = 1) -> dict:
    """The `config` object of the benchmark line, the same in both arms."""
    return {"workload": WORKLOAD, "fixed": [N, N, N], "moving": [N, N, N], "bins": BINS,
            "sampling": "random 10%", "samples": samples, "seed": SEED, "transform": "VersorRigid3D",
            "pose": POSE,
            "l2": "flushed before every evaluation (256 MiB write, then a 256 MiB read of another buffer so the "
                  "write-backs fall outside the timed region)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


# the learned initialiser's weights, trained by the library's own kernels with
#   python bench.py --initnet --initnet-save sitk-rs_b200/sitk_b200/data/initnet_128cubed.npz
WEIGHTS = os.path.join(ROOT, "sitk-rs_b200", "sitk_b200", "data", "initnet_128cubed.npz")


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class ClockSampler:
    """nvidia-smi clock/throttle samples during the run (read-only queries)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        loaded = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _kernel_source_hash() -> str:
    """Hash of the device code of the evaluation kernels: sampler.cuh, eval_device.cuh
    and the kernel section of mattes.cu (host code there does not change the traffic)."""
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "sitk-rs_b200", "csrc")
    for name in ("sampler.cuh", "eval_device.cuh"):
        with open(os.path.join(csrc, name), "rb") as f:
            h.update(f.read())
    with open(os.path.join(csrc, "mattes.cu"), encoding="utf-8") as f:
        text = f.read()
    a = text.index("// Kernels. The fused evaluation")
    b = text.index("// Set-up kernels:")
    h.update(text[a:b].encode())
    return h.hexdigest()[:16]


def _traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if it was taken on the
    current kernel source."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        if d.get("source_hash") != _kernel_source_hash():
            return None
        return d["kernels"][kernel]["dram_bytes_per_launch"]
    except Exception:
        return None


def make_workload(seed: int):
    from sitk_b200 import synth
    pair = synth.config1_pair(seed, N)
    return pair


def time_oracle(pair, draw, nthreads: int, budget_s: float, min_evals: int = 1):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    g = oracle.make_geometry((N, N, N))
    center = [(N - 1) / 2.0] * 3
    times = []
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        oracle.evaluate(pair.fixed, g, pair.moving, g, BINS, 2, POSE, center, draw=draw, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
        if len(times) >= min_evals and time.perf_counter() - t_start >= budget_s:
            break
    return times


def cpu_protocol(pair, draw, nthreads: int, runs: int = 6, warm_s: float = 2.0):
    """The CPU baseline protocol: at least warm_s seconds of untimed evaluations, then
    the median of `runs` timed ones (seconds per evaluation, and the runs)."""
    time_oracle(pair, draw, nthreads, warm_s, min_evals=1)
    times = time_oracle(pair, draw, nthreads, 0.0, min_evals=runs)
    return statistics.median(times), times


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    pair = make_workload(SEED)
    draw = oracle.draw_samples(N ** 3, 2, PCT, SEED)
    cores = os.cpu_count() or 1
    # at least 2 s and `warmup` evaluations untimed, then `steps` timed evaluations
    time_oracle(pair, draw, cores, 2.0, min_evals=max(args.warmup, 1))
    times = time_oracle(pair, draw, cores, 0.0, min_evals=args.steps)
    total = sum(times)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(int(draw.size), world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full evaluations of the workload after a >= 2 s warm-up "
                                   f"(C++ FP64 restatement of the reference CPU metric, {cores} threads, "
                                   "per-thread histograms folded in thread order)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def time_registration(pair, ctx, dev):
    """One full registration of the pair as the 256³ rigid workload runs it: pyramid
    shrink 4/2/1 with sigma 2/1/0 voxels built on the device, 32 bins, 10 % random
    sampling per level, VersorRigid3D from the centred initializer, regular-step
    gradient descent (physical-shift scales, learning rate estimated once per level)
    with up to 200 iterations per level. Wall time around the whole call (level
    images, sample draws, metric set-up and every iteration), plus the target
    registration error of the result at the fixed grid's corners against the known
    generating transform. One untimed registration of a small synthetic pair runs first,
    so the first use of the pyramid and set-up kernels in the process (their modules load
    on first launch) stays out of the wall time."""
    import torch
    import sitk_b200 as sb
    from sitk_b200 import registration, synth
    w = synth.make_pair(48, 8, SEED + 1, 5.0, 3.0, (0.95, 1.05))
    wf = sb.DeviceImage.upload(w.fixed, ctx=ctx)
    wm = sb.DeviceImage.upload(w.moving, ctx=ctx)
    wc, wtr = registration.centered_initialize(wf, wm)
    registration.register_multilevel(wf, wm, sb.VersorRigid3DTransform((0.0, 0.0, 0.0), wtr, wc),
                                     shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
                                     sigmas_physical=False, bins=BINS, strategy=sb.SAMPLING_RANDOM,
                                     percentage=PCT, seed=SEED, iterations=20)
    wf.free()
    wm.free()
    f = sb.DeviceImage.upload(pair.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(pair.moving, ctx=ctx)
    c, tr = registration.centered_initialize(f, m)
    t = sb.VersorRigid3DTransform((0.0, 0.0, 0.0), tr, c)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = registration.register_multilevel(f, m, t, shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0),
                                           sigmas_physical=False, bins=BINS, strategy=sb.SAMPLING_RANDOM,
                                           percentage=PCT, seed=SEED, iterations=200)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    # truth: moving(y) = fixed(A(y − c) + c + t), so the fixed→moving point map is
    # x ↦ Aᵀ(x − c − t) + c for the rotation A
    a = np.asarray(pair.matrix)
    st = np.asarray(sb.transform_stage(t)).reshape(-1)
    mat, off = st[:9].reshape(3, 3), st[9:12]
    err = []
    for k in range(8):
        x = np.array([(N - 1) * ((k >> d) & 1) for d in range(3)], dtype=np.float64)
        truth = a.T @ (x - pair.center - pair.translation) + pair.center
        err.append(np.linalg.norm(mat @ x + off - truth))
    f.free()
    m.free()
    return {"schedule": "shrink 4/2/1, sigma 2/1/0 voxels, 200 iterations max per level",
            "wall_s": wall, "registrations_per_s": 1.0 / wall,
            "iterations": [lv.iterations for lv in res.levels],
            "stop": [lv.stop_reason for lv in res.levels],
            "evaluations": sum(lv.evaluations for lv in res.levels),
            "final_value": res.levels[-1].value,
            "tre_corners_mm": {"mean": float(np.mean(err)), "max": float(np.max(err))}}


def time_full_grid(metric, t, l2_flush, steps: int):
    """The same pair and pose with every voxel of the 256³ fixed grid a sample
    (16,777,216 samples): value+derivative evaluations, L2 flushed before each, device
    time per evaluation and per kernel (CUDA events), and the histogram pass's
    roofline: per pass S·4 B (fixed) + min(V_m, 8S)·4 B (moving)."""
    from sitk_b200.metric import enable_timing, read_timing
    S = int(metric.info()["n_samples"])
    for _ in range(3):
        l2_flush()
        metric.evaluate(t)
    out = {}
    for per_kernel in (False, True):
        enable_timing(metric, True, per_kernel=per_kernel)
        read_timing(metric)
        for _ in range(steps):
            l2_flush()
            r = metric.evaluate(t)
        ms, nev = read_timing(metric)
        enable_timing(metric, False)
        if per_kernel:
            out["kernel_ms"] = {"k_hist": ms[1] / nev, "k_deriv": ms[2] / nev}
        else:
            out["ms_per_eval"] = ms[0] / nev
    peak, peak_kind = _peaks()
    pass_bytes = S * 4 + min(N ** 3, 8 * S) * 4
    kh = out["kernel_ms"]["k_hist"]
    return {"samples": S, "evals_per_s": 1e3 / out["ms_per_eval"], "ms_per_eval": out["ms_per_eval"],
            "kernel_ms": out["kernel_ms"], "steps": steps, "value": r.value, "valid": r.valid_points,
            "roofline": {"bound": "hbm", "kernel": "k_hist", "bytes_alg_per_launch": pass_bytes,
                         "achieved": pass_bytes / (kh / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": pass_bytes / (kh / 1e3) / 1e9 / peak, "peak_source": peak_kind},
            "evaluation_roofline": {"bytes_alg_per_eval": 2 * pass_bytes,
                                    "frac": 2 * pass_bytes / (out["ms_per_eval"] / 1e3) / 1e9 / peak}}


def time_learned(args):
    """The batched + learned form against the plain single-pair GPU driver on held-out
    128³ pairs (rotation ±20°, translation ±20 mm, scale 0.9–1.1; affine, 50 bins, 10 %
    random sampling, ≤ 200 iterations): the network (the committed weights) proposes
    each pair's start, the batched optimizer refines all pairs together, and a proposal
    counts only when its refined metric value is within 1e-3 of the plain run's final
    value from the centred start, or lower. Host wall clock around synchronous calls."""
    from sitk_b200 import initnet as I
    net = I.InitNet(seed=SEED, max_batch=64)
    meta = net.load(WEIGHTS)
    spec = I.PairSpec(n=128, nblobs=40, rot_deg=20.0, trans_mm=20.0, scale=(0.9, 1.1))
    run = I.PlainRun(bins=50, percentage=0.1, iterations=200)
    first = 10_000_001
    ev = I.evaluate(net, range(first, first + args.learned_pairs), spec, run, single_pairs=args.learned_single)
    net.close()
    rps = ev["registrations_per_s"]
    accepted_rate = ev["accepted"] * rps["batched_learned"]
    return {"pairs": ev["pairs"], "held_out_seeds": [first, first + args.learned_pairs - 1],
            "accepted": ev["accepted"], "registrations_per_s": accepted_rate,
            "batched_learned_registrations_per_s": rps["batched_learned"],
            "plain_single_pair_registrations_per_s": rps["single_pair_plain"],
            "speedup_vs_plain_single_pair": accepted_rate / rps["single_pair_plain"],
            "batched_plain_registrations_per_s": rps["batched_plain"],
            "iterations": ev["iterations"], "tre_mm_p50": {k: v["p50"] for k, v in ev["tre_mm"].items()},
            "single_pair_iterations_to_plain_final": ev["single_pair_iterations_to_plain_final"],
            "weights": os.path.relpath(WEIGHTS, ROOT), "training": meta,
            "timing": "host wall clock around synchronous library calls; metric creation excluded"}


def time_batch(ctx, dev, seed: int):
    """The batched workload: 64 affine pairs, edge n ~ U{48..192} per pair (seeded),
    50 bins, 20 % random sampling, regular-step gradient descent (≤ 100 iterations)
    from the identity, all pairs advanced together (mi_batch_*: CUDA-graph replay,
    autotuned shape). Pairs are generated on the device (mi_synth_pair). Reported
    beside the single-pair driver run pair by pair on the same pairs."""
    import torch
    import sitk_b200 as sb
    from sitk_b200 import registration, synth
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = [int(v) for v in rng.integers(48, 193, size=64)]
    fixed, moving = [], []
    t0 = time.perf_counter()
    for i, n in enumerate(sizes):
        f, m, _ = synth.make_pair_device(n, 20, seed + i, 10.0, 5.0, (0.95, 1.05), ctx=ctx)
        fixed.append(f)
        moving.append(m)
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    centers = [[(n - 1) / 2.0] * 3 for n in sizes]
    start = np.tile(np.concatenate([np.eye(3).ravel(), np.zeros(3)]), (64, 1))
    batch = registration.BatchRegistration(fixed, moving, bins=50, kind=0, centers=centers,
                                           strategy=sb.SAMPLING_RANDOM, percentage=0.2,
                                           seeds=[seed + i for i in range(64)])
    t0 = time.perf_counter()
    batch.register(start, iterations=100, autotune=True)  # first call: autotune + graph build
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    params, res = batch.register(start, iterations=100, autotune=True)  # cached shape and graph
    wall = time.perf_counter() - t0
    chunk, copies, nchunks = batch.shape()
    ev = np.array([r.evaluations for r in res], dtype=np.float64)
    # device-timed: from the run's first pass to the optimizer step at which each pair stopped
    per_pair = batch.pair_seconds()
    batch.close()
    # the single-pair driver, pair after pair
    plain = []
    for i, n in enumerate(sizes):
        metric = sb.DeviceMattesMetric.from_device_sampled(fixed[i], moving[i], bins=50, strategy=sb.SAMPLING_RANDOM,
                                                           percentage=0.2, seed=seed + i)
        t = sb.AffineTransform(np.eye(3), (0.0, 0.0, 0.0), centers[i])
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        registration.register_rsgd(metric, t, iterations=100)
        plain.append(time.perf_counter() - t1)
        metric.close()
    for img in fixed + moving:
        img.free()
    return {"pairs": 64, "edge": [min(sizes), max(sizes)], "bins": 50, "sampling": "random 20%",
            "samples_total": int(sum(int(0.2 * n ** 3) for n in sizes)),
            "generate_s": gen_s, "first_call_s": tune_s, "wall_s": wall, "registrations_per_s": 64 / wall,
            "per_pair_s": {"p50": float(np.percentile(per_pair, 50)), "p99": float(np.percentile(per_pair, 99)),
                           "timing": "device global timer, run start to the step at which the pair stopped"},
            "evaluations": {"mean": float(ev.mean()), "max": int(ev.max())},
            "shape": {"chunk": chunk, "copies": copies, "chunks": nchunks},
            "single_pair_driver": {"wall_s": float(sum(plain)), "registrations_per_s": 64 / sum(plain),
                                   "per_pair_s": {"p50": float(np.percentile(plain, 50)),
                                                  "p99": float(np.percentile(plain, 99))}}}


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import sitk_b200 as sb
    from sitk_b200.metric import enable_timing, read_timing

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local_rank
    torch.cuda.set_device(dev)
    ctx = sb.Context(dev)
    pair = make_workload(SEED + rank)
    f = sb.DeviceImage.upload(pair.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(pair.moving, ctx=ctx)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=BINS, strategy=sb.SAMPLING_RANDOM,
                                                       percentage=PCT, seed=SEED)
    # the whole 256³ grid as the sample set (16.8 M samples): the survey's full-grid point
    full_metric = None if args.no_full_grid or rank != 0 else sb.DeviceMattesMetric.from_device(f, m, BINS)
    siblings = None
    if not args.no_siblings and rank == 0:
        siblings = {name: cls.from_device_sampled(f, m, strategy=sb.SAMPLING_RANDOM, percentage=PCT, seed=SEED)
                    for name, cls in (("mean_squares", sb.DeviceMeanSquaresMetric),
                                      ("correlation", sb.DeviceCorrelationMetric))}
    f.free()
    m.free()
    info = metric.info()
    S = int(info["n_samples"])
    t = sb.VersorRigid3DTransform(POSE[:3], POSE[3:], [(N - 1) / 2.0] * 3)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    from sitk_b200.metric import get_fused, set_fused
    if args.form == "fused":
        set_fused(metric, True)
    fused = get_fused(metric)
    if args.corners == "tiles":
        # the histogram pass's opt-in corner source: TMA-staged moving tiles
        from sitk_b200.metric import set_tile_staging
        set_tile_staging(metric, True)
        if full_metric is not None:
            set_tile_staging(full_metric, True)
    launches_per_eval = 1 if fused else 2
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    nflush = max(2 * l2, 256 << 20) // 4
    flush_w = torch.empty(nflush, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r = torch.zeros(nflush, dtype=torch.float32, device=f"cuda:{dev}")

    def l2_flush():
        # write a buffer larger than L2 (evicts every line of the evaluation's data),
        # then read another one, so the write's dirty lines are written back here and
        # not during the next evaluation; queued on the evaluation's stream
        with torch.cuda.stream(stream):
            flush_w.zero_()
            torch.sum(flush_r)

    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
    for _ in range(max(args.warmup, 3)):
        l2_flush()
        metric.evaluate(t)
    # settle clocks under load (untimed)
    t_end = time.perf_counter() + args.settle
    while time.perf_counter() < t_end:
        metric.evaluate(t)

    def timed_loop(per_kernel: bool):
        # The flush is queued on the evaluation's own stream with no host wait after
        # it: an evaluation's launches queue while the flush runs, and its events
        # (recorded by the library before its first launch and after its result copy)
        # measure the evaluation on the device, not the host's launch latency.
        enable_timing(metric, True, per_kernel=per_kernel)
        read_timing(metric)
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            l2_flush()
            metric.evaluate(t)
        torch.cuda.synchronize(dev)
        w = time.perf_counter() - w0
        if dist:
            dist.barrier()
        ms, nev = read_timing(metric)
        enable_timing(metric, False)
        return ms, nev, w

    # value: whole evaluations, two events each
    ms, nev, wall = timed_loop(False)
    dev_ms = ms[0]
    # kernel durations for the roofline: events after every kernel as well
    ms_k, nev_k, _ = timed_loop(True)

    # End to end: the call as a user makes it, from an idle stream: torch events
    # bracket the whole synchronous call (parameter upload as kernel arguments,
    # launches, the device-to-host copy of value and derivative, the host wait).
    ev_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    last = None
    for i in range(args.steps):
        l2_flush()
        torch.cuda.synchronize(dev)
        ev_s[i].record(stream)
        last = metric.evaluate(t)
        ev_e[i].record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in zip(ev_s, ev_e))
    if dist:
        tt = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_ms, e2e_ms = tt.tolist()
    if sampler:
        sampler.stop()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    per_step_ms = dev_ms / args.steps
    value = world * args.steps / (dev_ms / 1e3)
    e2e_value = world * args.steps / (e2e_ms / 1e3)
    vm = N ** 3
    pass_bytes = S * 4 + min(vm, 8 * S) * 4  # one pass: fixed f32 + moving f32 (per-unit figure × S)
    if fused:
        kern = {"k_eval": ms_k[1] / nev_k}
        dom, bytes_alg = "k_eval", 2 * pass_bytes  # both passes in one launch
    else:
        hname = "k_hist_tile" if args.corners == "tiles" else "k_hist"
        kern = {hname: ms_k[1] / nev_k, "k_deriv": ms_k[2] / nev_k}  # k_deriv forms the tail itself
        dom, bytes_alg = hname, pass_bytes
    peak, peak_kind = _peaks()
    achieved = bytes_alg / (kern[dom] / 1e3) / 1e9
    traffic = _traffic(dom)

    # serial CPU baseline on a bounded sample (rank 0, N=1 only)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        draw = oracle.draw_samples(vm, 2, PCT, SEED)
        med, times = cpu_protocol(pair, draw, 1)
        cpu = {"value": 1.0 / med, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"median of {len(times)} full evaluations of the same workload after a >= 2 s "
                         "warm-up, serial C++ FP64 restatement of the reference CPU metric "
                         f"(runs {min(times):.3f}-{max(times):.3f} s)"}

    clocks = sampler.summary() if sampler else None
    sib = None
    if siblings:
        # the reference's other device metrics on the same samples and pose: value +
        # derivative, device time per evaluation (events), L2 flushed before each
        sib = {}
        for name, sm in siblings.items():
            for _ in range(3):
                sm.evaluate(t)
            enable_timing(sm, True)
            read_timing(sm)
            for _ in range(min(args.steps, 50)):
                l2_flush()
                sm.evaluate(t)
            sms, snev = read_timing(sm)
            enable_timing(sm, False)
            sib[name] = {"evals_per_s": snev / (sms[0] / 1e3), "ms_per_eval": sms[0] / snev,
                         "launches_per_eval": 1 if name == "mean_squares" else 2}
            sm.close()
        # the same metric through a cubic B-spline transform (mesh 8³ over the fixed
        # image, coefficients N(0, 1 mm), seeded): value + derivative of all 3·11³
        # coefficients, timed end to end on the stream (torch events around the call)
        from sitk_b200.transforms import BSplineTransform
        from sitk_b200.metric import geometry
        bst = BSplineTransform.from_image_domain(geometry((N, N, N)), (8, 8, 8))
        bst.set_parameters(np.random.default_rng(SEED).standard_normal(bst.nparams))
        for _ in range(3):
            metric.evaluate(bst)
        bs_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        for e0, e1 in bs_ev:
            l2_flush()
            torch.cuda.synchronize(dev)
            e0.record(stream)
            metric.evaluate(bst)
            e1.record(stream)
        torch.cuda.synchronize(dev)
        bms = sum(a.elapsed_time(b) for a, b in bs_ev) / len(bs_ev)
        sib["mattes_bspline_8x8x8"] = {"evals_per_s": 1e3 / bms, "ms_per_eval": bms, "parameters": bst.nparams,
                                       "timing": "end to end per call (events around the synchronous call)"}
    full = None
    if full_metric is not None:
        full = time_full_grid(full_metric, t, l2_flush, min(args.steps, 50))
        full_metric.close()
    reg = None if args.no_registration else time_registration(pair, ctx, dev)
    learned = None
    if not args.no_learned and rank == 0 and os.path.exists(WEIGHTS):
        learned = time_learned(args)
    batch = None if args.no_batch else time_batch(ctx, dev, SEED)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE, "data": "synthetic",
        "config": workload_config(S, world),
        "form": "fused (one cooperative kernel)" if fused else "split (two kernels)",
        "corners": ("TMA-staged moving tiles" if args.corners == "tiles" else "moving-volume texture"),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * (6 + 3),
                "d2h_bytes_per_step": 8 * (2 + 6)},
        "gpu_launches": launches_per_eval * args.steps,  # in the timed loop of `value`
        "kernel_ms": kern,
        "sample_points_per_s": 2 * S * value / world,
        "wall_ms_per_step": 1e3 * wall / args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "bytes_alg_per_launch": bytes_alg},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "result": {"value": last.value, "valid": last.valid_points},
        "full_grid": full,
        "registration": reg,
        "batch": batch,
        "learned": learned,
        "other_metrics": sib,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_initnet(args, rank: int, world: int, local_rank: int):
    """The learned-initialiser study on 128³ pairs (rotation ±20°, translation ±20 mm,
    scale 0.9–1.1): labelled set generated and registered on the device, network
    trained by the library's tensor-core kernels, then held-out pairs registered
    from the centred initialiser and from the network's proposal. The headline is
    the batched + learned form's rate of registrations that reach the plain run's
    final metric value within 1e-3, against the plain single-pair GPU driver started
    from the centred initialiser. One GPU; other ranks exit."""
    import torch
    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    from sitk_b200 import initnet as I
    spec = I.PairSpec(n=128, nblobs=40, rot_deg=20.0, trans_mm=20.0, scale=(0.9, 1.1))
    run = I.PlainRun(bins=50, percentage=0.1, iterations=200)
    data = I.labelled_set(range(1, 1 + args.initnet_train), spec, run)
    label_s = data["seconds"]
    c = [(spec.n - 1) / 2.0] * 3
    label_tre = [I.target_error(lb, t, c, 0.3 * spec.n) for lb, t in zip(data["labels"], data["truth"])]
    net = I.InitNet(seed=SEED, max_batch=64)
    losses, train_s = I.train(net, data["x"], data["labels"], epochs=args.initnet_epochs)
    del data
    if args.initnet_save:
        os.makedirs(os.path.dirname(os.path.abspath(args.initnet_save)), exist_ok=True)
        net.save(args.initnet_save, training_pairs=args.initnet_train, epochs=args.initnet_epochs, seed=SEED,
                 first_seed=1, loss_first_epoch=losses[0], loss_last_epoch=losses[-1],
                 command=f"python bench.py --initnet --initnet-train {args.initnet_train} "
                         f"--initnet-epochs {args.initnet_epochs} --initnet-save <path>")
    ev = I.evaluate(net, range(10_000_001, 10_000_001 + args.initnet_test), spec, run,
                    single_pairs=args.initnet_single)
    net.close()
    rps = ev["registrations_per_s"]
    value = ev["accepted"] * rps["batched_learned"]
    line = {
        "metric": "registrations/s reaching the plain run's final MI within 1e-3 (batched + learned initialiser)",
        "value": value, "unit": "registrations/s", "n_gpus": 1, "steps": args.initnet_test, "warmup": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 metric reductions, bf16 network operands (f32 accumulation)", "data": "synthetic",
        "config": {"workload": "learned initialiser: 128^3 f32 blob pairs (40 blobs), rotation +-20 deg, "
                               "translation +-20 mm, scale 0.9-1.1; affine, 50 bins, 10% random sampling, "
                               "regular-step gradient descent <= 200 iterations",
                   "training_pairs": args.initnet_train, "epochs": args.initnet_epochs,
                   "test_pairs": args.initnet_test},
        "plain_gpu_single_pair": {"registrations_per_s": rps["single_pair_plain"], "pairs": args.initnet_single},
        "speedup_vs_plain_gpu": value / rps["single_pair_plain"],
        "labels": {"seconds": label_s, "tre_to_truth_mm_p50": float(np.median(label_tre))},
        "training": {"seconds": train_s, "loss_first_epoch": losses[0], "loss_last_epoch": losses[-1]},
        "study": ev,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gemm_study(args, rank: int, world: int, local_rank: int):
    """The learned initialiser's tensor-core GEMM (mi_gemm_bf16_tn: C = A·Bᵀ, BF16
    operands, FP32 accumulation in tensor memory) on the shapes its layers run for a
    64-pair batch (forward im2col products and the weight gradients, whose K is the
    batch's voxel count), plus square shapes where the tensor cores, not memory, bound
    it. Each call is synchronous; per-call device time from CUDA events around
    `--steps` calls on the library's stream (the per-call launch and result check are
    in it, which dominates the small shapes: the ncu launch list gives their kernel
    time). Results are checked against torch's FP32 product of the same operands."""
    import ctypes
    import torch
    import sitk_b200 as sb
    from sitk_b200 import _lib
    if rank != 0:
        return 0
    torch.cuda.set_device(local_rank)
    ctx = sb.Context(local_rank)
    L = _lib.load()
    L.mi_gemm_bf16_tn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.mi_gemm_bf16_tn.restype = ctypes.c_int
    stream = torch.cuda.ExternalStream(ctx.stream(), device=local_rank)
    shapes = [("conv0 forward", 262144, 16, 56), ("conv1 forward", 32768, 32, 432), ("conv2 forward", 4096, 64, 864),
              ("conv3 forward", 512, 128, 1728), ("fc1 forward", 64, 256, 1024),
              ("conv0 weight gradient", 16, 56, 262144), ("conv1 weight gradient", 32, 432, 32768),
              ("conv2 weight gradient", 64, 864, 4096), ("square 4096", 4096, 4096, 4096),
              ("square 8192", 8192, 8192, 8192)]
    if args.gemm_shape:
        # one product only (e.g. for a profiler capture): "MxNxK"
        M_, N_, K_ = (int(x) for x in args.gemm_shape.lower().split("x"))
        shapes = [(f"{M_}x{N_}x{K_}", M_, N_, K_)]
    peak_t = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak_t = float(json.load(fh)["bf16_tflops"])
    except Exception:
        peak_t = 1590.0
    hbm, _ = _peaks()
    out = []
    g = torch.Generator(device="cpu").manual_seed(SEED)
    for name, M, N, K in shapes:
        A = torch.randn((M, K), generator=g).to(torch.bfloat16).cuda()
        B = torch.randn((N, K), generator=g).to(torch.bfloat16).cuda()
        C = torch.empty((M, N), dtype=torch.float32, device="cuda")

        def call():
            _lib.check(L.mi_gemm_bf16_tn(ctx.handle, M, N, K, A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N),
                       ctx.handle)

        for _ in range(2):
            call()
        ref = (A.float() @ B.float().T)
        err = float((C - ref).abs().max() / ref.abs().max())
        reps = max(3, min(args.steps, 50))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        flops = 2.0 * M * N * K
        bytes_ = 2.0 * (M * K + N * K) + 4.0 * M * N
        out.append({"shape": name, "M": M, "N": N, "K": K, "ms_per_call": ms, "tflops": flops / (ms / 1e3) / 1e12,
                    "tflops_frac_of_measured_bf16": flops / (ms / 1e3) / 1e12 / peak_t,
                    "gbs": bytes_ / (ms / 1e3) / 1e9, "gbs_frac_of_measured_hbm": bytes_ / (ms / 1e3) / 1e9 / hbm,
                    "max_rel_err_vs_fp32": err})
        del A, B, C, ref
    print(json.dumps({"metric": "tensor-core GEMM (mi_gemm_bf16_tn) per call", "unit": "TFLOP/s", "n_gpus": 1,
                      "dtype": "bf16 operands, f32 accumulation", "peak_bf16_tflops": peak_t,
                      "peak_hbm_gbs": hbm, "shapes": out}), flush=True)
    return 0


def bf16_round(v):
    """f32 → nearest BF16 (ties to even), widened back to f32 (finite inputs)."""
    b = np.ascontiguousarray(v, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(v))


def run_storage_study(args, rank: int, world: int, local_rank: int):
    """The large-volume case: n³ (default 512³) f32 blob pair (120 blobs, rotation
    ±10°, translation ±5 mm), Euler3D, 64 bins, 20 % random sampling. The metric runs
    with the moving volume stored as f32 and as BF16; each is timed (device events,
    L2 flushed before every evaluation) and compared with the FP64 oracle on the f32
    volumes (the storage error) — and the BF16 form also with the oracle on the
    rounded volume (the parity contract). One GPU; other ranks exit."""
    import torch

    import sitk_b200 as sb
    from sitk_b200 import synth
    from sitk_b200.metric import enable_timing, read_timing
    if rank != 0:
        return 0
    dev = local_rank
    torch.cuda.set_device(dev)
    ctx = sb.Context(dev)
    n = args.storage_n
    bins, pct = 64, 0.2
    f, m, _ = synth.make_pair_device(n, 120, SEED + 3, 10.0, 5.0, None, ctx=ctx)
    c = [(n - 1) / 2.0] * 3
    t = sb.Euler3DTransform((0.02, -0.015, 0.03), (0.8, -0.6, 0.4), c)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    nflush = max(2 * l2, 256 << 20) // 4
    flush_w = torch.empty(nflush, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r = torch.zeros(nflush, dtype=torch.float32, device=f"cuda:{dev}")
    peak, peak_kind = _peaks()
    runs = {}
    for storage in ("f32", "bf16"):
        metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=bins, strategy=sb.SAMPLING_RANDOM,
                                                           percentage=pct, seed=SEED, moving_storage=storage)
        S = int(metric.info()["n_samples"])
        for _ in range(3):
            metric.evaluate(t)
        enable_timing(metric, True, per_kernel=True)
        read_timing(metric)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush_w.zero_()
                torch.sum(flush_r)
            mv = metric.evaluate(t)
        torch.cuda.synchronize(dev)
        ms, nev = read_timing(metric)
        enable_timing(metric, False)
        b_m = 4 if storage == "f32" else 2
        pass_bytes = S * 4 + min(n ** 3, 8 * S) * b_m
        k_hist = ms[1] / nev
        runs[storage] = {"value": mv.value, "derivative": [float(x) for x in mv.derivative],
                         "valid": mv.valid_points, "ms_per_eval": ms[0] / nev, "evals_per_s": nev / (ms[0] / 1e3),
                         "kernel_ms": {"k_hist": k_hist, "k_deriv": ms[2] / nev},
                         "roofline_k_hist": {"bytes_alg": pass_bytes,
                                             "achieved_gbs": pass_bytes / (k_hist / 1e3) / 1e9,
                                             "frac": pass_bytes / (k_hist / 1e3) / 1e9 / peak}}
        metric.close()
    fixed_h = f.to_host()
    moving_h = m.to_host()
    f.free()
    m.free()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    g = oracle.make_geometry((n, n, n))
    draw = oracle.draw_samples(n ** 3, 2, pct, SEED)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = oracle.evaluate(fixed_h, g, moving_h, g, bins, t.kind, t.params, t.fixed_params, draw=draw, nthreads=cores)
    oracle_s = time.perf_counter() - t0
    ref_b = oracle.evaluate(fixed_h, g, bf16_round(moving_h), g, bins, t.kind, t.params, t.fixed_params, draw=draw,
                            nthreads=cores)

    def err(run, r):
        d = np.asarray(run["derivative"])
        rd = np.asarray(r["derivative"])
        return {"value_rel": abs(run["value"] - r["value"]) / abs(r["value"]),
                "derivative_max_abs_over_max": float(np.max(np.abs(d - rd)) / np.max(np.abs(rd))),
                "valid_equal": run["valid"] == r["valid"]}

    line = {
        "metric": "MI value+derivative evals/sec, moving volume stored f32 and bf16",
        "value": runs["bf16"]["evals_per_s"], "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": 3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (bf16 storage)",
        "data": "synthetic",
        "config": {"workload": f"{n}^3 f32 blob pair, Euler3D, 64 bins, 20% random sampling, value+derivative",
                   "samples": int(draw.size), "l2": "flushed before every evaluation"},
        "runs": runs,
        "error_vs_fp64_oracle_on_f32_volumes": {"f32": err(runs["f32"], ref), "bf16": err(runs["bf16"], ref)},
        "bf16_vs_oracle_on_rounded_volume": err(runs["bf16"], ref_b),
        "oracle": {"value": ref["value"], "derivative": [float(x) for x in ref["derivative"]],
                   "seconds": oracle_s, "threads": cores},
        "peak": {"hbm_gbs": peak, "source": peak_kind},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-registration", action="store_true",
                    help="skip the full three-level registration run reported beside the metric")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 64-pair batched registration run reported beside the metric")
    ap.add_argument("--no-siblings", action="store_true",
                    help="skip the mean-squares and correlation timings reported beside the metric")
    ap.add_argument("--form", default="split", choices=["split", "fused"],
                    help="launch form of an evaluation: two kernels, or one cooperative kernel")
    ap.add_argument("--gemm-shape", default=None,
                    help="with --gemm-study: time this one product only, given as MxNxK")
    ap.add_argument("--corners", default="texture", choices=["texture", "tiles"],
                    help="corner source of the histogram pass: the moving volume's texture, or TMA-staged tiles")
    ap.add_argument("--settle", type=float, default=1.0,
                    help="seconds of untimed evaluations before the timed region (clock ramp)")
    ap.add_argument("--initnet", action="store_true",
                    help="run the learned-initialiser study instead of the metric benchmark")
    ap.add_argument("--initnet-train", type=int, default=20000)
    ap.add_argument("--initnet-test", type=int, default=512)
    ap.add_argument("--initnet-epochs", type=int, default=20)
    ap.add_argument("--initnet-single", type=int, default=32)
    ap.add_argument("--initnet-save", default=None,
                    help="write the trained network's weights to this .npz file")
    ap.add_argument("--no-full-grid", action="store_true",
                    help="skip the full-grid (every voxel a sample) point reported beside the metric")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the batched + learned-initialiser comparison reported beside the metric")
    ap.add_argument("--learned-pairs", type=int, default=128)
    ap.add_argument("--learned-single", type=int, default=16)
    ap.add_argument("--storage-study", action="store_true",
                    help="run the f32/bf16 moving-storage study (512^3) instead of the metric benchmark")
    ap.add_argument("--storage-n", type=int, default=512)
    ap.add_argument("--gemm-study", action="store_true",
                    help="time the learned initialiser's tensor-core GEMM on its layer shapes instead")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.initnet:
        return run_initnet(args, rank, world, local_rank)
    if args.storage_study:
        return run_storage_study(args, rank, world, local_rank)
    if args.gemm_study:
        return run_gemm_study(args, rank, world, local_rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
