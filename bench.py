#!/usr/bin/env python
"""Benchmark: vertex-substeps/s of the batched Stable Cosserat Rods substep on B200.

Workload (one "step" = one advance(1/30 s) of every scene = 34 substeps x 8 Newton
iterations): the batched uneven-scene configuration - up to 512 independent random-walk
yarn piles (k ~ U{1..64} yarns, 64..4096 vertices per yarn, log-uniform), added until the
next scene would pass 8,388,608 vertices; per-scene kBend log-uniform in [1e-9, 1e-7],
kStretch 2e-2, kCollision 1e-7, mu 0.3, yarn radius 0.5 mm, gravity -9.8, first vertex of
each yarn pinned.  Synthetic, seeded (no dataset exists for this path).

  python bench.py [--gpus N --steps K --warmup W]      # the CUDA engine (one JSON line)
  python bench.py --impl reference ...                 # the reference algorithm on the host

Under torchrun the scenes of the one batch are split over the ranks by greedy bin packing of
their vertex counts (strong scaling, no collective on the data path); the time is the max over
ranks of the device time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "vertex-substeps/s on 1 B200, batched vs plain at ≤1e-4 rel err vs FP64; HBM %"
UNIT = "vertex-substeps/s"
FRAME = 1.0 / 30.0
MAX_H = 1e-3
SUBSTEPS = int(np.ceil(np.float32(FRAME) / np.float32(MAX_H)))  # 34
NUM_ITR = 8
SEED = 7
# Algorithmic bytes per vertex per Newton iteration (position solve 92 + orientation 84)
# plus 4 bytes per contact-list entry: the per-unit figure of the roofline.
ITER_BYTES_BASE = 176
ITER_BYTES_PER_CONTACT = 4


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-plain", action="store_true", help="skip the plain per-scene advance() loop")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--cap", type=int, default=8388608, help="vertex cap of the batched workload")
    p.add_argument("--shape", default="", help="fixed Newton kernel shape threads,lanes,pipelined (default: autotune)")
    p.add_argument("--workload", default="batched", choices=["batched", "serve", "twist", "pile", "readme"])
    p.add_argument("--pile-frames", type=int, default=60, help="pile: frames")
    p.add_argument("--readme-frames", type=int, default=150, help="readme: frames")
    p.add_argument("--rate", type=float, default=4.0, help="serve: Poisson arrival rate (requests/s)")
    p.add_argument("--duration", type=float, default=10.0, help="serve: arrival window (s)")
    p.add_argument("--frames", type=int, default=30, help="serve: frames per request; twist: frames (0 = 300)")
    p.add_argument("--every", type=int, default=30, help="twist: sample interval in frames")
    p.add_argument("--gravity", type=float, default=-9.8, help="twist: gravity along y (m/s^2)")
    p.add_argument("--budget-gb", type=float, default=120.0, help="serve: device-memory budget")
    p.add_argument("--setup-threads", type=int, default=4, help="serve: host threads generating request geometry")
    p.add_argument("--max-batch-verts", type=int, default=8_000_000, help="serve: vertices per frame (0: budget only)")
    p.add_argument("--drain", type=float, default=30.0, help="serve: seconds the admitted requests may finish in")
    p.add_argument("--alone-sample", type=int, default=40, help="serve: requests timed alone")
    return p.parse_args()


def workload_desc(spec):
    yarns, lens, _ = spec
    n = int(sum(int(l.sum()) for l in lens))
    return n, {
        "workload": "batched uneven scenes: %d random-walk yarn piles, %d vertices, %d yarns" % (
            len(yarns), n, int(sum(yarns))),
        "scenes": len(yarns),
        "vertices": n,
        "substeps_per_step": SUBSTEPS,
        "newton_iterations": NUM_ITR,
        "step": "advance(1/30 s) of the whole batch (%d substeps of h=1/%d s)" % (SUBSTEPS, SUBSTEPS * 30),
        "l2": "inputs larger than L2 (one Newton iteration alone moves ~260 B of DRAM traffic per vertex, "
              "%.1f GB for %.1fM vertices, against 126 MB of L2), no flush" % (n * 260e-9, n / 1e6),
        "seed": SEED,
        "parallelism": "one GPU",
    }


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.th.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-vertex DRAM bytes of one Newton iteration from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_iter_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def oracle_sample(spec, target_verts, mode, seed=SEED):
    """The first scenes of the batch totalling >= target_verts vertices, assembled and
    configured on the oracle side (same geometry and parameters as the GPU batch)."""
    import oracle
    from yarnball_b200 import scenes

    yarns, lens, kbend = spec
    k, tot = 0, 0
    while k < len(yarns) and tot < target_verts:
        tot += int(lens[k].sum())
        k += 1
    # the same seeded geometry as the GPU batch, from the host-only build of the generator
    # (this CPU path loads no CUDA library); scene s depends only on (seed, s)
    flat = np.concatenate(lens[:k]).astype(np.int32)
    pos_all = oracle.random_walks_batch(seed, yarns[:k], flat)
    counts = [int(l.sum()) for l in lens[:k]]
    offs = np.concatenate([[0], np.cumsum(counts)])
    pos_list = [pos_all[offs[s]:offs[s + 1]] for s in range(k)]
    orc = oracle.build_scenes(pos_list, lens[:k], kbend[:k], scenes.PILE_META, mode=mode)
    return orc, k, tot


def cpu_baseline_sample(spec, target_verts=1_000_000, reps_seconds=10.0, mode=None):
    """The oracle (FP32 as the reference writes it, OpenMP over all host cores) on the first
    scenes of the batch totalling >= target_verts vertices: one substep per repetition."""
    import oracle
    from yarnball_b200 import scenes

    orc, k, tot = oracle_sample(spec, target_verts, oracle.FP32 if mode is None else mode)
    h = float(np.float32(FRAME) / np.float32(SUBSTEPS))
    reps, t0 = 0, time.perf_counter()
    while True:
        orc.advance(h, h)
        reps += 1
        el = time.perf_counter() - t0
        if el >= reps_seconds or reps >= 50:
            break
    return {"value": tot * reps / el, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port",
            "sample": "first %d scenes (%d vertices) of the same batch, %d substep(s) of h=1/%d s, FP32 OpenMP"
                      % (k, tot, reps, SUBSTEPS * 30), "seconds": el}


def run_reference(args):
    """Reference arm: the reference's algorithm on the host cores (the reference has no CPU path
    for it, so this is the CPU oracle's restatement, pinned to the reference's kernels by the
    tests), FP32, all host threads; each step = one substep of a bounded sample of the batch.
    Loads no CUDA library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    from yarnball_b200 import scenes

    spec = scenes.batched_spec(SEED, 512, args.cap)
    _, cfg = workload_desc(spec)
    orc, k, tot = oracle_sample(spec, 400_000, oracle.FP32)
    # the workload is the GPU arm's; each timed step is a bounded sample of it
    cfg["timed_sample"] = {
        "scenes": k, "vertices": tot, "yarns": int(sum(spec[0][:k])), "substeps_per_step": 1,
        "what": "the first %d scenes (%d vertices) of this workload, one substep of h=1/%d s per step "
                "(the metric is per vertex-substep, as the GPU arm's)" % (k, tot, SUBSTEPS * 30)}
    h = float(np.float32(FRAME) / np.float32(SUBSTEPS))
    for _ in range(args.warmup):
        orc.advance(h, h)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.advance(h, h)
    el = time.perf_counter() - t0
    value = tot * args.steps / el
    cores = oracle.max_threads()
    sample = "first %d scenes (%d vertices) of the batch, one substep of h=1/%d s per step" % (k, tot, SUBSTEPS * 30)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU implementation of the substep; this arm runs the oracle's CPU "
                "restatement of it (oracle/, strict Jacobi, FP32, OpenMP), which the tests pin to the "
                "reference's own kernels (compiled unchanged from its sources for the GPU by oracle/refbuild)",
    }
    print(json.dumps(out))


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from yarnball_b200 import scenes, sharding

    # One batch for the whole job: its scenes are split over the ranks by greedy bin packing of
    # their vertex counts (no collective on the data path; strong scaling).
    spec = scenes.batched_spec(SEED, 512, args.cap)
    _, cfg = workload_desc(spec)
    sizes = [int(l.sum()) for l in spec[1]]
    parts = sharding.partition_scenes(sizes, world)
    mine = parts[rank]
    n = int(sum(sizes[i] for i in mine))
    if world > 1:
        cfg["parallelism"] = "scenes split over %d GPUs by greedy bin packing (strong scaling)" % world
        cfg["vertices_per_rank_max"] = int(max(sum(sizes[i] for i in p) for p in parts))
    sim, _ = scenes.build_batched(seed=SEED, spec=spec, indices=mine)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        sim.advance(FRAME)
    if args.shape:
        # A fixed Newton-kernel shape "threads,lanes,pipelined" (lanes 0 = balanced kernel).
        tune_threads, tune_lanes, tune_pipe = [int(x) for x in args.shape.split(",")]
        sim.set_tuning(tune_threads, tune_lanes, True, bool(tune_pipe))
        tune_ms = None
    else:
        # Autotuner: Newton-kernel shape (threads per block, lanes per vertex) timed on this state.
        tune_threads, tune_lanes, tune_pipe, tune_ms = sim.autotune()
    cfg["newton_kernel_shape"] = {"threads": tune_threads, "lanes_per_vertex": tune_lanes, "pipelined": tune_pipe,
                                  "autotune_ms_per_launch": tune_ms}
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        gpu_id = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        gpu_id = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]
    # The host arrays keep the state at the start of the timed frames: the end-to-end run below
    # uploads it again and replays the same frames, so both numbers measure the same work.
    sim.download()
    clocks = ClockSampler(gpu_id)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = sim.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sim.advance(FRAME)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop()
    launches = sim.launch_count() - l0
    ms = e0.elapsed_time(e1)
    ms_max, n_all = sharding.reduce_timing(ms, n, device="cuda")
    value = n_all * SUBSTEPS * args.steps / (ms_max / 1e3)

    # Per-kernel device times of one more frame (events around each kernel class).
    prof_ms, prof_launches = sim.profile_advance(FRAME)
    total_pairs, segs_with, max_cols = sim.collisionStats()
    nseg = int(((sim.verts["flags"] & 2) != 0).sum())
    cbar = 2.0 * total_pairs / max(nseg, 1)
    iter_launches = max(1, prof_launches["iter"])
    iter_ms = prof_ms["iter"] / iter_launches
    bytes_per_launch = n * (ITER_BYTES_BASE + ITER_BYTES_PER_CONTACT * cbar)
    achieved = bytes_per_launch / (iter_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    tr = load_traffic()
    traffic, traffic_src = None, None
    if tr and tr.get("vertices") == n and tr.get("warmup") == args.warmup:
        # captured on this workload at the first Newton launch of the timed region; the mean
        # launch of the region has more contacts, so scale by the algorithmic bytes
        traffic = tr["dram_bytes_per_launch"] * bytes_per_launch / tr["algorithmic_bytes_per_launch"]
        traffic_src = ("ncu capture of the first Newton launch of this workload after %d warm-up frames "
                       "(c = %.2f), scaled to the mean launch's algorithmic bytes (%s)") % (
            tr["warmup"], tr["cbar_at_capture"], tr["summary"])
    elif tr:
        # another state or size: the captured traffic per algorithmic byte
        traffic = tr["dram_bytes_per_launch"] * bytes_per_launch / tr["algorithmic_bytes_per_launch"]
        traffic_src = "ncu capture (%d vertices, %d warm-up frames, c = %.2f) scaled by the algorithmic bytes (%s)" % (
            tr["vertices"], tr["warmup"], tr["cbar_at_capture"], tr["summary"])
    prof_total = sum(prof_ms.values())
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": traffic, "traffic_source": traffic_src,
        "kernel": "k_iter (fused Newton position solve + orientation update)",
        "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
        "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": iter_ms, "cbar": cbar,
        "kernel_share": {k: v / prof_total for k, v in prof_ms.items()},
        "kernel_ms_per_frame": prof_ms,
    }

    # End to end through the public API with host buffers: upload + advance + download, from
    # the state the timed frames started from (the host arrays still hold it; upload restores
    # positions, velocities and rotors, and clears the Kahan terms), for as many frames.
    h2d = n * (32 + 12 + 16 + 16)
    d2h = n * (32 + 12 + 16)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    f0.record(stream)
    e2e_steps = args.steps
    for _ in range(e2e_steps):
        sim.upload()
        sim.advance(FRAME)
        sim.download()
    f1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    ems, _ = sharding.reduce_timing(f0.elapsed_time(f1), n, device="cuda")
    e2e = {"value": n_all * SUBSTEPS * e2e_steps / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": e2e_steps, "wall_s": wall,
           "api": "yb_upload + yb_advance + yb_download (pinned host arrays)",
           "frames": "the timed frames again, from the state uploaded at the first step"}

    diag = sim.diagnostics()
    pens = sim.penetrations()
    min_dist = sim.min_pair_distance()
    plain = None
    if not args.no_plain and rank == 0 and world == 1:
        plain = run_plain(spec, stream, (tune_threads, tune_lanes, tune_pipe))
    sim.close()
    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_baseline_sample(spec)
    acc = None
    if rank == 0:
        acc = accuracy_sample(spec, (tune_threads, tune_lanes, tune_pipe))

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches) * world,
            "clocks": ck, "plain": plain,
            "batched_over_plain": (value / plain["value"]) if plain else None,
            "contacts": {"pairs": total_pairs, "segments_with_contacts": segs_with, "max_per_segment": max_cols,
                         "cbar": cbar},
            # every listed contact at the start of every substep of the run (warm-up included):
            # centre-lines crossing (distance 0) and hard cores touching (distance <= 2 radius)
            "interpenetrations": {"min_centre_line_distance_m": min_dist, "zero_distance": int(min_dist <= 0.0),
                                  "hard_core_contacts": pens, "two_radius_m": 2 * float(scenes.RADIUS)},
            "diagnostics": diag, "accuracy": acc,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def accuracy_sample(spec, shape, target_verts=1_000_000):
    """FP32 production build against the FP64 build of the same kernels (which the tests tie to
    the FP64 CPU oracle) on the first scenes of the workload (about 1M vertices), one frame from
    the same state: max position difference over max displacement."""
    from yarnball_b200 import scenes, sharding

    yarns, lens, kbend = spec
    k, tot = 0, 0
    while k < len(lens) and tot < target_verts:
        tot += int(lens[k].sum())
        k += 1
    sub = sharding.subset_spec(spec, list(range(k)))
    out = {}
    for prec in ("fp32", "fp64"):
        sim, _ = scenes.build_batched(seed=SEED, spec=sub, precision=prec)
        sim.set_tuning(shape[0], shape[1], True, bool(shape[2]))
        x0 = sim.read_state_f64()[0]
        sim.advance(FRAME)
        out[prec] = sim.read_state_f64()[0]
        sim.close()
    disp = float(np.abs(out["fp64"] - x0).max())
    err = float(np.abs(out["fp32"] - out["fp64"]).max())
    return {"vs": "FP64 build of the same kernels", "rel_err_1_frame": err / disp, "max_abs_err_m": err,
            "max_displacement_m": disp, "vertices": tot, "scenes": k, "frames": 1, "bound": 1e-4}


def run_plain(spec, stream, shape):
    """The drop-in path: one Sim per scene, advance() called scene after scene."""
    import torch

    from yarnball_b200 import scenes

    yarns, lens, kbend = spec
    flat = np.concatenate(lens).astype(np.int32)
    pos_all = scenes.random_walks_batch(SEED, yarns, flat)
    counts = [int(l.sum()) for l in lens]
    sims = []
    off = 0
    for s in range(len(yarns)):
        sm = scenes.Sim(counts[s])
        scenes.fill_yarns(sm, pos_all[off:off + counts[s]], lens[s], pin_first=True)
        for k, val in scenes.PILE_META.items():
            setattr(sm.meta, k, val)
        sm.configure()
        sm.setKBend(kbend[s])
        sm.setKStretch(2e-2)
        sm.maxH = MAX_H
        sm.upload()
        sm.set_stream(stream.cuda_stream)
        sm.set_tuning(shape[0], shape[1], True, shape[2])
        sims.append(sm)
        off += counts[s]
    for sm in sims:
        sm.advance(FRAME)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = 2
    l0 = sum(sm.launch_count() for sm in sims)
    e0.record(stream)
    for _ in range(steps):
        for sm in sims:
            sm.advance(FRAME)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sum(sm.launch_count() for sm in sims) - l0
    for sm in sims:
        sm.close()
    n = sum(counts)
    return {"value": n * SUBSTEPS * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "gpu_launches": int(launches), "scenes": len(sims)}


def run_serve(args):
    """Serving loop: Poisson arrivals in real time (config 5: --rate 200 --duration 60),
    continuous batching on one GPU with request geometry generated on host threads while the
    frames run (the frame thread makes every CUDA call).
    Arrivals stop after the window; the requests already in the batch then finish (no new
    admissions, at most --drain seconds) and the rest of the queue is reported as not served.
    Beside it, a sample of the same requests served one at a time through plain advance().
    Under torchrun every rank runs its own server on its GPU and takes every world-th request of
    the one arrival stream (sharding.route_requests); no collective on the data path, rank 0
    gathers the reports and prints the job's line."""
    import torch

    from yarnball_b200 import serve, sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    all_reqs = serve.poisson_requests(args.rate, args.duration, frames=args.frames)
    mine = set(sharding.route_requests([r.id for r in all_reqs], world, rank))
    reqs = [r for r in all_reqs if r.id in mine]
    server = serve.Server(budget_bytes=args.budget_gb * 1e9, shape=(128, 0), stream=torch.cuda.Stream(),
                          setup_threads=args.setup_threads, max_batch_vertices=args.max_batch_verts or None)
    if dist:
        dist.barrier()
    pending = list(reqs)
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while pending and pending[0].arrival <= now:
            server.submit(pending.pop(0))
        in_window = now <= args.duration
        if not in_window and (now > args.duration + args.drain or not any(
                r.done_frames < r.frames for r in server.active)):
            break
        if not server.busy():
            if not pending:
                break
            time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
            continue
        server.step(now, admit=in_window)
        done_t = time.perf_counter() - t0
        for r in server.finished:
            if r.finished_at is None:
                r.finished_at = done_t
    wall = time.perf_counter() - t0
    arrived = [r for r in reqs if r.arrival <= min(wall, args.duration)]
    done = [r for r in reqs if r.finished_at is not None]
    report = {
        "wall": wall, "served_work": float(sum(server.frame_sizes)) * SUBSTEPS,  # vertex-substeps advanced
        "dev_s": sum(server.frame_ms) / 1e3,
        "arrived_work": [r.vertices * SUBSTEPS * r.frames for r in arrived],
        "arrived_vertices": [r.vertices for r in arrived],
        "admitted": sum(1 for r in reqs if r.admitted_at is not None), "completed": len(done),
        "work": sum(r.vertices * SUBSTEPS * r.frames for r in done),
        "lat": [r.finished_at - r.arrival for r in done], "wait": [r.admitted_at - r.arrival for r in done],
        "frame_ms": list(server.frame_ms), "admit_ms": list(server.admit_ms), "gather_ms": list(server.gather_ms),
        "frame_sizes": [float(x) for x in server.frame_sizes], "queue_end": len(server.queue),
        "queue_max": max(server.queue_lengths) if server.queue_lengths else 0, "gathers": server.gathers,
    }
    server.close()
    reports = sharding.gather_to_rank0(report)
    if rank == 0:
        # a sample of rank 0's requests, each alone through plain advance(), one after the other
        sample = arrived[: args.alone_sample]
        service = []
        for r in sample:
            sim = serve.build_request_sim(r, (128, 0))
            st = torch.cuda.Stream()
            sim.set_stream(st.cuda_stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(r.frames):
                sim.advance(FRAME)
            e1.record(st)
            e1.synchronize()
            service.append(e0.elapsed_time(e1) / 1e3)
            sim.close()
        alone_tp = sum(r.vertices * SUBSTEPS * r.frames for r in sample) / max(sum(service), 1e-9)

        def cat(key):
            return [x for rep in reports for x in rep[key]]

        wall_max = max(rep["wall"] for rep in reports)
        served_work = sum(rep["served_work"] for rep in reports)
        dev_s = max(rep["dev_s"] for rep in reports)
        arrived_work = cat("arrived_work")
        mean_req_work = float(np.mean(arrived_work)) if arrived_work else 0.0
        batched_tp = served_work / max(wall_max, 1e-9)
        queue_end = sum(rep["queue_end"] for rep in reports)
        out = {
            "metric": "serving: request latency and vertex-substeps/s under Poisson arrivals", "unit": "s",
            "n_gpus": world, "rate_per_s": args.rate, "arrival_window_s": args.duration,
            "frames_per_request": args.frames, "budget_gb": args.budget_gb,
            "max_batch_vertices": args.max_batch_verts or None, "setup_threads": args.setup_threads,
            "routing": "one server per GPU, request i on rank i mod %d" % world,
            "requests": {"arrived": len(arrived_work), "admitted": sum(rep["admitted"] for rep in reports),
                         "completed": sum(rep["completed"] for rep in reports), "queued_at_end": queue_end},
            "request_latency_s": serve.percentiles(cat("lat")), "queue_wait_s": serve.percentiles(cat("wait")),
            "frame_latency_ms": serve.percentiles(cat("frame_ms")), "frames": len(cat("frame_ms")),
            "frame_boundary_ms": {"admission_host": serve.percentiles(cat("admit_ms")),
                                  "regather_host": serve.percentiles(cat("gather_ms")),
                                  "what": "host time at each frame boundary before the frame's advance: building "
                                          "the admitted requests as one-scene Sims (configure, upload) and "
                                          "re-gathering the batch (yb_batch_gather device copies included); "
                                          "frame_latency_ms is the device time of the advance"},
            "batch_vertices": serve.percentiles(cat("frame_sizes")),
            "queue_length": {"max": max(rep["queue_max"] for rep in reports), "end": queue_end},
            "gathers": sum(rep["gathers"] for rep in reports),
            "throughput_vertex_substeps_per_s": batched_tp,
            "device_throughput_vertex_substeps_per_s": served_work / max(dev_s, 1e-9),
            "completed_work_vertex_substeps": sum(rep["work"] for rep in reports), "wall_s": wall_max,
            "offered_load_vertex_substeps_per_s": mean_req_work * args.rate,
            "sustainable_rate_per_s": batched_tp / mean_req_work if mean_req_work else None,
            "alone": {"requests": len(sample), "throughput_vertex_substeps_per_s": alone_tp,
                      "service_s": serve.percentiles(service)},
            "batched_over_alone": (batched_tp / world) / alone_tp if alone_tp else None,
            "request_vertices": serve.percentiles(cat("arrived_vertices")),
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_twist(args):
    """Cable twist: 49 straight yarns (7 x 7 grid, 1.1 mm pitch) of 8192 vertices, both ends
    pinned, the top pins rotated about the bundle axis at 2 pi rad/s by the device pin driver;
    the FP32 production build against the FP64 build of the same kernels from identical inputs.
    Every `--every` frames: relative position error (max difference / max displacement), the
    largest angle between corresponding segment rotors, and the bundle twist (mean angle of
    the yarns' vertices at half and 0.9 of the height about the bundle axis, unwrapped) of both builds.  The run
    stops at the first frame where either build reports an error (the reference throws on
    MAX_COLLISIONS_PER_SEGMENT, YarnBall.cu:283-285); that frame and the largest contact count
    per segment of every sample are reported."""
    import torch

    from yarnball_b200 import YarnBallError, scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    frames = args.frames if args.frames else 300
    every = max(1, args.every)
    sims, centers = {}, {}
    for prec in ("fp32", "fp64"):
        sims[prec] = scenes.build_twist(precision=prec, meta={"gravity": (0.0, args.gravity, 0.0)})
        sims[prec].set_tuning(128, 0, True, False)
        _, centers[prec] = scenes.device_twist(sims[prec], omega=2 * math.pi)
    x0 = sims["fp64"].read_state_f64()[0]
    n = sims["fp64"].numVerts
    verts = 8192
    c = centers["fp64"]
    levels = {}
    for frac in (0.5, 0.9):  # fraction of the height; the driven pins are at the top
        idx = np.arange(49) * verts + int(frac * (verts - 1))
        idx = idx[np.hypot(x0[idx, 0] - c[0], x0[idx, 2] - c[2]) > 1e-4]  # the centre yarn has no angle
        levels[frac] = (idx, np.arctan2(x0[idx, 2] - c[2], x0[idx, 0] - c[0]))

    def twist_of(p, prev):
        out = {}
        for frac, (idx, a0) in levels.items():
            a = np.arctan2(p[idx, 2] - c[2], p[idx, 0] - c[0]) - a0
            out[frac] = prev[frac] + (a - prev[frac] + np.pi) % (2 * np.pi) - np.pi  # unwrap against the last frame
        return out

    def rotor_angle(q1, q2):
        s = np.sign(np.sum(q1 * q2, axis=1, keepdims=True))
        s[s == 0] = 1
        return 2 * np.arctan2(np.linalg.norm(q1 - s * q2, axis=1), np.linalg.norm(q1 + s * q2, axis=1))

    seg = (sims["fp64"].verts["flags"] & 2) != 0
    rows, ms = [], {"fp32": 0.0, "fp64": 0.0}
    tw = {p: {frac: np.zeros(len(idx)) for frac, (idx, _) in levels.items()} for p in ("fp32", "fp64")}
    stopped, done = {}, 0
    for f in range(1, frames + 1):
        for prec in ("fp32", "fp64"):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            try:
                sims[prec].advance(FRAME)
            except YarnBallError as err:
                stopped[prec] = {"frame": f, "error": str(err)}
            e1.record()
            e1.synchronize()
            ms[prec] += e0.elapsed_time(e1)
        if stopped:
            break
        done = f
        pa, _, qa = sims["fp32"].read_state_f64()
        pb, _, qb = sims["fp64"].read_state_f64()
        for prec, p in (("fp32", pa), ("fp64", pb)):  # unwrapped every frame
            tw[prec] = twist_of(p, tw[prec])
        if f % every == 0 or f == frames:
            rows.append({"frame": f, "rel_pos_err": float(np.abs(pa - pb).max() / max(np.abs(pb - x0).max(), 1e-30)),
                         "max_rotor_angle_rad": float(rotor_angle(qa[seg], qb[seg]).max()),
                         "twist_fp64_rad": {str(fr): float(tw["fp64"][fr].mean()) for fr in levels},
                         "twist_err_rad": {str(fr): float(np.abs(tw["fp32"][fr] - tw["fp64"][fr]).max()) for fr in levels},
                         "penetrations_fp32": sims["fp32"].penetrations(),
                         "min_pair_distance_m": {p: sims[p].min_pair_distance() for p in sims},
                         "max_contacts_per_segment": {p: sims[p].collisionStats()[2] for p in sims}})
    for s in sims.values():
        s.close()
    out = {"metric": "cable twist: FP32 vs FP64 build per frame", "unit": "relative / rad", "vertices": n,
           "frames": done, "frames_requested": frames, "stopped": stopped or None,
           "substeps_per_frame": SUBSTEPS, "samples": rows,
           "throughput_vertex_substeps_per_s": {p: n * SUBSTEPS * max(done, 1) / (ms[p] / 1e3) for p in ms},
           "config": {"workload": "cable twist, 49 yarns x 8192 vertices, 2 pi rad/s, device pin driver",
                      "gravity_y": args.gravity}}
    print(json.dumps(out))


def run_pile(args):
    """Contact-heavy pile, plain FP32: 1024 random-walk yarns x 256 vertices (262,144) in a
    10 cm cube, first vertex of each yarn pinned, one scene advanced frame by frame for
    `--pile-frames` frames (60) through advance(1/30).  Reports device-timed throughput over
    all frames, the mean and largest contact count per segment every 10 frames (against the
    128 cap), per-kernel times of one more frame, the Newton iteration's fraction of measured
    HBM bandwidth on algorithmic bytes, the interpenetration measures, and the FP32 build
    against the FP64 build after one frame from identical inputs."""
    import torch

    from yarnball_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    frames = max(1, args.pile_frames)
    ref = scenes.build_pile(seed=1, precision="fp64")
    sim = scenes.build_pile(seed=1)
    n = sim.numVerts
    nseg = int(((sim.verts["flags"] & 2) != 0).sum())
    x0 = sim.read_state_f64()[0]
    # accuracy: one frame of both builds from the same inputs
    sim.advance(FRAME)
    ref.advance(FRAME)
    pa, pb = sim.read_state_f64()[0], ref.read_state_f64()[0]
    acc = {"vs": "FP64 build of the same kernels", "frames": 1,
           "rel_err": float(np.abs(pa - pb).max() / max(np.abs(pb - x0).max(), 1e-30)),
           "max_abs_err_m": float(np.abs(pa - pb).max())}
    ref.close()
    sim.close()
    sim = scenes.build_pile(seed=1)
    sim.advance(FRAME)
    tune = sim.autotune()
    sim.close()
    sim = scenes.build_pile(seed=1)
    sim.set_tuning(tune[0], tune[1], True, bool(tune[2]))
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    samples, ms_total = [], 0.0
    l0 = sim.launch_count()
    for f in range(1, frames + 1):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.advance(FRAME)
        e1.record(stream)
        e1.synchronize()
        ms_total += e0.elapsed_time(e1)
        if f == 1:
            ms_first = e0.elapsed_time(e1)  # includes the instantiation of the substep graphs
        if f % 10 == 0 or f == 1 or f == frames:
            tot, segs_with, mx = sim.collisionStats()
            samples.append({"frame": f, "cbar": 2.0 * tot / max(nseg, 1), "max_per_segment": mx,
                            "segments_with_contacts": segs_with})
    launches = sim.launch_count() - l0
    prof_ms, prof_launches = sim.profile_advance(FRAME)
    tot, _, _ = sim.collisionStats()
    cbar = 2.0 * tot / max(nseg, 1)
    iter_ms = prof_ms["iter"] / max(1, prof_launches["iter"])
    achieved = n * (ITER_BYTES_BASE + ITER_BYTES_PER_CONTACT * cbar) / (iter_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    value = n * SUBSTEPS * frames / (ms_total / 1e3)
    out = {"metric": "vertex-substeps/s (contact-heavy pile, plain FP32, one scene)", "value": value, "unit": UNIT,
           "frames": frames, "ms_per_frame": ms_total / frames, "ms_first_frame": ms_first,
           "gpu_launches": int(launches), "vertices": n,
           "newton_kernel_shape": {"threads": tune[0], "lanes_per_vertex": tune[1], "pipelined": bool(tune[2]),
                                   "autotune_ms_per_launch": tune[3]},
           "contacts": samples, "kernel_ms_per_frame": prof_ms,
           "newton_hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                          "peak_kind": peak_kind, "avg_launch_ms": iter_ms, "cbar": cbar},
           "interpenetrations": {"min_centre_line_distance_m": sim.min_pair_distance(),
                                 "hard_core_contacts": sim.penetrations(), "two_radius_m": 2 * float(scenes.RADIUS)},
           "accuracy": acc,
           "config": {"workload": "contact-heavy pile: 1024 random-walk yarns x 256 vertices (262,144) in a 10 cm "
                                  "cube, radius 2.5e-5 m, barrier 9.5e-4 m, mu 0.3, kBend 1e-8, kStretch 2e-2, "
                                  "first vertex pinned, maxH 1e-3", "seed": 1}}
    sim.close()
    print(json.dumps(out))


def run_readme(args):
    """Config 1, the README two-yarn scene (README.md:104-127; 64 vertices): 150 frames of
    advance(1/30 s) = 5100 substeps through the plain drop-in path, device-timed; beside it the
    same frames on the reference's own kernels on this GPU (compiled unchanged from its sources
    by oracle/refbuild, when built; their BVH query is a brute-force stand-in, trivial at 64
    vertices) and on the CPU oracle (FP32, OpenMP).  Accuracy: the engine's positions against
    the FP64 oracle after the first and the last frame (relative to the motion), and the largest
    distance between the engine's and the reference kernels' trajectories over the run."""
    import torch

    import oracle
    from yarnball_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    frames = max(1, args.readme_frames)
    sim = scenes.build_readme()
    sim.download()
    v, vel, q, qr = sim.verts.copy(), sim.vels.astype(np.float32).copy(), sim.qs.copy(), sim.qRests.copy()
    meta = sim.scene_meta(0).as_struct()
    x0 = v["pos"].astype(np.float64)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    for _ in range(max(0, args.warmup)):  # warm-up on separate copies: the timed run starts at t = 0
        w = scenes.build_readme()
        w.advance(FRAME)
        w.close()
    torch.cuda.synchronize()
    l0 = sim.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(frames):
        sim.advance(FRAME)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sim.launch_count() - l0
    work = 64 * SUBSTEPS * frames
    final = sim.read_state_f64()[0]
    sim.close()
    # end to end with host copies every frame (upload, advance, download)
    sim = scenes.build_readme()
    w0 = time.perf_counter()
    for _ in range(frames):
        sim.upload()
        sim.advance(FRAME)
        sim.download()
    wall_e2e = time.perf_counter() - w0
    sim.close()
    # accuracy against the FP64 oracle, distance to the reference kernels' trajectory
    eng = scenes.build_readme()
    orc = oracle.from_sim(eng, mode=oracle.FP64)
    refk, ref_err = None, None
    try:
        from oracle import reference as R

        if R.available():
            refk = R.RefSim(v, vel, q, qr, meta, variant="fma")
        else:
            ref_err = "reference kernels not built (oracle/_ref)"
    except Exception as e:  # reported, not fatal: the reference build is test infrastructure
        ref_err = str(e)
    acc, traj = {}, 0.0
    for f in range(1, frames + 1):
        eng.advance(FRAME)
        orc.advance(FRAME, MAX_H)
        pe = eng.read_state_f64()[0]
        if refk is not None:
            refk.advance(FRAME)
            traj = max(traj, float(np.abs(pe - refk.read("verts")["pos"].astype(np.float64)).max()))
        if f in (1, frames):
            po = orc.state()["pos"]
            acc["frame_%d" % f] = float(np.abs(pe - po).max() / max(np.abs(po - x0).max(), 1e-30))
    eng.close()
    orc.close()
    if refk is not None:
        refk.close()
        timer = R.RefSim(v, vel, q, qr, meta, variant="fma")
        timer.advance(FRAME)  # warm-up (module load)
        timer.close()
        timer = R.RefSim(v, vel, q, qr, meta, variant="fma")
        rc, rms = timer.time_advance(FRAME, frames)
        timer.close()
        ref_cuda = {"value": work / (rms / 1e3), "unit": UNIT, "ms": rms, "status": rc,
                    "what": "the reference's own kernels (fused multiply-adds, as its build compiles them) on "
                            "this GPU, launched with the reference's shapes and schedule; brute-force BVH stand-in"}
    else:
        ref_cuda = {"unavailable": ref_err}
    orc = oracle.from_sim(scenes.build_readme(), mode=oracle.FP32)
    t0 = time.perf_counter()
    for _ in range(frames):
        orc.advance(FRAME, MAX_H)
    cpu_s = time.perf_counter() - t0
    orc.close()
    out = {"metric": "vertex-substeps/s (README two-yarn scene, plain advance)", "value": work / (ms / 1e3),
           "unit": UNIT, "frames": frames, "substeps": SUBSTEPS * frames, "ms": ms, "ms_per_frame": ms / frames,
           "gpu_launches": int(launches),
           "e2e": {"value": work / wall_e2e, "unit": UNIT, "wall_s": wall_e2e,
                   "h2d_bytes_per_step": 64 * (32 + 12 + 16 + 16), "d2h_bytes_per_step": 64 * (32 + 12 + 16),
                   "api": "yb_upload + yb_advance + yb_download per frame (host wall clock)"},
           "reference_cuda": ref_cuda,
           "cpu_baseline": {"value": work / cpu_s, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port",
                            "sample": "the same %d frames, FP32 OpenMP" % frames},
           "accuracy": {"rel_err_vs_fp64_oracle": acc, "bound": 1e-4,
                        "max_dist_to_reference_kernels_m": traj if refk is not None else None,
                        "final_displacement_m": float(np.abs(final - x0).max())},
           "config": {"workload": "README two-yarn scene: 2 yarns x 32 vertices, pins 0/32/63, kCollision 1e-7, "
                                  "kBend 1e-8, kStretch 2e-2, maxH 1e-3, advance(1/30) x %d" % frames}}
    print(json.dumps(out))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "twist":
        run_twist(args)
    elif args.workload == "pile":
        run_pile(args)
    elif args.workload == "readme":
        run_readme(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
