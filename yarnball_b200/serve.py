"""Continuous-batching request loop for many independent yarn scenes on one GPU.

No reference counterpart (the reference advances one Sim per call).  Each request is a
scene that asks for a number of frames of 1/30 s.  The server keeps every admitted scene's
state on the device between frames and advances all of them with one batched advance() per
frame, so requests of different sizes share every kernel launch:

  * a request waits in a FIFO queue; host threads generate the geometry of the head of the
    queue while the frames run, a bounded number of vertices ahead, so that host work overlaps
    device work;
  * a request whose geometry is ready is admitted at the next frame boundary if the
    device-memory budget (two batch allocations) and the optional per-frame vertex cap allow;
    the frame thread then builds it as a one-scene Sim (configure, upload): every CUDA call of
    the server is made by the frame thread, so no allocation or release of another thread can
    meet a graph capture or a frame in flight;
  * when membership changes, the batch is rebuilt by copying every remaining and newly
    admitted scene device to device (yb_batch_gather), reusing the previous batch's
    allocation when it is large enough (two allocations alternate);
  * after a scene's last frame only its range of the batch is downloaded.

Because a scene's state travels with it and every substep re-detects contacts, a scene
gives bit-identical results alone and inside any mix (detectionPeriod 1, same Newton kernel
shape, multi-block kernels), which tests/test_gpu_serving.py checks.  A scene of at most 256
vertices simulated alone takes the one-block small-simulation path instead, which agrees with
the multi-block kernels to rounding.
"""
import collections
import math
import time
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np

from . import scenes
from .sim import Sim

FRAME = 1.0 / 30.0


class Request:
    def __init__(self, rid, arrival, spec, frames=30, seed=0):
        self.id = rid
        self.arrival = arrival        # seconds (server clock)
        self.spec = spec              # (yarn lengths, kBend)
        self.frames = frames
        self.seed = seed
        self.done_frames = 0
        self.staging = None           # one-scene Sim until admitted
        self.future = None            # its geometry, generated on a host thread
        self.admitted_at = None
        self.finished_at = None
        self.result = None            # (positions, velocities, rotors) after the last frame
        self.vertices = int(np.sum(spec[0]))


def request_geometry(req):
    lens = np.asarray(req.spec[0], np.int32)
    # pile density at most that of the 1024 x 256 pile in a 10 cm cube
    cube = scenes.CUBE * max(1.0, lens.sum() / 262144.0) ** (1.0 / 3.0)
    return scenes.random_walks(req.seed, lens, cube=cube)


def build_request_sim(req, shape=None, meta=None, pos=None):
    lens, kbend = req.spec
    lens = np.asarray(lens, np.int32)
    if pos is None:
        pos = request_geometry(req)
    sim = Sim(int(lens.sum()))
    scenes.fill_yarns(sim, pos, lens, pin_first=True)
    for k, v in dict(scenes.PILE_META, **(meta or {})).items():
        setattr(sim.meta, k, v)
    sim.configure()
    sim.setKBend(kbend)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    if shape:
        sim.set_tuning(shape[0], shape[1], True, len(shape) > 2 and shape[2])
    return sim


def run_alone(req, shape=None):
    """Reference for the mixed result: the request simulated by itself."""
    sim = build_request_sim(req, shape)
    for _ in range(req.frames):
        sim.advance(FRAME)
    sim.download()
    out = (sim.verts["pos"].copy(), sim.vels.copy(), sim.qs.copy())
    sim.close()
    return out


class Server:
    """Continuous batching on one GPU.

    budget_bytes        device memory for the batch (two allocations, gathered alternately)
    max_batch_vertices  optional cap on the vertices advanced per frame: it bounds the frame
                        latency (a frame's time grows with the batch) at the price of queueing
    setup_threads       host threads that generate request geometry ahead of admission, while
                        frames run; 0 generates it on the frame thread
    prefetch_vertices   how many vertices of queued requests may have geometry staged ahead
    """

    def __init__(self, budget_bytes=120e9, shape=(128, 0), bytes_per_vertex=None, capacity_headroom=1.25,
                 stream=None, setup_threads=4, prefetch_vertices=4_000_000, max_batch_vertices=None):
        self.budget = float(budget_bytes)
        self.shape = shape
        self.bpv = bytes_per_vertex
        self.headroom = capacity_headroom
        self.stream = stream
        self.prefetch = int(prefetch_vertices)
        self.max_batch = max_batch_vertices
        self.pool = ThreadPoolExecutor(setup_threads) if setup_threads > 0 else None
        self.queue = collections.deque()
        self.active = []              # requests in batch scene order
        self.batch = None
        self.spare = None
        self.finished = []
        self.frame_ms = []            # device time of each batched frame
        self.admit_ms = []            # host time of each frame boundary's admissions (one-scene Sims built)
        self.gather_ms = []           # host time of each re-gather (device copies included, 0 without one)
        self.frame_sizes = []         # vertices advanced in each frame
        self.queue_lengths = []       # queued requests at each frame boundary
        self.gathers = 0

    # ---- memory accounting -------------------------------------------------------------
    def _bytes_per_vertex(self, sim):
        if self.bpv is None:
            self.bpv = sim.device_bytes() / max(sim.numVerts, 1)
        return self.bpv

    def _staged_vertices(self):
        return sum(r.vertices for r in self.queue if r.future is not None)

    def _build(self, r):
        """The admitted request as a one-scene Sim (frame thread)."""
        return build_request_sim(r, self.shape, pos=r.future.result())

    # ---- request flow ---------------------------------------------------------------
    def submit(self, req):
        """Queues a request; its geometry is generated on a host thread when the prefetch window
        allows."""
        req.future = None
        self.queue.append(req)
        self._stage()

    def _stage(self):
        staged = self._staged_vertices()
        for r in self.queue:  # FIFO: stage the head of the queue first
            if r.future is not None:
                continue
            if staged > 0 and staged + r.vertices > self.prefetch:
                break
            if self.pool is None:
                f = Future()
                f.set_result(request_geometry(r))
                r.future = f
            else:
                r.future = self.pool.submit(request_geometry, r)
            staged += r.vertices

    def _admit(self):
        joined = []
        verts = sum(r.vertices for r in self.active)
        joinedVerts = 0
        while self.queue:
            r = self.queue[0]
            if r.future is None:
                break
            if not r.future.done():
                break  # geometry not ready: the batch goes on without it
            if (self.active or joined) and self.bpv is not None:
                # two batch allocations of the grown size and the one-scene Sims of this frame's
                # admissions (released after the gather) must fit the budget
                need = (2 * self.headroom * (verts + r.vertices) + joinedVerts + r.vertices) * self.bpv
                if need > self.budget or (self.max_batch and verts + r.vertices > self.max_batch):
                    break
            sim = self._build(r)
            self._bytes_per_vertex(sim)
            self.queue.popleft()
            r.staging = sim
            joined.append(r)
            verts += r.vertices
            joinedVerts += r.vertices
        self._stage()
        return joined

    def _close_later(self, sim):
        sim.close()

    def _regather(self, keep, joined):
        sources = [(self.batch, i) for i in keep] + [(r.staging, 0) for r in joined]
        members = [self.active[i] for i in keep] + joined
        if not sources:
            if self.batch is not None:
                self.spare, self.batch = self.batch, None
            self.active = []
            return
        total = sum(r.vertices for r in members)
        new = Sim.gather(sources, recycle=self.spare, capacity=int(total * self.headroom))
        self.gathers += 1
        if self.spare is not None and new is not self.spare:
            self._close_later(self.spare)
        self.spare = self.batch
        self.batch = new
        self.batch.set_tuning(self.shape[0], self.shape[1], True, len(self.shape) > 2 and self.shape[2])
        if self.stream is not None:
            self.batch.set_stream(self.stream.cuda_stream)
        for r in joined:  # gather has finished its copies: the staging copies can go
            self._close_later(r.staging)
            r.staging = None
        self.active = members

    def step(self, now, admit=True):
        """One frame boundary: retire, admit (unless admit is False), re-gather if needed,
        advance one frame."""
        if admit and not self.active and self.queue and self.queue[0].future is not None:
            self.queue[0].future.result()  # an idle server waits for its next request
        self.queue_lengths.append(len(self.queue))
        keep = [i for i, r in enumerate(self.active) if r.done_frames < r.frames]
        t0 = time.perf_counter()
        joined = self._admit() if admit else []
        t1 = time.perf_counter()
        for r in joined:
            r.admitted_at = now
        if len(keep) != len(self.active) or joined:
            self._regather(keep, joined)
        t2 = time.perf_counter()
        if not self.active:
            return 0.0
        self.admit_ms.append((t1 - t0) * 1e3)
        self.gather_ms.append((t2 - t1) * 1e3)
        import torch

        if self.stream is None:  # the batch must run on the stream the events are recorded on
            self.stream = torch.cuda.Stream()
            self.batch.set_stream(self.stream.cuda_stream)
        st = self.stream
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        self.batch.advance(FRAME)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        self.frame_ms.append(ms)
        self.frame_sizes.append(self.batch.numVerts)
        for i, r in enumerate(self.active):
            r.done_frames += 1
            if r.done_frames == r.frames:
                self.batch.download_scene(i)
                o0, o1 = self.batch.sceneOffsets[i], self.batch.sceneOffsets[i + 1]
                r.result = (self.batch.verts["pos"][o0:o1].copy(), self.batch.vels[o0:o1].copy(),
                            self.batch.qs[o0:o1].copy())
                self.finished.append(r)
        return ms

    def busy(self):
        return bool(self.queue) or any(r.done_frames < r.frames for r in self.active)

    def close(self):
        if self.pool is not None:
            self.pool.shutdown(wait=True)
        for b in (self.batch, self.spare):
            if b is not None:
                b.close()
        self.batch = self.spare = None


def poisson_requests(rate, duration, seed=11, median_verts=16384, sigma=1.5, lo=64, hi=1_000_000, frames=30):
    """Poisson arrivals at `rate` per second for `duration` seconds; each request is a scene of
    total vertex count lognormal(median, sigma) clipped to [lo, hi], split into pile-style
    yarns (64..4096 vertices, log-uniform), kBend log-uniform in [1e-9, 1e-7]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        total = int(np.clip(np.exp(rng.normal(math.log(median_verts), sigma)), lo, hi))
        lens = []
        left = total
        while left > 0:
            m = int(np.exp(rng.uniform(math.log(64), math.log(4096))))
            m = min(m, left)
            if m < 3:
                lens[-1] += m
                break
            lens.append(m)
            left -= m
        kb = float(10 ** rng.uniform(-9, -7))
        out.append(Request(len(out), t, (np.array(lens, np.int32), kb), frames=frames, seed=seed * 1000003 + len(out)))
    return out


def percentiles(x):
    if not x:
        return {"p50": None, "p95": None, "p99": None}
    a = np.asarray(x, np.float64)
    return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)), "p99": float(np.percentile(a, 99))}
