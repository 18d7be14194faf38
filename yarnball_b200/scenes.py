"""Synthetic scenes for the benchmark and tests (seeded, no files needed).

  readme     the two-yarn example of the reference README (64 vertices)
  pile       random-walk yarn pile in a 10 cm cube (1024 yarns x 256 vertices by default)
  twist      7 x 7 bundle of straight yarns, both ends pinned, one end rotated
  batched    up to 512 independent pile-style scenes of uneven size in one flat array

Yarn radius 0.5 mm maps to radius = 0.05 r and barrierThickness = 1.9 r, the reference's
own `curveRadius` mapping (KittenEngine/YarnBall/io/jsonBuilder.cpp:44-49).
"""
import ctypes
import math

import numpy as np

from . import _abi
from ._abi import ptr
from .sim import Sim

YARN_RADIUS = 0.5e-3
RADIUS = np.float32(0.05 * YARN_RADIUS)
BARRIER = np.float32(1.9 * YARN_RADIUS)
SEG_LEN = 2e-3
CUBE = 0.1
TURN_SIGMA = 0.3
# initial gap: no pair closer than 2 radius + 0.1 barrierThickness (normalised gap d >= 0.1)
MIN_DIST = float(2 * RADIUS + 0.1 * BARRIER)


def readme_positions():
    """README.md:104-127: p_i = (2e-5 i (i-16) + 0.002, -0.002 i, 0), p_{i+32} = x-mirror."""
    seg = np.float32(0.002)
    pos = np.zeros((64, 3), np.float32)
    for i in range(32):
        x = np.float32(np.float32(np.float32(0.00002) * np.float32(i)) * np.float32(i - 16)) + seg * np.float32(1)
        y = -seg * np.float32(i)
        pos[i] = (x, y, 0.0)
        pos[i + 32] = (-x, y, 0.0)
    return pos


def build_readme(precision="fp32"):
    sim = Sim(64, precision=precision)
    sim.verts["pos"][:] = readme_positions()
    for i in (0, 32, 63):
        sim.verts["invMass"][i] = 0.0
    sim.verts["flags"][31] = 0
    sim.meta.kCollision = 1e-7
    sim.configure()
    sim.setKBend(1e-8)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim


def random_walks(seed, yarn_lengths, seg_len=SEG_LEN, cube=CUBE, sigma=TURN_SIGMA, min_dist=MIN_DIST):
    lib = _abi.load()
    lens = np.ascontiguousarray(yarn_lengths, dtype=np.int32)
    out = np.zeros((int(lens.sum()), 3), np.float32)
    st = lib.yb_scene_random_walks(int(seed), len(lens), ptr(lens, ctypes.c_int32), seg_len, cube, sigma, min_dist,
                                   ptr(out, ctypes.c_float))
    if st != 0:
        raise RuntimeError("random walk generation failed (%d)" % st)
    return out


def random_walks_batch(seed, yarns_per_scene, yarn_lengths, seg_len=SEG_LEN, cube=CUBE, sigma=TURN_SIGMA,
                       min_dist=MIN_DIST, threads=0):
    lib = _abi.load()
    yps = np.ascontiguousarray(yarns_per_scene, dtype=np.int32)
    lens = np.ascontiguousarray(yarn_lengths, dtype=np.int32)
    out = np.zeros((int(lens.sum()), 3), np.float32)
    st = lib.yb_scene_random_walks_batch(int(seed), len(yps), ptr(yps, ctypes.c_int32), ptr(lens, ctypes.c_int32),
                                         seg_len, cube, sigma, min_dist, ptr(out, ctypes.c_float), int(threads))
    if st != 0:
        raise RuntimeError("batched random walk generation failed (%d)" % st)
    return out


PILE_META = dict(kCollision=1e-7, frictionCoeff=0.3, radius=float(RADIUS), barrierThickness=float(BARRIER))


def fill_yarns(sim, pos, yarn_lengths, offset=0, pin_first=True, pin_last=False):
    """Writes yarn polylines into sim.verts starting at vertex `offset` (breaks between yarns)."""
    n = len(pos)
    v = sim.verts[offset:offset + n]
    v["pos"][:] = pos
    ends = np.cumsum(yarn_lengths) - 1
    starts = ends - np.asarray(yarn_lengths) + 1
    fl = v["flags"].copy()
    fl[ends] = 0
    v["flags"][:] = fl
    if pin_first:
        im = v["invMass"].copy()
        im[starts] = 0.0
        v["invMass"][:] = im
    if pin_last:
        im = v["invMass"].copy()
        im[ends] = 0.0
        v["invMass"][:] = im


def build_pile(seed=1, yarns=1024, verts=256, precision="fp32", num_itr=None, meta=None, cube=CUBE):
    lens = np.full(yarns, verts, np.int32)
    pos = random_walks(seed, lens, cube=cube)
    sim = Sim(int(lens.sum()), precision=precision)
    fill_yarns(sim, pos, lens, pin_first=True)
    for k, val in dict(PILE_META, **(meta or {})).items():
        setattr(sim.meta, k, val)
    if num_itr is not None:
        sim.meta.numItr = num_itr
    sim.configure()
    sim.setKBend(1e-8)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim


def twist_positions(grid=7, pitch=1.1e-3, verts=8192, seg_len=SEG_LEN):
    pos = np.zeros((grid * grid * verts, 3), np.float32)
    c = (grid - 1) / 2.0
    k = 0
    for i in range(grid):
        for j in range(grid):
            pos[k:k + verts, 0] = (i - c) * pitch
            pos[k:k + verts, 1] = np.arange(verts) * seg_len
            pos[k:k + verts, 2] = (j - c) * pitch
            k += verts
    return pos


def build_twist(grid=7, verts=8192, precision="fp32", meta=None):
    lens = np.full(grid * grid, verts, np.int32)
    pos = twist_positions(grid, 1.1e-3, verts)
    sim = Sim(int(lens.sum()), precision=precision)
    fill_yarns(sim, pos, lens, pin_first=True, pin_last=True)
    for k, val in dict(PILE_META, **(meta or {})).items():
        setattr(sim.meta, k, val)
    sim.configure()
    sim.setKBend(1e-8)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim


class TwistDriver:
    """Rotates the pinned top end of every yarn about the bundle axis (+y through the bundle
    centre) at `omega` rad/s, prescribing pin velocity (next - pos) / dt, the mechanism of
    KittenEngine/main.cpp:54-87 (download, move pins, upload each frame)."""

    def __init__(self, sim, omega=2 * math.pi):
        sim.download()
        self.sim = sim
        self.omega = omega
        self.init = sim.verts["pos"].copy()
        ymax = self.init[:, 1].max()
        self.top = np.where((sim.verts["invMass"] == 0) & (self.init[:, 1] > 0.5 * ymax))[0]
        self.center = 0.5 * (self.init.min(0) + self.init.max(0))
        self.t = 0.0

    def _rot(self, p, ang):
        # rotateY of main.cpp:68-69 (right-handed about +y)
        c, s = math.cos(ang), math.sin(ang)
        d = p - self.center
        out = d.copy()
        out[:, 0] = c * d[:, 0] + s * d[:, 2]
        out[:, 2] = -s * d[:, 0] + c * d[:, 2]
        return out + self.center

    def frame(self, dt):
        sim = self.sim
        sim.download()
        p0 = self._rot(self.init[self.top], self.omega * self.t)
        p1 = self._rot(self.init[self.top], self.omega * (self.t + dt))
        sim.verts["pos"][self.top] = p0.astype(np.float32)
        sim.vels[self.top] = ((p1 - p0) / dt).astype(np.float32)
        sim.upload()
        sim.advance(dt)
        self.t += dt


def device_twist(sim, omega=2 * math.pi, t_start=0.0, t_end=1e30):
    """Same motion as TwistDriver, performed on the device by the kinematic pin driver:
    pinned vertices in the upper half rotate about the bundle axis (+y through the centre)."""
    sim.download()
    p = sim.verts["pos"].astype(np.float64)
    ymax = p[:, 1].max()
    top = (sim.verts["invMass"] == 0) & (p[:, 1] > 0.5 * ymax)
    center = 0.5 * (p.min(0) + p.max(0))
    groups = np.where(top, 1, 0).astype(np.uint8)
    sim.set_pin_motion(groups, [dict(center=center, axis=(0, 1, 0), omega=omega, tStart=t_start, tEnd=t_end)])
    return groups, center


def batched_spec(seed=7, num_scenes=512, cap=8388608, max_yarns=64, min_len=64, max_len=4096):
    """Scene sizes of the batched workload: k ~ U{1..max_yarns} yarns per scene, vertices per
    yarn log-uniform in [min_len, max_len], kBend log-uniform in [1e-9, 1e-7]; scenes are
    added until the next one would exceed `cap` vertices.  Draws use numpy's PCG64 seeded
    with `seed`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    yarns, lens, kbend = [], [], []
    total = 0
    for _ in range(num_scenes):
        k = int(rng.integers(1, max_yarns + 1))
        ls = np.exp(rng.uniform(math.log(min_len), math.log(max_len), size=k)).astype(np.int32)
        kb = float(10 ** rng.uniform(-9, -7))
        if total + int(ls.sum()) > cap:
            break
        yarns.append(k)
        lens.append(ls)
        kbend.append(kb)
        total += int(ls.sum())
    return yarns, lens, kbend


def batched_positions(seed, spec, indices=None, threads=0):
    """Vertex positions of the scenes `indices` (default: all) of a batched spec, one array per
    scene.  Scene i is seeded from (seed, i), its index in the full spec, so a subset (the
    scenes one rank of a multi-GPU run simulates) holds exactly the geometry those scenes have
    in the whole batch."""
    yarns, lens, _ = spec
    if indices is None:
        indices = list(range(len(yarns)))
    last = max(indices) + 1 if len(indices) else 0
    if last == 0:
        return []
    flat = np.concatenate(lens[:last]).astype(np.int32)
    pos = random_walks_batch(seed, yarns[:last], flat, threads=threads)
    offs = np.concatenate([[0], np.cumsum([int(l.sum()) for l in lens[:last]])]).astype(np.int64)
    return [pos[offs[i]:offs[i + 1]] for i in indices]


def build_batched(seed=7, num_scenes=512, cap=8388608, precision="fp32", spec=None, threads=0, indices=None):
    """The batched workload (or the subset `indices` of its scenes) as one batch."""
    full = spec if spec is not None else batched_spec(seed, num_scenes, cap)
    if indices is None:
        indices = list(range(len(full[0])))
    yarns = [full[0][i] for i in indices]
    lens = [full[1][i] for i in indices]
    kbend = [full[2][i] for i in indices]
    pos_list = batched_positions(seed, full, indices, threads=threads)
    counts = [int(l.sum()) for l in lens]
    sim = Sim(scenes=counts, precision=precision)
    off = 0
    for s, l in enumerate(lens):
        fill_yarns(sim, pos_list[s], l, offset=off, pin_first=True)
        off += counts[s]
    sim.set_meta_all(**PILE_META)
    sim.configure()
    for s, kb in enumerate(kbend):
        sim.setKBend(kb, scene=s)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim, (yarns, lens, kbend)


def build_scene_alone(spec, s, seed=7, precision="fp32"):
    """Scene s of a batched spec as its own plain Sim (same geometry and parameters)."""
    yarns, lens, kbend = spec
    flat = np.concatenate(lens).astype(np.int32)
    pos_all = random_walks_batch(seed, yarns, flat)
    counts = [int(l.sum()) for l in lens]
    off = int(sum(counts[:s]))
    sim = Sim(counts[s], precision=precision)
    fill_yarns(sim, pos_all[off:off + counts[s]], lens[s], pin_first=True)
    for k, val in PILE_META.items():
        setattr(sim.meta, k, val)
    sim.configure()
    sim.setKBend(kbend[s])
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim
