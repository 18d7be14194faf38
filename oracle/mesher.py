"""Restatement of the reference's fibre mesher (Sim::exportFiberMesh,
KittenEngine/YarnBall/io/fiberMesher.cpp:9-157), used only by the tests as the checker for
yb_export_fiber_mesh.

The random stream is restated exactly (fastPRNG's fastXS64::xoroshiro128p: state = two chained
SplitMix64 outputs of the seed, rotations 24 / 16 / 37; a draw is the low 32 bits divided by
(float)UINT32_MAX, clamped to [0, 1]), as are the decisions that depend on float rounding
(fibre vertices per segment, fuzz strands per segment, the running twist angle).  The three
draws of one vector are taken x, y, z (the reference leaves the order to its compiler).
Geometry is evaluated in float64; the library's float32 GPU evaluation agrees to rounding.

PARITY UNPINNED: the reference cannot be compiled here, so the stream is checked against the
published SplitMix64 output for seed 0 and the rest against this restatement only.
"""
import math

import numpy as np

M64 = (1 << 64) - 1
F = np.float32


def splitmix64(v):
    z = (v + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


class Xoroshiro128p:
    def __init__(self, seed):
        self.s0 = splitmix64(seed)
        self.s1 = splitmix64(self.s0)

    @staticmethod
    def _rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & M64

    def next(self):
        r = (self.s0 + self.s1) & M64
        s1 = self.s1 ^ self.s0
        self.s0 = self._rotl(self.s0, 24) ^ s1 ^ ((s1 << 16) & M64)
        self.s1 = self._rotl(s1, 37)
        return r

    def uniform(self):
        x = F(F(self.next() & 0xFFFFFFFF) / F(4294967295.0))
        return float(min(max(x, F(0)), F(1)))


def _round_half_away(x):
    f = math.floor(x)
    return int(f + 1) if x - f >= 0.5 else int(f)


def _cmr(a, b, c, d, t):
    mix = lambda x, y, s: x * (1 - s) + y * s
    a0, a1, a2 = mix(a, b, t + 1), mix(b, c, t), mix(c, d, t - 1)
    return mix(mix(a0, a1, (t + 1) * 0.5), mix(a1, a2, t * 0.5), t)


def _rotate(q, v):
    qv, w = q[:3], q[3]
    a = w * v + np.cross(qv, v)
    c = np.dot(v, qv)
    return w * a + np.cross(qv, a) + c * qv


def _frame(q0, q1, q2, t):
    v = q0 * (1 - (t + 0.5)) + q1 * (t + 0.5) if t < 0.5 else q1 * (1 - (t - 0.5)) + q2 * (t - 0.5)
    return v / np.linalg.norm(v)


def fiber_mesh(pos, qs, lrest, flags, radius, barrier):
    """Returns (fiber vertices, fiber line index lists, fuzz vertices, fuzz line pairs), with
    OBJ (1-based, global) indices, in the order the reference writes them."""
    pos = np.asarray(pos, np.float64)
    qs = np.asarray(qs, np.float64)
    n = len(pos)
    r = F(F(radius) + F(0.5) * F(barrier))
    frizz_amp = float(F(0.2) * r)
    twist_rate = 1200.0
    fiber_radius = F(F(F(0.6) * r) / F(math.sqrt(8.0)))
    height = F(F(0.3) * r)
    orbit = float(F(F(F(0.9) * r) - fiber_radius) - F(frizz_amp))
    two_pi = F(2.0 * math.pi)
    has_next = lambda i: (int(flags[i]) & 2) != 0
    has_prev = lambda i: (int(flags[i]) & 1) != 0
    segs = []
    cur = F(0)
    for i in range(n):
        if not has_next(i):
            continue
        lr = F(lrest[i])
        nh = max(int(math.ceil(F(lr / height))), 1)
        a = i - 1 if has_prev(i) else i
        b = i + 2 if has_next(i + 1) else i + 1
        q0 = qs[i - 1] if has_prev(i) else qs[i]
        q2 = qs[i + 1] if has_next(i + 1) else qs[i]
        segs.append(dict(i=i, nh=nh, lr=float(lr), twist=float(cur), pts=(pos[a], pos[i], pos[i + 1], pos[b]),
                         q=(q0, qs[i], q2)))
        cur = F(cur + F(F(1200.0) * lr))
        cur = F(cur - F(two_pi * F(math.floor(F(cur / two_pi)))))
    rng = Xoroshiro128p(0x12345678)
    fiber_v, fiber_l = [], []
    for fid in range(8):
        start = len(fiber_v)
        si = 0
        for i in range(n):
            if not has_next(i):
                if len(fiber_v) - start > 2:
                    fiber_l.append(list(range(start + 1, len(fiber_v) + 1)))
                start = len(fiber_v)
                continue
            s = segs[si]
            si += 1
            for hi in range(s["nh"]):
                t = hi / s["nh"]
                p = _cmr(*s["pts"], t)
                fr = _frame(*s["q"], t)
                ang = s["twist"] + twist_rate * t * s["lr"] + fid / 8.0 * 2 * math.pi
                tw = np.array([0.0, math.cos(ang), math.sin(ang)]) * orbit
                if hi:
                    d = np.array([rng.uniform() for _ in range(3)])
                    tw = tw + frizz_amp * (d * 2 - 1)
                fiber_v.append(p + _rotate(fr, tw))
    fuzz_v, fuzz_l = [], []
    base = len(fiber_v)
    for s in segs:
        nf = _round_half_away(float(F(F(F(2 * F(rng.uniform())) * F(s["lr"])) * F(1.25e4))))
        for _ in range(nf):
            t = rng.uniform()
            p = _cmr(*s["pts"], t)
            fr = _frame(*s["q"], t)
            d = np.array([rng.uniform() for _ in range(3)]) * 2 - 1
            off = d + (np.array([rng.uniform() for _ in range(3)]) * 2 - 1)
            off[0] *= 0.1
            off = 0.9 * orbit * off / np.linalg.norm(off)
            d = d * (float(r) * (0.8 + 0.2 * rng.uniform()))
            for hi in (0, 1):
                fuzz_v.append(p + _rotate(fr, hi * d + off))
            k = base + len(fuzz_v)
            fuzz_l.append((k - 1, k))
    return np.array(fiber_v), fiber_l, np.array(fuzz_v), fuzz_l


def parse_obj(text):
    """Sections of an OBJ file written by the mesher: {name: (vertices, lines)}."""
    out, cur = {}, None
    for line in text.splitlines():
        if line.startswith("o "):
            cur = line[2:].strip()
            out[cur] = ([], [])
        elif line.startswith("v "):
            out[cur][0].append([float(x) for x in line.split()[1:4]])
        elif line.startswith("l "):
            out[cur][1].append([int(x) for x in line.split()[1:]])
    return {k: (np.array(v), l) for k, (v, l) in out.items()}
