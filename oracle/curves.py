"""Restatement of the reference's curve readers and Catmull-Rom resampler, used only by the
tests as the checker for the library's readers (yb_read_bcc / yb_read_obj / yb_read_poly,
yb_resample_cmr).

  cmr_spline         Kit::cmrSpline              KittenEngine/includes/modules/Common.h:683-694
  sample_curve       Resample::sampleCurve       KittenEngine/YarnBall/io/resample.h:10-18
  resample_coords    resampleCMRCoords           resample.h:20-83
  two_direction      twoDirectionResampleCMRCoords resample.h:85-141
  resample_cmr       resampleCMR                 resample.h:143-187
  curves_bcc/obj/poly readFromBCC/OBJ/Poly       KittenEngine/YarnBall/io/reader.cpp:49-295
  from_curves        createFromCurves            reader.cpp:13-47

Arithmetic follows the reference's operation order in double precision (glm::mix(x, y, a) =
x * (1 - a) + y * a), so the library's C++ (built with -ffp-contract=off) agrees bit for bit.
Where the reference reads or writes out of bounds the restatement does what the library does
(and says so at the spot): resampling needs at least 4 control points, and the end alignment
and the merge blend skip indices outside the list.

PARITY UNPINNED: the reference cannot be compiled here (glm, jsoncpp absent), so this
restatement is checked against hand-worked cases in the tests, not against reference output.
"""
import math
import re
import struct

import numpy as np

HAS_NEXT = 2


def _mix(x, y, a):
    return tuple(xi * (1.0 - a) + yi * a for xi, yi in zip(x, y))


def cmr_spline(p0, p1, p2, p3, t):
    a0 = _mix(p0, p1, t + 1)
    a1 = _mix(p1, p2, t + 0)
    a2 = _mix(p2, p3, t - 1)
    b0 = _mix(a0, a1, (t + 1) * 0.5)
    b1 = _mix(a1, a2, (t + 0) * 0.5)
    return _mix(b0, b1, t)


def sample_curve(cmr, t):
    si = min(max(int(math.floor(t)), 1), len(cmr) - 3)
    p = [tuple(float(c) for c in cmr[si + k]) for k in (-1, 0, 1, 2)]
    return cmr_spline(p[0], p[1], p[2], p[3], t - si)


def _len2(a, b):
    d = [x - y for x, y in zip(a, b)]
    return (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]


def resample_coords(cmr, start, end, tar):
    ts = []
    MIN_STEP = 0.2
    step = MIN_STEP if end > start else -MIN_STEP
    r2 = tar * tar
    i = start
    last = sample_curve(cmr, i)
    ts.append(i)
    while (i < end) if end > start else (i > end):
        i += step
        pos = sample_curve(cmr, i)
        l0 = _len2(pos, last)
        if l0 > r2:
            l0 = math.sqrt(l0)
            lo, hi = i - step, i
            if lo > hi:
                lo, hi = hi, lo
            t0 = i
            i -= 0.5 * step
            for _ in range(8):
                x = sample_curve(cmr, i)
                d = math.sqrt(_len2(x, last))
                i += (i - t0) * (tar - d) / (d - l0)
            i = min(max(i, lo), hi)
            ts.append(i)
            last = sample_curve(cmr, i)
    if len(ts) == 1:
        ts.append(end)
    else:
        d = math.sqrt(_len2(sample_curve(cmr, ts[-1]), sample_curve(cmr, end)))
        dt = ts[-1] - ts[-2]
        if d > 0.5 * tar:
            ts.append(end)
        else:
            ts[-1] = end
        dt -= ts[-1] - ts[-2]
        n = min(len(ts), 8)
        for k in range(n):
            at = len(ts) - 2 - k
            if at >= 0:  # the reference writes ts[-1] for lists of 8 or fewer
                ts[at] -= dt * (n - k) / float(n)
    return ts


def two_direction(cmr, start, end, tar):
    fwd = resample_coords(cmr, start, end, tar)
    bwd = resample_coords(cmr, end, start, tar)
    B = 8
    if len(fwd) > 4 * B and len(bwd) > 4 * B:
        min_err = math.inf
        sx, sy = 2 * B, 2 * B
        j = len(bwd) - 1 - B
        for i in range(B, len(fwd) - 8):
            t = fwd[i]
            while j > 0 and bwd[j] < t:
                j -= 1
            t0 = bwd[j + 1]
            if min_err > abs(t - t0):
                min_err = abs(t - t0)
                sx, sy = i, j + 1
            t1 = bwd[j]
            if min_err > abs(t1 - t):
                min_err = abs(t1 - t)
                sx, sy = i, j
        merged = list(fwd[:sx])
        mid = 0.5 * (fwd[sx] + bwd[sy])
        merged.append(mid)
        for k in range(sy - 1, -1, -1):
            merged.append(bwd[k])
        dt = fwd[sx] - mid
        for k in range(B):
            at = sx - k - 1
            if 0 <= at < len(merged):
                merged[at] -= dt * (B - k) / (1.0 + B)
        dt = bwd[sy] - mid
        for k in range(B):
            at = sx + k + 1
            if 0 <= at < len(merged):  # the reference does not check this bound
                merged[at] -= dt * (B - k) / (1.0 + B)
        return merged
    return fwd


def resample_cmr(cmr, start, end, tar):
    """Float32 points resampled at about `tar` spacing (the reference's resampleCMR)."""
    cmr = [tuple(float(c) for c in p) for p in np.asarray(cmr, np.float32)]
    if len(cmr) < 4:  # the reference's sampleCurve reads cmr[-1] here
        return np.asarray(cmr, np.float32).reshape(-1, 3)
    ts0 = two_direction(cmr, start, end, tar)
    total, err0 = 0.0, 0.0
    last = sample_curve(cmr, ts0[0])
    for t in ts0[1:]:
        pos = sample_curve(cmr, t)
        ln = math.sqrt(_len2(pos, last))
        err0 = max(err0, abs(ln - tar))
        total += ln
        last = pos
    avg = total / (len(ts0) - 1)
    ts1 = two_direction(cmr, start, end, avg)
    last = sample_curve(cmr, ts1[0])
    err1 = 0.0
    for t in ts1[1:]:
        pos = sample_curve(cmr, t)
        ln = math.sqrt(_len2(pos, last))
        err1 = max(err1, abs(ln - avg))
        last = pos
    ts = ts0 if err0 < err1 else ts1
    return np.asarray([sample_curve(cmr, t) for t in ts], np.float64).astype(np.float32)


def transform_points(points, T):
    """vec3(T * vec4(p, 1)) for a column-major 4x4 float matrix T (glm order of operations:
    (c0 x + c1 y) + (c2 z + c3 w), in float32)."""
    T = np.asarray(T, np.float32).reshape(4, 4)  # T[col][row]
    p = np.asarray(points, np.float32)
    one = np.float32(1)
    out = np.empty_like(p)
    for r in range(3):
        a = (T[0, r] * p[:, 0]).astype(np.float32) + (T[1, r] * p[:, 1]).astype(np.float32)
        b = (T[2, r] * p[:, 2]).astype(np.float32) + (T[3, r] * one).astype(np.float32)
        out[:, r] = (a.astype(np.float32) + b.astype(np.float32)).astype(np.float32)
    return out


def curves_bcc(data, target, T, break_up, allow_resample):
    target = float(np.float32(target))  # the readers take targetSegLen as a float
    sign, bc, kind, dims, up, nc, npts = struct.unpack_from("<3sB2sbbQQ", data, 0)
    if sign != b"BCC" or bc != 0x44:
        raise ValueError("Unsupported BCC file")
    poly = kind == b"PL"
    if not poly and kind != b"C0":
        raise ValueError("Not polyline or uniform CMR spline")
    if dims != 3:
        raise ValueError("Only curves in 3D are supported")
    off, curves, closed = 64, [], []
    for _ in range(nc):
        (m,) = struct.unpack_from("<i", data, off)
        off += 4
        is_closed = m < 0
        m = abs(m)
        pts = np.frombuffer(data, np.float32, 3 * m, off).reshape(m, 3)
        off += 12 * m
        pts = transform_points(pts, T)
        if allow_resample and not poly:
            pts = resample_cmr(pts, 1, len(pts) - 2, target)
        if m < 3:
            continue
        closed.append(is_closed and not break_up)
        curves.append(np.asarray(pts, np.float32))
    return curves, closed


def curves_obj(text, target, T, break_up, allow_resample):
    target = float(np.float32(target))  # the readers take targetSegLen as a float
    verts, lines = [], []
    for line in text.splitlines():
        tok = line.split()
        if not tok:
            continue
        if tok[0] == "v":
            verts.append([float(x) for x in tok[1:4]])
        elif tok[0] == "l":
            idx = []
            for x in tok[1:]:  # istream >> int: a leading integer, then stop at the rest
                m = re.match(r"[+-]?\d+", x)
                if not m:
                    break
                idx.append(int(m.group()))
                if m.end() != len(x):
                    break
            if idx:
                lines.append(idx)
    V = transform_points(np.asarray(verts, np.float32).reshape(-1, 3), T)
    curves, closed = [], []
    for idx in lines:
        c = V[np.asarray(idx) - 1]
        is_closed = idx[0] == idx[-1]
        if break_up and is_closed:
            c = c[:-1]
            is_closed = False
        if allow_resample:
            c = resample_cmr(c, 1, len(c) - 2, target)
        if len(c) < 4:
            continue
        curves.append(np.asarray(c, np.float32))
        closed.append(is_closed)
    return curves, closed


def curves_poly(text, target, T, break_up, allow_resample):
    target = float(np.float32(target))  # the readers take targetSegLen as a float
    pts, segs, is_point = [], [], True
    lines = text.split("\n")
    if lines and lines[-1] == "":  # std::getline yields no empty line after a final newline
        lines.pop()
    for line in lines:
        if line == "POINTS":
            is_point = True
            continue
        if line == "POLYS":
            is_point = False
            continue
        if line == "END":
            break
        tok = line.replace(":", " : ", 1).split()
        if is_point:
            if len(tok) < 5 or tok[1] != ":":
                raise ValueError("Error parsing .poly. Point parse error.")
            pts.append([float(tok[2]), float(tok[3]), float(tok[4])])
            if int(tok[0]) != len(pts):
                raise ValueError("Error parsing .poly. Point id mismatch.")
        else:
            if len(tok) < 4 or tok[1] != ":":
                raise ValueError("Error parsing .poly. Segment parse error.")
            segs.append((int(tok[2]) - 1, int(tok[3]) - 1))
    P = transform_points(np.asarray(pts, np.float32).reshape(-1, 3), T)
    nbr = [[] for _ in range(len(P))]  # neighbours in segment order
    for a, b in segs:
        nbr[a].append(b)
        nbr[b].append(a)
    visited = [False] * len(P)
    curves, closed = [], []
    for i in range(len(P)):
        if visited[i]:
            continue
        if len(nbr[i]) > 2:
            raise ValueError("Graphs not allowed.")
        if len(nbr[i]) > 1:
            continue
        c, cur = [], i
        while not visited[cur]:
            visited[cur] = True
            c.append(P[cur])
            nxt = [x for x in nbr[cur] if not visited[x]]
            if not nbr[cur]:
                break
            if nxt:
                cur = nxt[0]
        if len(c) < 4:
            continue
        # the reference resamples open curves whether or not resampling is allowed
        curves.append(resample_cmr(np.asarray(c), 1, len(c) - 2, target))
        closed.append(False)
    for i in range(len(P)):
        if visited[i]:
            continue
        if len(nbr[i]) != 2:
            raise ValueError("Graphs not allowed.")
        c, cur = [], i
        while True:
            visited[cur] = True
            c.append(P[cur])
            found, is_end = False, False
            for x in nbr[cur]:
                if not visited[x]:
                    cur = x
                    found = True
                    break
                if x == i:
                    is_end = True
            if not found:
                if not is_end:
                    raise ValueError("Closed curve not closed.")
                break
        c = np.asarray(c, np.float32)
        if allow_resample:
            c = resample_cmr(c, 1, len(c) - 2, target)
        if len(c) < 4:
            continue
        curves.append(np.asarray(c, np.float32))
        closed.append(not break_up)
    return curves, closed


def from_curves(curves, closed):
    """Vertex positions, flags and connection indices of createFromCurves."""
    n = sum(len(c) for c in curves)
    pos = np.zeros((n, 3), np.float32)
    flags = np.full(n, 2, np.uint32)  # hasNext, Sim::Sim default
    cid = np.full(n, -1, np.int32)
    off = 0
    for c, cl in zip(curves, closed):
        m = len(c)
        pos[off:off + m] = c
        flags[off + m - 1] = 0
        if cl:
            cid[off] = off + m - 1
            cid[off + m - 1] = off
        off += m
    return pos, flags, cid


def glue_endpoints(pos, flags, cid, radius, scene_ranges=None):
    """Sim::glueEndpoints (io/jsonBuilder.cpp:174-212) with the library's fixed order: the
    nearest vertex (|i - j| > 2, same scene, float32 distance ((dx dx + dy dy) + dz dz then
    sqrt), first minimum) of every endpoint is found on the positions at the call, then joins
    are applied in ascending endpoint order when both ends are still free.  Returns new
    (pos, cid)."""
    pos = np.asarray(pos, np.float32).copy()
    cid = np.asarray(cid, np.int32).copy()
    flags = np.asarray(flags, np.uint32)
    n = len(pos)
    if scene_ranges is None:
        scene_ranges = [(0, n)]
    snap = pos.copy()
    found = []
    for a, b in scene_ranges:
        for i in range(a, b):
            has_prev = i > a and (int(flags[i - 1]) & HAS_NEXT) != 0
            has_next = (int(flags[i]) & HAS_NEXT) != 0
            if has_prev == has_next:
                continue
            d = snap[a:b] - snap[i]
            d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
            dist = np.sqrt(d2.astype(np.float32)).astype(np.float32)
            j = np.arange(a, b)
            dist[np.abs(j - i) <= 2] = np.inf
            k = int(np.argmin(dist))
            found.append((i, a + k, dist[k]))
    for i, j, dmin in found:
        if np.isfinite(dmin) and dmin <= np.float32(radius) and cid[j] < 0 and cid[i] < 0:
            cid[j] = i
            cid[i] = j
            mid = (np.float32(0.5) * (pos[i] + pos[j])).astype(np.float32)
            pos[i] = mid
            pos[j] = mid
    return pos, cid
