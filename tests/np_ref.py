"""Second, independent restatement of one substep in numpy/Python loops (FP64, small N).

Written separately from the C++ oracle so that the two can check each other; follows the
same reference expressions:
  initItr            KittenEngine/YarnBall/sim/iteration.cu:7-41
  buildCollisionList KittenEngine/YarnBall/sim/collision.cu:39-92 (all pairs, no broadphase)
  recomputeStepLimit KittenEngine/YarnBall/sim/collision.cu:121-159
  cosseratItr        KittenEngine/YarnBall/sim/cosserat.cu:20-207 (strict Jacobi)
  quaternionLambda   KittenEngine/YarnBall/sim/cosserat.cu:209-253 (strict Jacobi)
  endItr             KittenEngine/YarnBall/sim/iteration.cu:48-61
"""
import numpy as np

HAS_PREV, HAS_NEXT, HAS_NEXT_ORI, FIX_ORI = 1, 2, 4, 8
# (1 - SAFETY_MARGIN) * 0.5 with the FP32 constant 0.1f (collision.cu:129,155)
SAFE = (1.0 - float(np.float32(0.1))) * 0.5


def closest(a1, b0, b1):
    """segmentClosestPoints(0, a1, b0, b1) (Common.h:318-336) in FP64."""
    A1 = b1 - b0
    a = a1 @ a1
    b = a1 @ A1
    c = A1 @ A1
    with np.errstate(all="ignore"):
        v = (b * (a1 @ b0) - a * (A1 @ b0)) / (a * c - b * b)
        if not np.isfinite(v):
            v = 0.5
        v = min(max(v, 0.0), 1.0)
        u = min(max(((b0 * (1 - v) + b1 * v) @ a1) / a, 0.0), 1.0)
        v = min(max(((u * a1 - b0) @ A1) / c, 0.0), 1.0)
    return u, v


def qmul(l, r):
    lq, rq = l[:3], r[:3]
    return np.concatenate([l[3] * rq + r[3] * lq + np.cross(lq, rq), [l[3] * r[3] - lq @ rq]])


def qinv(q):
    return np.array([-q[0], -q[1], -q[2], q[3]])


def qrot(q, v):
    qq, w = q[:3], q[3]
    a = w * v + np.cross(qq, v)
    return w * a + np.cross(qq, a) + (v @ qq) * qq


def barrier(d, kCol, invb):
    """(dH, ff) of E = -kCollision (d-1)^2 ln d on the normalised gap (cosserat.cu:121-125)."""
    invd, logd = 1.0 / d, np.log(d)
    dH = (-3 + (2 + invd) * invd - 2 * logd) * kCol * invb
    ff = -(1 - d) * (d - 1 + 2 * d * logd) * invd * kCol
    return dH, ff


class Params:
    def __init__(self, meta):
        g = np.array(meta["gravity"], np.float64)
        self.h = float(meta["h"])
        self.lastH = float(meta["lastH"])
        self.g = g
        self.drag = float(meta["drag"])
        self.D = float(meta["damping"]) / self.h
        self.accel = float(meta["accelerationRatio"])
        self.twoR = 2 * float(meta["radius"])
        self.invb = 1.0 / float(meta["barrierThickness"])
        self.kCol = float(meta["kCollision"]) * self.invb
        self.fricK = float(meta["kFriction"])
        self.mu = float(meta["frictionCoeff"])
        dr = float(meta["radius"]) + 0.5 * float(meta["barrierThickness"])
        self.sdr = dr * float(meta["detectionScaler"])
        self.stepBase = dr * (float(meta["detectionScaler"]) - 1)
        self.numItr = int(meta["numItr"])


def substep(st, meta):
    """One substep on dict state st (pos, vel, lastVel, q, qRest, invMass, lRest, kStretch,
    cid, flags), FP64; returns (new state, contact lists, step limits)."""
    p = Params(meta)
    pos, vel, lastVel = st["pos"].copy(), st["vel"].copy(), st["lastVel"].copy()
    q, qRest = st["q"].copy(), st["qRest"]
    im, lRest, kS, cid, fl = st["invMass"], st["lRest"], st["kStretch"], st["cid"], st["flags"]
    n = len(pos)
    h = p.h
    # predictor
    dx = h * vel
    y = dx + h * h * p.g
    g2 = p.g @ p.g
    for i in range(n):
        if im[i] != 0 and g2 > 0:
            a = (vel[i] - lastVel[i]) / p.lastH
            s = min(max((a @ p.g) / g2, 0.0), 1.0)
            dx[i] = dx[i] + (h * h * s) * p.g
    lastVel = vel.copy()
    segs = [i for i in range(n) if fl[i] & HAS_NEXT]
    # detection: every pair, the narrow-phase filter with the lower index as segment A
    cols = {i: [] for i in range(n)}
    for ai, x in enumerate(segs):
        for yy in segs[ai + 1:]:
            c0, c1 = cid[x], cid[x + 1]
            if c0 in (yy, yy + 1) or c1 in (yy, yy + 1) or abs(yy - x) <= 2:
                continue
            a0 = pos[x]
            a1, b0, b1 = pos[x + 1] - a0, pos[yy] - a0, pos[yy + 1] - a0
            u, v = closest(a1, b0, b1)
            d2 = np.sum((u * a1 - (b0 * (1 - v) + b1 * v)) ** 2)
            r = 2 * p.sdr + np.sqrt(max(dx[x] @ dx[x], dx[x + 1] @ dx[x + 1])) + np.sqrt(
                max(dx[yy] @ dx[yy], dx[yy + 1] @ dx[yy + 1]))
            if d2 < r * r:
                cols[x].append(yy)
                cols[yy].append(x)
    for i in cols:
        cols[i].sort()
    # step limit
    sl = np.full(n, np.inf)
    for k in segs:
        a0 = pos[k]
        a1 = pos[k + 1] - a0
        m = p.stepBase + np.sqrt(dx[k] @ dx[k])
        for o in cols[k]:
            b0, b1 = pos[o] - a0, pos[o + 1] - a0
            u, v = closest(a1, b0, b1)
            m = min(m, SAFE * np.linalg.norm(u * a1 - (b0 * (1 - v) + b1 * v)))
        sl[k] = m
    e1 = np.array([1.0, 0.0, 0.0])
    for _ in range(p.numItr):
        fA = np.zeros((n, 3)); fB = np.zeros((n, 3)); HA = np.zeros((n, 3, 3)); HB = np.zeros((n, 3, 3))
        for i in range(n):
            f = np.zeros(3); H = np.zeros((3, 3)); f2 = np.zeros(3); H2 = np.zeros((3, 3))
            if im[i] != 0:
                H += np.eye(3) / (im[i] * h * h)
                f += (y[i] - dx[i]) / (h * h * im[i])
            if cid[i] >= 0:
                c = cid[i]
                f -= 40 * ((pos[i] - pos[c]) + (dx[i] - dx[c]) + p.D * dx[i])
                H += np.eye(3) * 40 * (1 + p.D)
            if fl[i] & HAS_NEXT:
                p0, p1, d0, d1 = pos[i], pos[i + 1], dx[i], dx[i + 1]
                invl = 1.0 / lRest[i]
                c = ((p1 - p0) + (d1 - d0)) * invl - qrot(q[i], e1)
                k = kS[i] * invl
                dd = k * invl
                f += k * c - p.D * dd * d0
                f2 += -k * c - p.D * dd * d1
                H += np.eye(3) * dd * (1 + p.D)
                H2 += np.eye(3) * dd * (1 + p.D)
                for j in cols[i]:
                    b0, b1, db0, db1 = pos[j], pos[j + 1], dx[j], dx[j + 1]
                    u, v = closest((p1 - p0) + (d1 - d0), (b0 - p0) + (db0 - d0), (b1 - p0) + (db1 - d0))
                    dpos = (p0 * (1 - u) + p1 * u) - (b0 * (1 - v) + b1 * v)
                    ddpos = (d0 * (1 - u) + d1 * u) - (db0 * (1 - v) + db1 * v)
                    nrm = dpos + ddpos
                    dist = np.linalg.norm(nrm)
                    nrm = nrm / dist
                    wa, wb = 1 - u, u
                    gap = (dist - p.twoR) * p.invb
                    if gap > 1:
                        continue
                    gap = max(gap, 1e-3)
                    dH, ff = barrier(gap, p.kCol, p.invb)
                    f += (ff * wa - p.D * dH * wa * wa * (nrm @ d0)) * nrm
                    f2 += (ff * wb - p.D * dH * wb * wb * (nrm @ d1)) * nrm
                    dH *= 1 + p.D
                    nn = np.outer(nrm, nrm)
                    H += nn * dH * wa * wa
                    H2 += nn * dH * wb * wb
                    uu = ddpos - (nrm @ ddpos) * nrm
                    ul = np.linalg.norm(uu)
                    if ul > 0:
                        f1 = min(p.fricK, p.mu * ff / ul)
                        f -= f1 * wa * uu
                        f2 -= f1 * wb * uu
                        H += (np.eye(3) - nn) * wa * wa * f1
                        H2 += (np.eye(3) - nn) * wb * wb * f1
            fA[i], HA[i], fB[i], HB[i] = f, H, f2, H2
        ndx = dx.copy()
        for i in range(n):
            f, H = fA[i].copy(), HA[i].copy()
            s_l = sl[i] if fl[i] & HAS_NEXT else np.inf
            if fl[i] & HAS_PREV:
                f += fB[i - 1]
                H += HB[i - 1]
                s_l = min(s_l, sl[i - 1])
            if im[i] != 0:
                d = dx[i] + p.accel * np.linalg.solve(H, f)
                ln = np.linalg.norm(d)
                if ln > s_l and ln > 0:
                    d = d * (s_l / ln)
                ndx[i] = d
        dx = ndx
        nq = q.copy()
        for i in range(n):
            if (fl[i] & FIX_ORI) or not (fl[i] & HAS_NEXT):
                continue
            v = ((pos[i + 1] - pos[i]) + (dx[i + 1] - dx[i])) / lRest[i] * (-2 * kS[i])
            b = np.zeros(4)
            if fl[i] & HAS_PREV:
                s = 1.0 if qmul(qinv(q[i - 1]), q[i]) @ qRest[i - 1] > 0 else -1.0
                b += s * qmul(q[i - 1], qRest[i - 1])
            if fl[i] & HAS_NEXT_ORI:
                s = 1.0 if qmul(qinv(q[i]), q[i + 1]) @ qRest[i] > 0 else -1.0
                b += s * qmul(q[i + 1], qinv(qRest[i]))
            if np.linalg.norm(b) == 0:
                continue  # one-segment yarn: the closed form is 0/0, orientation kept
            lam = np.linalg.norm(v) + np.linalg.norm(b)
            r = qmul(qmul(np.concatenate([v, [0.0]]), b), np.array([1.0, 0, 0, 0])) + lam * b
            nq[i] = r / np.linalg.norm(r)
        q = nq
    newvel = vel.copy()
    for i in range(n):
        if im[i] != 0:
            newvel[i] = dx[i] / h * (1 - p.drag * h)
    pos = pos + dx
    return dict(st, pos=pos, vel=newvel, lastVel=lastVel, q=q), cols, sl
