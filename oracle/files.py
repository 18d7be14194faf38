"""Restatement of the reference's curve exporters, used only by the tests as the checker.

  bcc_bytes  Sim::exportToBCC  KittenEngine/YarnBall/io/fileExport.cpp:6-63
  obj_text   Sim::exportToOBJ  KittenEngine/YarnBall/io/fileExport.cpp:65-100
  read_bcc   the inverse of bcc_bytes (header fields and curves)

Inputs are the host vertex records (numpy structured array with 'pos' and 'flags'), i.e.
what the reference writes after its download().  The reference leaves the 40 fileInfo bytes
of the header uninitialised; this restatement writes zeros.
"""
import struct

import numpy as np

HAS_NEXT = 2


def curve_runs(flags):
    """Runs [start, end] of consecutive vertices with hasNext; end is the vertex that closes
    the run (the first one without hasNext), fileExport.cpp:33-46."""
    runs, last, start = [], False, 0
    for i, f in enumerate(np.asarray(flags, np.uint32)):
        seg = (int(f) & HAS_NEXT) != 0
        if seg and not last:
            start = i
        elif not seg and last:
            runs.append((start, i))
        last = seg
    return runs


def bcc_bytes(verts, as_polyline=False):
    runs = curve_runs(verts["flags"])
    total = sum(e - s + 1 for s, e in runs)
    kind = b"PL" if as_polyline else b"C0"
    out = [struct.pack("<3sB2sbbQQ40s", b"BCC", 0x44, kind, 3, 1, len(runs), total, b"\0" * 40)]
    pos = np.ascontiguousarray(verts["pos"], np.float32)
    for s, e in runs:
        out.append(struct.pack("<i", e - s + 1))
        out.append(pos[s:e + 1].tobytes())
    return b"".join(out)


def read_bcc(data):
    sign, bc, kind, dims, up, nc, npts, _ = struct.unpack_from("<3sB2sbbQQ40s", data, 0)
    off, curves = 64, []
    for _ in range(nc):
        (m,) = struct.unpack_from("<i", data, off)
        off += 4
        curves.append(np.frombuffer(data, np.float32, 3 * m, off).reshape(m, 3))
        off += 12 * m
    return {"sign": sign, "byteCount": bc, "curveType": kind, "dimensions": dims, "upDimension": up,
            "curveCount": nc, "totalControlPointCount": npts, "curves": curves, "end": off}


def obj_text(verts):
    """C printf %.16f of a float promoted to double, as the reference's fprintf."""
    lines = ["# YarnBall Sim\n\n", "o YarnBall\n\n", "# Vertices (in meters)\n"]
    for p in np.asarray(verts["pos"], np.float32):
        lines.append("v %.16f %.16f %.16f\n" % (float(p[0]), float(p[1]), float(p[2])))
    lines.append("\n# Curves\n")
    last = False
    for i, f in enumerate(np.asarray(verts["flags"], np.uint32)):
        seg = (int(f) & HAS_NEXT) != 0
        if seg:
            if not last:
                lines.append("l %d" % (i + 1))
            lines.append(" %d" % (i + 2))
        elif last:
            lines.append("\n")
        last = seg
    return "".join(lines)
