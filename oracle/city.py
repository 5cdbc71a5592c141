"""Seeded synthetic city in pure Python -- TEST INFRASTRUCTURE ONLY.

A restatement of the product's city generator (lbm_city_generate) so that
the reference arm of bench.py can build its geometry without loading the
product library: the same SplitMix64 stream, street-grid spans, block
shuffle and box triangulation, hence bit-identical float32 triangles
(tests/test_city_restatement.py holds it to the product generator).  Also a
binary STL writer in the layout GeometryEngine::load reads (06:49-58, 06:70-86).
"""
import struct

import numpy as np

_M64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & _M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & _M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def uniform(self, lo, hi):
        """Integer in [lo, hi], both inclusive."""
        if hi <= lo:
            return lo
        return lo + self.next() % (hi - lo + 1)


def _spans(rng, n, fp, street, margin):
    """Footprint spans of [margin, n - margin): widths in [fp0, fp1], gaps of
    at least `street` plus up to street // 2."""
    out = []
    x, end = margin, n - margin
    while x + fp[0] <= end:
        w = rng.uniform(fp[0], fp[1])
        if x + w > end:
            w = end - x
        if w < fp[0]:
            break
        out.append((x, x + w))
        x += w + street + rng.uniform(0, street // 2)
    return out


_QUADS = ((0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7))


def box_triangles(x0, y0, z0, x1, y1, z1):
    """12 outward-facing triangles of an axis-aligned box, [12, 9] float32."""
    v = ((x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1),
         (x0, y1, z1))
    out = []
    for q in _QUADS:
        for tri in ((q[0], q[1], q[2]), (q[0], q[2], q[3])):
            out.append([c for i in tri for c in v[i]])
    return np.asarray(out, dtype=np.float32)


def city_boxes(nx, ny, seed, dx=1.0, fp=(20, 60), height=(10, 80), coverage=0.40, street=8, margin=0):
    """Boxes (x0, y0, 0, x1, y1, h) in metres and the plan coverage reached."""
    rng = SplitMix64(seed)
    xs = _spans(rng, nx, fp, street, margin)
    ys = _spans(rng, ny, fp, street, margin)
    blocks = [(a, b) for a in range(len(xs)) for b in range(len(ys))]
    for i in range(len(blocks) - 1, 0, -1):
        j = rng.uniform(0, i)
        blocks[i], blocks[j] = blocks[j], blocks[i]
    total = float(nx) * float(ny)
    covered = 0.0
    boxes = []
    for a, b in blocks:
        if covered / total >= coverage:
            break
        sx, sy = xs[a], ys[b]
        h = rng.uniform(height[0], height[1])
        boxes.append((sx[0] * dx, sy[0] * dx, 0.0, sx[1] * dx, sy[1] * dx, h * dx))
        covered += float(sx[1] - sx[0]) * float(sy[1] - sy[0])
    return boxes, covered / total


def city_triangles(nx, ny, seed, **kw):
    boxes, cov = city_boxes(nx, ny, seed, **kw)
    if not boxes:
        return np.zeros((0, 9), dtype=np.float32), cov
    return np.concatenate([box_triangles(*b) for b in boxes]), cov


def crop_boxes(boxes, x0, y0, x1, y1):
    """The boxes clipped to the plan window [x0, x1) x [y0, y1), moved so the
    window starts at the origin.  Columns inside the window see the same
    heights, so the window's voxelised mask is that of the whole city."""
    out = []
    for bx0, by0, bz0, bx1, by1, bz1 in boxes:
        cx0, cy0, cx1, cy1 = max(bx0, x0), max(by0, y0), min(bx1, x1), min(by1, y1)
        if cx0 < cx1 and cy0 < cy1:
            out.append((cx0 - x0, cy0 - y0, bz0, cx1 - x0, cy1 - y0, bz1))
    return out


def stl_write(path, tris):
    """Binary STL: 80-byte header, uint32 count, 50-byte records (normal,
    three vertices, attribute), float32 little-endian."""
    t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    with open(path, "wb") as fh:
        fh.write(b"synthetic city (oracle restatement)".ljust(80, b"\0"))
        fh.write(struct.pack("<I", len(t)))
        for v in t:
            a = v[3:6].astype(np.float64) - v[0:3]
            b = v[6:9].astype(np.float64) - v[0:3]
            n = np.cross(a, b)
            ln = np.linalg.norm(n)
            nf = (n / ln).astype(np.float32) if ln > 0 else np.zeros(3, np.float32)
            fh.write(nf.astype("<f4").tobytes() + v.astype("<f4").tobytes() + b"\0\0")
