"""CPU restatement of the reference's mesh voxelization.  TEST INFRASTRUCTURE ONLY.

Plain-Python binary64 restatement of geom::voxelize and
geom::signed_distance_band (src/geom/voxel_grid.cpp:84-140) with the
bounding-volume tree of src/geom/winding_number.cpp:164-309, for the small
cases the tests run (a few thousand cells, a few hundred triangles).  It is a
checker of the device path, never part of it.

Differences from the reference that the tests allow for: the tree's leaves
hold the same triangles but in sorted order (the reference's order comes from
std::nth_element), so node sums and the winding sum run in another order
(last-bit differences); the distance is the minimum over every triangle,
which equals the pruned tree search exactly.
"""
from __future__ import annotations

import math

FOUR_PI = 4.0 * math.pi


def hypot3(x, y, z):
    """norm of src/geom/include/orrery/geom/vector3.h:57-59 (the standard
    library's three-argument hypot: largest magnitude times the root of the
    sum of squared ratios)."""
    x, y, z = abs(x), abs(y), abs(z)
    m = (z if y < z else y) if x < y else (z if x < z else x)
    if m == 0.0:
        return 0.0
    qx, qy, qz = x / m, y / m, z / m
    return m * math.sqrt(qx * qx + qy * qy + qz * qz)


def _sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def _add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def _mul(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def _div(a, s):
    return (a[0] / s, a[1] / s, a[2] / s)


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _norm(a):
    return hypot3(*a)


def solid_angle(p, a, b, c):
    """winding_number.cpp:101-122."""
    ra, rb, rc = _sub(a, p), _sub(b, p), _sub(c, p)
    la, lb, lc = _norm(ra), _norm(rb), _norm(rc)
    if not (la > 0.0) or not (lb > 0.0) or not (lc > 0.0):
        return 0.0
    ua, ub, uc = _div(ra, la), _div(rb, lb), _div(rc, lc)
    num = _dot(ua, _cross(ub, uc))
    den = 1.0 + _dot(ua, ub) + _dot(ub, uc) + _dot(uc, ua)
    return 2.0 * math.atan2(num, den)


def winding_direct(vertices, triangles, p):
    """winding_number.cpp:124-130: direct sum over every triangle."""
    s = 0.0
    for t in triangles:
        s += solid_angle(p, vertices[t[0]], vertices[t[1]], vertices[t[2]])
    return s / FOUR_PI


def _segment_point(p, a, b):
    ab = _sub(b, a)
    l2 = _dot(ab, ab)
    if not (l2 > 0.0):
        return a
    t = _dot(_sub(p, a), ab) / l2
    t = 0.0 if t < 0.0 else (1.0 if 1.0 < t else t)
    return _add(a, _mul(ab, t))


def _edges_point(p, a, b, c):
    best = _segment_point(p, a, b)
    d = _sub(best, p)
    best2 = _dot(d, d)
    for q in (_segment_point(p, b, c), _segment_point(p, c, a)):
        d = _sub(q, p)
        d2 = _dot(d, d)
        if d2 < best2:
            best, best2 = q, d2
    return best


def closest_point(p, a, b, c):
    """winding_number.cpp:131-176 (Ericson 5.1.5 with degenerate fallbacks)."""
    ab, ac = _sub(b, a), _sub(c, a)
    n = _cross(ab, ac)
    if not (_dot(n, n) > 0.0):
        return _edges_point(p, a, b, c)
    ap = _sub(p, a)
    d1, d2 = _dot(ab, ap), _dot(ac, ap)
    if d1 <= 0.0 and d2 <= 0.0:
        return a
    bp = _sub(p, b)
    d3, d4 = _dot(ab, bp), _dot(ac, bp)
    if d3 >= 0.0 and d4 <= d3:
        return b
    vc = d1 * d4 - d3 * d2
    if vc <= 0.0 and d1 >= 0.0 and d3 <= 0.0:
        return _add(a, _mul(ab, d1 / (d1 - d3)))
    cp = _sub(p, c)
    d5, d6 = _dot(ab, cp), _dot(ac, cp)
    if d6 >= 0.0 and d5 <= d6:
        return c
    vb = d5 * d2 - d1 * d6
    if vb <= 0.0 and d2 >= 0.0 and d6 <= 0.0:
        return _add(a, _mul(ac, d2 / (d2 - d6)))
    va = d3 * d6 - d5 * d4
    if va <= 0.0 and (d4 - d3) >= 0.0 and (d5 - d6) >= 0.0:
        return _add(b, _mul(_sub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))))
    s = va + vb + vc
    if not (s > 0.0):
        return _edges_point(p, a, b, c)
    return _add(_add(a, _mul(ab, vb / s)), _mul(ac, vc / s))


class Tree:
    """MeshTree (winding_number.cpp:178-279) with beta 2 and leaves of 8."""

    def __init__(self, vertices, triangles, beta=2.0, leaf=8):
        self.v = [tuple(map(float, x)) for x in vertices]
        self.t = [tuple(int(i) for i in x) for x in triangles]
        self.beta = beta
        self.leaf = leaf
        if self.v:
            lo = [min(x[k] for x in self.v) for k in range(3)]
            hi = [max(x[k] for x in self.v) for k in range(3)]
            ext = max(hi[k] - lo[k] for k in range(3))
        else:
            ext = 0.0
        self.scale = math.ldexp(1.0, math.frexp(ext)[1] - 1) if ext > 0.0 and math.isfinite(ext) else 1.0
        self.nodes = []
        if self.t:
            self._build(list(range(len(self.t))))

    def _centroid(self, t):
        a, b, c = (self.v[i] for i in self.t[t])
        return _div(_add(_add(a, b), c), 3.0)

    def _build(self, tris):
        idx = len(self.nodes)
        self.nodes.append(None)
        corners = [self.v[i] for t in tris for i in self.t[t]]
        lo = tuple(min(c[k] for c in corners) for k in range(3))
        hi = tuple(max(c[k] for c in corners) for k in range(3))
        cents = [self._centroid(t) for t in tris]
        area_vec, weighted, area = (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 0.0
        for t, c in zip(tris, cents):
            a, b, d = (self.v[i] for i in self.t[t])
            n2 = _cross(_div(_sub(b, a), self.scale), _div(_sub(d, a), self.scale))
            half = 0.5 * _norm(n2)
            area_vec = _add(area_vec, _mul(n2, 0.5))
            weighted = _add(weighted, _mul(c, half))
            area += half
        centre = _div(weighted, area) if area > 0.0 else _mul(_add(lo, hi), 0.5)
        node = {"lo": lo, "hi": hi, "centre": centre, "area": area_vec, "tris": None, "kids": None}
        if len(tris) <= self.leaf:
            node["tris"] = tris
            node["radius"] = max(_norm(_sub(self.v[i], centre)) for t in tris for i in self.t[t])
        else:
            e = [max(c[k] for c in cents) - min(c[k] for c in cents) for k in range(3)]
            axis = 0 if (e[0] >= e[1] and e[0] >= e[2]) else (1 if e[1] >= e[2] else 2)
            order = sorted(range(len(tris)), key=lambda i: (cents[i][axis], tris[i]))
            ordered = [tris[i] for i in order]
            half = len(tris) // 2
            left = self._build(ordered[:half])
            right = self._build(ordered[half:])
            node["kids"] = (left, right)
            node["radius"] = max(_norm(_sub(self.nodes[k]["centre"], centre)) + self.nodes[k]["radius"]
                                 for k in (left, right))
        self.nodes[idx] = node
        return idx

    def winding(self, p):
        if not self.nodes:
            return 0.0
        s = 0.0
        stack = [0]
        while stack:
            n = self.nodes[stack.pop()]
            d = _sub(n["centre"], p)
            dist = _norm(d)
            if dist > self.beta * n["radius"]:
                flux = _dot(n["area"], _div(d, dist))
                if flux != 0.0:
                    r = self.scale / dist
                    s += flux * r * r
                continue
            if n["tris"] is not None:
                for t in n["tris"]:
                    a, b, c = (self.v[i] for i in self.t[t])
                    s += solid_angle(p, a, b, c)
                continue
            stack.append(n["kids"][0])
            stack.append(n["kids"][1])
        return s / FOUR_PI


def distance(vertices, triangles, p, max_distance):
    """Distance from p to the closest triangle, or max_distance when none is
    closer (the result of MeshTree::distance, by exhaustive search)."""
    best2 = max_distance * max_distance
    if len(triangles) == 0:
        return max_distance
    for t in triangles:
        a, b, c = (tuple(map(float, vertices[i])) for i in t)
        q = _sub(closest_point(p, a, b, c), p)
        d2 = _dot(q, q)
        best2 = d2 if d2 < best2 else best2
    return math.sqrt(best2)


def voxelize(vertices, triangles, origin, spacing, n, threshold=0.5):
    """Solid flags and winding numbers of every cell, x fastest."""
    tree = Tree(vertices, triangles)
    solid, wind = [], []
    nx, ny, nz = n
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                p = (origin[0] + (i + 0.5) * spacing, origin[1] + (j + 0.5) * spacing,
                     origin[2] + (k + 0.5) * spacing)
                w = tree.winding(p)
                wind.append(w)
                solid.append(1 if w >= threshold else 0)
    return solid, wind


def signed_distance_band(vertices, triangles, origin, spacing, n, solid, band_cells=3.0):
    band = band_cells * spacing
    dist, inb = [], []
    nx, ny, nz = n
    c = 0
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                p = (origin[0] + (i + 0.5) * spacing, origin[1] + (j + 0.5) * spacing,
                     origin[2] + (k + 0.5) * spacing)
                d = distance(vertices, triangles, p, band)
                inb.append(1 if d < band else 0)
                dist.append((-1.0 if solid[c] else 1.0) * d)
                c += 1
    return dist, inb, band
