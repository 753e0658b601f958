"""The voxelization oracle against the reference, and the library's host-side
grid logic (no GPU needed).

* The plain-Python restatement (oracle/voxel_oracle.py) reproduces the
  reference's geom::voxelize and geom::signed_distance_band fixtures
  (tests/golden/voxel_cases.npz, made by tests/golden/make_voxel_golden.py):
  solid flags and band distances exactly, winding numbers to 1e-12.
* It passes the reference's own known answers (tests/geom/test_voxel.cpp).
* orr_grid_around gives the reference's grids, and every refusal of
  orr_grid_around / orr_voxelize / orr_signed_distance_band carries the
  reference's text (tests/golden/voxel_messages.json); these refuse before
  any device work.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import voxel_oracle as V
from orrery_b200 import geometry as G
from orrery_b200._native import LbmError

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = np.load(os.path.join(GOLDEN, "voxel_cases.npz"))
NAMES = [str(n) for n in CASES["names"]]
MESSAGES = json.load(open(os.path.join(GOLDEN, "voxel_messages.json")))


def case(name):
    g = {k.split("/", 1)[1]: CASES[k] for k in CASES.files if k.startswith(name + "/")}
    g["n"] = [int(x) for x in g["n"]]
    return g


def cell_centre(g, c):
    nx, ny, _ = g["n"]
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    o, h = g["origin"], float(g["spacing"])
    return (o[0] + (i + 0.5) * h, o[1] + (j + 0.5) * h, o[2] + (k + 0.5) * h)


@pytest.mark.parametrize("name", NAMES)
def test_restatement_matches_reference(name):
    g = case(name)
    tree = V.Tree(g["vertices"], g["triangles"])
    band = float(g["band"])
    assert band == 3.0 * float(g["spacing"])
    cells = int(np.prod(g["n"]))
    # a deterministic sample of cells keeps the pure-Python check short
    for c in range(0, cells, 7 if len(g["triangles"]) < 1000 else 29):
        p = cell_centre(g, c)
        w = tree.winding(p)
        assert abs(w - g["winding"][c]) <= 1e-12, (c, w, g["winding"][c])
        assert (1 if w >= 0.5 else 0) == g["solid"][c]
        d = V.distance(g["vertices"], g["triangles"], p, band)
        assert (-1.0 if g["solid"][c] else 1.0) * d == g["distance"][c]
        assert (1 if d < band else 0) == g["in_band"][c]


def test_known_answers():
    """The reference's own checks (tests/geom/test_voxel.cpp:26-69, 207-260)."""
    o = (0.0, 0.0, 0.0)
    assert abs(V.solid_angle(o, (1, 0, 0), (0, 1, 0), (0, 0, 1)) - math.pi / 2) < 1e-15
    assert abs(V.solid_angle(o, (1, 0, 0), (0, 0, 1), (0, 1, 0)) + math.pi / 2) < 1e-15
    assert V.solid_angle((1, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)) == 0.0
    for s in (1e-150, 1e-3, 1.0, 1e3, 1e150):
        assert abs(V.solid_angle(o, (s, 0, 0), (0, s, 0), (0, 0, s)) - math.pi / 2) < 1e-14
    g = case("sphere")
    assert abs(V.winding_direct(g["vertices"], g["triangles"], (0.1, -0.2, 0.3)) - 1.0) < 1e-12
    assert abs(V.winding_direct(g["vertices"], g["triangles"], (1.5, 0.0, 0.2))) < 1e-12
    assert abs(V.winding_direct(g["vertices"], g["triangles"], (0.0, 0.0, 30.0))) < 1e-12
    h = case("open_hemisphere")
    assert V.winding_direct(h["vertices"], h["triangles"], (0.0, 0.0, 0.0)) > 0.25
    # closest points of degenerate triangles: a point, a segment
    p = (1.0, 2.0, 5.0)
    v = (1.0, 2.0, 3.0)
    q = V.closest_point(p, v, v, v)
    assert math.dist(q, p) == 2.0
    a, b = (0.0, 0.0, 0.0), (2.0, 0.0, 0.0)
    q = V.closest_point((3.0, 1.0, 0.0), a, b, b)
    assert abs(q[0] - 2.0) < 1e-15 and abs(q[1]) < 1e-15
    # the reference's vector length (its standard library's three-argument hypot)
    for x, want in zip(CASES["hypot/inputs"], CASES["hypot/values"]):
        assert V.hypot3(*map(float, x)) == want


@pytest.mark.parametrize("name", NAMES)
def test_grid_around_matches_reference(name):
    g = case(name)
    lo, hi = g["box"]
    s = G.grid_around(lo, hi, float(g["spacing"]), int(g["padding"]))
    assert [s.nx, s.ny, s.nz] == g["n"]
    assert np.array_equal(np.array(s.origin), g["origin"])


def test_refusal_texts():
    box = G.box_mesh(1.0, 1.0, 1.0)

    def refused(fn):
        with pytest.raises(LbmError) as e:
            fn()
        return str(e.value)

    m = MESSAGES
    assert refused(lambda: G.grid_around([0, 0, 0], [1, 1, 1], 0.0, 0)) == m["grid_spacing_zero"]
    assert refused(lambda: G.grid_around([0, 0, 0], [1, 1, 1], 1e-4, 0)) == m["grid_spacing_tiny"]
    assert refused(lambda: G.grid_around([1, 1, 1], [0, 0, 0], 0.25, 0)) == m["grid_unordered"]
    assert refused(lambda: G.grid_around([math.nan, 0, 0], [1, 1, 1], 0.25, 0)) == m["grid_nan"]
    assert refused(lambda: G.grid_around([-1e300, 0, 0], [1e300, 1, 1], 1.0, 0)) == m["grid_huge"]
    spec = lambda o, h, n: G.GridSpec(tuple(o), h, *n)   # noqa: E731
    assert refused(lambda: G.voxelize(box, spec([0, 0, 0], 0.5, [0, 4, 4]))) == m["voxelize_empty"]
    assert refused(lambda: G.voxelize(box, spec([0, 0, 0], 0.5, [1 << 62, 4, 4]))) == m["voxelize_wrapped"]
    assert refused(lambda: G.voxelize(box, spec([0, 0, 0], 0.5, [1 << 10, 1 << 10, 1 << 8]))) == m["voxelize_oversized"]
    assert refused(lambda: G.voxelize(box, spec([0, 0, 0], -0.5, [4, 4, 4]))) == m["voxelize_spacing"]
    assert refused(lambda: G.voxelize(box, spec([math.nan, 0, 0], 0.5, [4, 4, 4]))) == m["voxelize_origin"]
    assert refused(lambda: G.voxelize(box, spec([1.7e308, 0, 0], 1e307, [4, 4, 4]))) == m["voxelize_far"]
    assert refused(lambda: G.voxelize(box, spec([0, 0, 0], 0.5, [4, 4, 4]), math.nan)) == m["voxelize_threshold"]
    grid = G.VoxelGrid(spec([0, 0, 0], 0.5, [4, 4, 4]), np.zeros(64, np.uint8), None)
    assert refused(lambda: G.signed_distance_band(box, grid, 0.0)) == m["band_zero"]
    wrong = G.VoxelGrid(spec([0, 0, 0], 0.5, [4, 4, 5]), np.zeros(64, np.uint8), None)
    assert refused(lambda: G.signed_distance_band(box, wrong, 3.0)) == m["band_mismatch"]
    wide = G.VoxelGrid(spec([0, 0, 0], 1e300, [4, 4, 4]), np.zeros(64, np.uint8), None)
    assert refused(lambda: G.signed_distance_band(box, wide, 1e10)) == m["band_infinite"]
    flat = G.VoxelGrid(spec([0, 0, 0], 0.0, [4, 4, 4]), np.zeros(64, np.uint8), None)
    assert refused(lambda: G.signed_distance_band(box, flat, 3.0)) == m["band_grid"]
    # a corner index past the vertices is refused before any device work
    bad = G.TriangleMesh(box.vertices, np.array([[0, 1, 99]]))
    assert "out of range" in refused(lambda: G.voxelize(bad, spec([0, 0, 0], 0.5, [4, 4, 4])))


def test_own_meshes_are_closed_and_outward():
    for m, volume in ((G.box_mesh(1.0, 2.0, 3.0), 6.0),
                      (G.sphere_mesh(1.0, 64, 31), 4.0 / 3.0 * math.pi),
                      (G.sphere_cone_mesh(1.0, math.radians(25.0), 0.3, 64), None)):
        v, t = m.vertices, m.triangles
        signed = sum(float(np.dot(v[a], np.cross(v[b], v[c]))) for a, b, c in t) / 6.0
        assert signed > 0.0
        if volume is not None:
            assert abs(signed / volume - 1.0) < 0.01
        # every edge is shared by exactly two triangles, once in each direction
        edges = {}
        for a, b, c in t:
            for e in ((a, b), (b, c), (c, a)):
                edges[e] = edges.get(e, 0) + 1
        assert all(n == 1 and edges.get((e[1], e[0])) == 1 for e, n in edges.items())
