"""Golden fixtures of the mesh voxelization path, made by running the
reference's own geom::voxelize / geom::signed_distance_band / grid_around
(oracle/_ref, built from the reference sources) on small seeded cases.

    python tests/golden/make_voxel_golden.py

writes tests/golden/voxel_cases.npz and tests/golden/voxel_messages.json.
Needs the reference tree (to build oracle/_ref); the tests only read the
fixtures.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.normpath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from orrery_b200 import geometry as G  # noqa: E402


def open_hemisphere():
    v, t = O.reference_mesh("sphere", 1.0, 16, 0.4)
    keep = [i for i, tri in enumerate(t) if v[tri].mean(axis=0)[2] < 0.0]
    return v, t[keep]


def box_with_degenerates():
    v, t = O.reference_mesh("box", 1.0, 0.6, 0.4)
    v = np.concatenate([v, [[0.7, 0.1, 0.0], [0.9, 0.1, 0.0], [1.1, 0.1, 0.0]]])
    extra = np.array([[8, 8, 8], [8, 9, 10], [8, 9, 9]], np.uint32)   # a point, a line, a repeated edge
    return v, np.concatenate([t, extra])


def cases():
    out = []
    v, t = O.reference_mesh("sphere", 1.0, 16, 0.4)
    out.append(("sphere", v, t, 0.2, 2))
    v, t = O.reference_mesh("ellipsoid", 1.2, 0.6, 0.5, 24, 0.3)
    out.append(("ellipsoid", v, t, 0.15, 2))
    v, t = O.reference_mesh("cone", 0.5, 1.2, 20)
    out.append(("cone", v, t, 0.11, 2))
    v, t = O.reference_mesh("naca_wing", "2412", 1.0, 1.5, 24, 4)
    out.append(("naca_wing", v, t, 0.07, 2))
    v, t = open_hemisphere()
    out.append(("open_hemisphere", v, t, 0.2, 1))
    v, t = box_with_degenerates()
    out.append(("box_degenerate", v, t, 0.085, 2))
    m = G.sphere_cone_mesh(0.5, math.radians(25.0), 0.15, 24)
    out.append(("sphere_cone", m.vertices, m.triangles, 0.06, 3))
    return out


def messages():
    """Refusal texts of the reference for bad grids, thresholds and bands."""
    v, t = O.reference_mesh("box", 1.0, 1.0, 1.0)
    res = {}

    def grab(name, fn):
        try:
            fn()
            res[name] = ""
        except O.ReferenceError_ as e:
            res[name] = str(e)

    grab("grid_spacing_zero", lambda: O.reference_grid_around([0, 0, 0], [1, 1, 1], 0.0, 0))
    grab("grid_spacing_tiny", lambda: O.reference_grid_around([0, 0, 0], [1, 1, 1], 1e-4, 0))
    grab("grid_unordered", lambda: O.reference_grid_around([1, 1, 1], [0, 0, 0], 0.25, 0))
    grab("grid_nan", lambda: O.reference_grid_around([math.nan, 0, 0], [1, 1, 1], 0.25, 0))
    grab("grid_huge", lambda: O.reference_grid_around([-1e300, 0, 0], [1e300, 1, 1], 1.0, 0))
    grab("voxelize_empty", lambda: O.reference_voxelize(v, t, [0, 0, 0], 0.5, [0, 4, 4]))
    grab("voxelize_wrapped", lambda: O.reference_voxelize(v, t, [0, 0, 0], 0.5, [1 << 62, 4, 4]))
    grab("voxelize_oversized", lambda: O.reference_voxelize(v, t, [0, 0, 0], 0.5, [1 << 10, 1 << 10, 1 << 8]))
    grab("voxelize_spacing", lambda: O.reference_voxelize(v, t, [0, 0, 0], -0.5, [4, 4, 4]))
    grab("voxelize_origin", lambda: O.reference_voxelize(v, t, [math.nan, 0, 0], 0.5, [4, 4, 4]))
    grab("voxelize_far", lambda: O.reference_voxelize(v, t, [1.7e308, 0, 0], 1e307, [4, 4, 4]))
    grab("voxelize_threshold", lambda: O.reference_voxelize(v, t, [0, 0, 0], 0.5, [4, 4, 4], math.nan))
    solid = np.zeros(64, np.uint8)
    grab("band_zero", lambda: O.reference_signed_distance_band(v, t, [0, 0, 0], 0.5, [4, 4, 4], solid, 0.0))
    grab("band_mismatch", lambda: O.reference_signed_distance_band(v, t, [0, 0, 0], 0.5, [4, 4, 5], solid, 3.0))
    grab("band_infinite", lambda: O.reference_signed_distance_band(v, t, [0, 0, 0], 1e300, [4, 4, 4], solid, 1e10))
    grab("band_grid", lambda: O.reference_signed_distance_band(v, t, [0, 0, 0], 0.0, [4, 4, 4], solid, 3.0))
    return res


def main():
    arrays = {}
    names = []
    for name, v, t, spacing, padding in cases():
        lo, hi = v.min(axis=0), v.max(axis=0)
        origin, n = O.reference_grid_around(lo, hi, spacing, padding)
        solid, wind = O.reference_voxelize(v, t, origin, spacing, n)
        dist, inb, band = O.reference_signed_distance_band(v, t, origin, spacing, n, solid)
        p = name + "/"
        arrays[p + "vertices"] = v
        arrays[p + "triangles"] = t
        arrays[p + "box"] = np.array([lo, hi])
        arrays[p + "origin"] = origin
        arrays[p + "spacing"] = np.array(spacing)
        arrays[p + "padding"] = np.array(padding)
        arrays[p + "n"] = np.array(n, np.int64)
        arrays[p + "solid"] = solid
        arrays[p + "winding"] = wind
        arrays[p + "distance"] = dist
        arrays[p + "in_band"] = inb
        arrays[p + "band"] = np.array(band)
        names.append(name)
        print(name, len(t), "triangles", n, int(solid.sum()), "solid", int(inb.sum()), "in band")
    arrays["names"] = np.array(names)
    # the reference's vector length (std::hypot of three values) on seeded inputs
    rng = np.random.default_rng(3)
    inputs = rng.standard_normal((4000, 3)) * 10.0 ** rng.integers(-8, 8, (4000, 3))
    lib = O._geom_lib()
    arrays["hypot/inputs"] = inputs
    arrays["hypot/values"] = np.array([lib.ref_hypot3(*map(float, x)) for x in inputs])
    np.savez_compressed(os.path.join(HERE, "voxel_cases.npz"), **arrays)
    with open(os.path.join(HERE, "voxel_messages.json"), "w") as fh:
        json.dump(messages(), fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
