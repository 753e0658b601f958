"""Mesh voxelization on the device (orr_voxelize, orr_signed_distance_band)
against the reference's geom::voxelize and geom::signed_distance_band.

Bar: solid flags, band distances and band flags identical to the reference's;
winding numbers within 1e-12 (the only difference is the atan2 of the
solid angles).  Checked on the golden fixtures, on larger cases against the
reference library itself where it is built, and at the full 256 x 128 x 128
size through size-independent properties.
"""
import math
import os

import numpy as np
import pytest

from orrery_b200 import geometry as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = np.load(os.path.join(GOLDEN, "voxel_cases.npz"))
NAMES = [str(n) for n in CASES["names"]]
WINDING_TOL = 1e-12


def case(name):
    g = {k.split("/", 1)[1]: CASES[k] for k in CASES.files if k.startswith(name + "/")}
    spec = G.GridSpec(tuple(g["origin"]), float(g["spacing"]), *[int(x) for x in g["n"]])
    return g, G.TriangleMesh(g["vertices"], g["triangles"]), spec


@pytest.mark.parametrize("name", NAMES)
def test_golden_cases(name):
    g, mesh, spec = case(name)
    vox = G.voxelize(mesh, spec)
    assert np.array_equal(vox.solid, g["solid"])
    assert np.max(np.abs(vox.winding - g["winding"])) <= WINDING_TOL
    sdf = G.signed_distance_band(mesh, vox)
    assert sdf.band == float(g["band"])
    assert np.array_equal(sdf.distance, g["distance"])
    assert np.array_equal(sdf.in_band, g["in_band"])


def _reference():
    from oracle import oracle as O
    if not O.reference_available():
        pytest.skip("reference oracle library not built")
    return O


@pytest.mark.parametrize("shape", ["sphere_cone", "naca_wing"])
def test_against_reference_library(shape):
    """Meshes of a few thousand triangles on ~10^5 cells, against the reference
    library run here."""
    O = _reference()
    if shape == "sphere_cone":
        mesh = G.sphere_cone_mesh(0.5, math.radians(30.0), 0.12, 96, 24, 24)
        spacing = 0.02
    else:
        v, t = O.reference_mesh("naca_wing", "4415", 1.0, 1.2, 64, 16)
        mesh = G.TriangleMesh(v, t)
        spacing = 0.015
    lo, hi = mesh.bounds()
    spec = G.grid_around(lo, hi, spacing, 3)
    n = (spec.nx, spec.ny, spec.nz)
    solid, wind = O.reference_voxelize(mesh.vertices, mesh.triangles, spec.origin, spacing, n)
    vox = G.voxelize(mesh, spec)
    assert np.array_equal(vox.solid, solid)
    assert np.max(np.abs(vox.winding - wind)) <= WINDING_TOL
    dist, inb, band = O.reference_signed_distance_band(mesh.vertices, mesh.triangles, spec.origin, spacing, n,
                                                        solid)
    sdf = G.signed_distance_band(mesh, vox)
    assert sdf.band == band
    assert np.array_equal(sdf.distance, dist)
    assert np.array_equal(sdf.in_band, inb)


def test_full_size_properties():
    """A sphere of radius 32 cells in a 256 x 128 x 128 grid."""
    h = 1.0
    spec = G.GridSpec((-64.0, -64.0, -64.0), h, 256, 128, 128)
    mesh = G.sphere_mesh(32.0, 256, 127)
    vox = G.voxelize(mesh, spec)
    again = G.voxelize(mesh, spec)
    assert np.array_equal(vox.solid, again.solid) and np.array_equal(vox.winding, again.winding)
    polyhedron = sum(float(np.dot(mesh.vertices[a], np.cross(mesh.vertices[b], mesh.vertices[c])))
                     for a, b, c in mesh.triangles) / 6.0
    assert abs(vox.solid_count() * h ** 3 / polyhedron - 1.0) < 0.01
    # winding numbers are 0 or 1 away from the surface, to the tree's
    # far-field accuracy (the reference's own bound, test_voxel.cpp:259)
    sdf = G.signed_distance_band(mesh, vox)
    far = sdf.in_band == 0
    assert np.all(np.abs(vox.winding[far] - vox.solid[far]) < 0.05)
    assert np.all(np.abs(sdf.distance[far]) == sdf.band)
    assert np.all(np.abs(sdf.distance[~far]) < sdf.band)
    assert np.array_equal(np.signbit(sdf.distance), vox.solid == 1)
    # the band is the shell of cells within 3 cells of the sphere (polygon sagitta below 0.05)
    cz, cy, cx = np.meshgrid(np.arange(128) - 63.5, np.arange(128) - 63.5, np.arange(256) - 63.5, indexing="ij")
    r = np.sqrt(cx * cx + cy * cy + cz * cz).reshape(-1)
    inside_sure = (r < 32.0 - 0.1)
    assert np.all(vox.solid[inside_sure] == 1)
    assert np.all(vox.solid[r > 32.0 + 0.1] == 0)
    assert np.all(np.abs(np.abs(sdf.distance[~far]) - np.abs(r[~far] - 32.0)) < 0.1)


def test_threshold_and_empty_mesh():
    g, mesh, spec = case("sphere")
    high = G.voxelize(mesh, spec, threshold=1.5)
    assert high.solid_count() == 0
    low = G.voxelize(mesh, spec, threshold=-0.5)
    assert low.solid_count() == spec.cells()
    empty = G.TriangleMesh(np.zeros((0, 3)), np.zeros((0, 3), np.uint32))
    vox = G.voxelize(empty, spec)
    assert vox.solid_count() == 0 and np.all(vox.winding == 0.0)
    sdf = G.signed_distance_band(empty, vox)
    assert np.all(sdf.distance == sdf.band) and not sdf.in_band.any()
