"""Host transfers of full-size lattices.  Uploads and read-backs of 8 MiB or
more go through the library's pinned staging ring (chunks of 4 MiB, several
host threads); smaller ones take a plain copy.  These cases put every staged
path through lattices whose planes are not whole multiples of a chunk:
initialize (four field planes up), macroscopic (four planes back),
populations (the binary64 array, and the raw 4-byte values widened on the
host), and a mask upload of more than 8 MiB at creation.  An equilibrium
state returns its own fields, so a misplaced or stale chunk shows as an
error of order one."""
import numpy as np
import pytest

from orrery_b200 import solver as S
from orrery_b200.lbm3d import periodic_box
from orrery_b200.masks import SolidMask3D

pytestmark = pytest.mark.gpu

# 33,419,520 bytes per binary64 plane: eight chunks minus a ragged tail
SHAPE = (255, 127, 129)

# D3Q19 directions and weights in the solver's order (d3q19.h)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def _fields(seed):
    rng = np.random.default_rng(seed)
    n = SHAPE[0] * SHAPE[1] * SHAPE[2]
    rho = 1.0 + 0.05 * rng.standard_normal(n)
    u = [0.03 * rng.standard_normal(n) for _ in range(3)]
    return rho, u


@pytest.mark.parametrize("storage,tol", [("f64", 1e-13), ("f32", 2e-6)])
def test_initialize_and_macroscopic_round_trip(storage, tol):
    nx, ny, nz = SHAPE
    cfg = periodic_box(nx, ny, nz, 0.8)
    mask = SolidMask3D(nx, ny, nz, np.zeros(nx * ny * nz, np.uint8), None)
    rho, (ux, uy, uz) = _fields(7)
    with S.make_gpu_solver(cfg, mask, storage=storage) as s:
        s.initialize(rho, ux, uy, uz)
        m = s.macroscopic()
    assert np.abs(m.density - rho).max() < tol
    for got, want in ((m.velocity_x, ux), (m.velocity_y, uy), (m.velocity_z, uz)):
        assert np.abs(got - want).max() < tol


def _equilibrium(rho, ux, uy, uz):
    f = np.empty((19, rho.size))
    usq = ux * ux + uy * uy + uz * uz
    for i in range(19):
        cu = CX[i] * ux + CY[i] * uy + CZ[i] * uz
        f[i] = W[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return f.reshape(-1)


@pytest.mark.parametrize("storage,tol", [("f64", 1e-14), ("f32", 2e-7)])
def test_populations_read_back(storage, tol):
    nx, ny, nz = SHAPE
    cfg = periodic_box(nx, ny, nz, 0.8)
    mask = SolidMask3D(nx, ny, nz, np.zeros(nx * ny * nz, np.uint8), None)
    rho, (ux, uy, uz) = _fields(8)
    with S.make_gpu_solver(cfg, mask, storage=storage) as s:
        s.initialize(rho, ux, uy, uz)
        f = s.populations()
    assert np.abs(f - _equilibrium(rho, ux, uy, uz)).max() < tol


def test_mask_upload_of_a_full_size_lattice():
    """The class and bounce-back tables (21 MB here) go up in one staged
    upload: a solid slab's rest state and the mass of the fluid around it
    come back as placed."""
    nx, ny, nz = SHAPE
    cfg = periodic_box(nx, ny, nz, 0.8)
    solid = np.zeros((nz, ny, nx), np.uint8)
    solid[:, :, 100:110] = 1
    mask = SolidMask3D(nx, ny, nz, solid.reshape(-1), None)
    rho, (ux, uy, uz) = _fields(9)
    with S.make_gpu_solver(cfg, mask, storage="f64") as s:
        s.initialize(rho, ux, uy, uz)
        s.step(2)
        m = s.macroscopic()
        f = s.populations().reshape(19, -1)
    fluid = solid.reshape(-1) == 0
    # solids hold the rest populations and report no motion
    assert np.array_equal(f[:, ~fluid], np.repeat(W[:, None], (~fluid).sum(), 1))
    assert np.all(m.velocity_x[~fluid] == 0.0)
    assert abs(f[:, fluid].sum() - rho[fluid].sum()) < 1e-9 * fluid.sum()


def test_read_back_into_earlier_arrays():
    """macroscopic(out=...) and populations(out=...) write into the arrays of an
    earlier call (no fresh pages) and give the same bits; arrays of the wrong
    size or type are refused before anything is copied."""
    nx, ny, nz = SHAPE
    cfg = periodic_box(nx, ny, nz, 0.8)
    mask = SolidMask3D(nx, ny, nz, np.zeros(nx * ny * nz, np.uint8), None)
    rho, (ux, uy, uz) = _fields(10)
    with S.make_gpu_solver(cfg, mask) as s:
        s.initialize(rho, ux, uy, uz)
        m = s.macroscopic()
        f = s.populations()
        s.step(3)
        m2 = s.macroscopic(out=m)
        f2 = s.populations(out=f)
        assert m2 is m and f2 is f
        fresh, fresh_f = s.macroscopic(), s.populations()
        for a, b in ((m.density, fresh.density), (m.velocity_x, fresh.velocity_x),
                     (m.velocity_y, fresh.velocity_y), (m.velocity_z, fresh.velocity_z), (f, fresh_f)):
            assert np.array_equal(a, b)
        with pytest.raises(S.LbmError):
            s.populations(out=np.empty(10))
        bad = S.MacroFields3D(nx, ny, nz, m.density.astype(np.float32), m.velocity_x, m.velocity_y,
                              m.velocity_z, m.solid)
        with pytest.raises(S.LbmError):
            s.macroscopic(out=bad)
    # fields filled by another solver of the same size carry this solver's mask
    solid2 = np.zeros(nx * ny * nz, np.uint8)
    solid2[::7] = 1
    with S.make_gpu_solver(cfg, SolidMask3D(nx, ny, nz, solid2, None)) as s2:
        m3 = s2.macroscopic(out=m)
        assert m3 is m and np.array_equal(m.solid.reshape(-1), solid2)
        assert np.array_equal(s2.macroscopic().solid, m.solid)
