// geom::voxelize, geom::signed_distance_band and geom::grid_around on the B200
// library: the file a maintainer builds in place of src/geom/voxel_grid.cpp of
// the reference so that every caller (LbmAeroSolver3D::setup among them,
// lbm_aero_solver3d.cpp:249-258) voxelizes on the device.  Same declarations
// (src/geom/include/orrery/geom/voxel_grid.h), same results: the solid flags,
// band flags and distances are the reference's bit for bit, the winding
// numbers within 1e-12; refusals throw std::invalid_argument with the
// reference's texts.  Device 0 unless ORR_VOXEL_DEVICE names another.
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "orrery/geom/voxel_grid.h"
#include "orrery_lbm.h"

namespace orrery::geom {
namespace {

struct FlatMesh {
    std::vector<double> vertices;
    std::vector<std::uint32_t> triangles;
    orr_mesh view{};
    explicit FlatMesh(const TriangleMesh& m) {
        vertices.reserve(3 * m.vertices.size());
        for (const Vector3& v : m.vertices) {
            vertices.insert(vertices.end(), {v.x, v.y, v.z});
        }
        triangles.reserve(3 * m.triangles.size());
        for (const Triangle& t : m.triangles) {
            triangles.insert(triangles.end(), {t[0], t[1], t[2]});
        }
        view = orr_mesh{vertices.data(), m.vertices.size(), triangles.data(), m.triangles.size()};
    }
};

orr_grid_spec spec_of(const GridSpec& s) {
    orr_grid_spec o{};
    o.origin[0] = s.origin.x;
    o.origin[1] = s.origin.y;
    o.origin[2] = s.origin.z;
    o.spacing = s.spacing;
    o.nx = s.nx;
    o.ny = s.ny;
    o.nz = s.nz;
    return o;
}

int device() {
    const char* d = std::getenv("ORR_VOXEL_DEVICE");
    return d != nullptr ? std::atoi(d) : 0;
}

// Cells of a grid whose count is in range (checked without wrapping), else 1:
// the library refuses such a grid before it writes anything.
std::size_t output_cells(const GridSpec& s) {
    const bool ok = s.nx > 0 && s.ny > 0 && s.nz > 0 && s.nx <= max_grid_cells / s.ny &&
                    s.nx * s.ny <= max_grid_cells / s.nz;
    return ok ? s.cells() : 1;
}

[[noreturn]] void raise(orr_status status) {
    if (status == ORR_ERR_INVALID) {
        throw std::invalid_argument(orr_last_error());
    }
    throw std::runtime_error(orr_last_error());
}

} // namespace

Vector3 GridSpec::centre(std::size_t i, std::size_t j, std::size_t k) const noexcept {
    return origin + Vector3{(static_cast<double>(i) + 0.5) * spacing, (static_cast<double>(j) + 0.5) * spacing,
                            (static_cast<double>(k) + 0.5) * spacing};
}

std::size_t VoxelGrid::solid_count() const noexcept {
    std::size_t n = 0;
    for (const std::uint8_t s : solid) {
        n += s == 1 ? 1 : 0;
    }
    return n;
}

GridSpec grid_around(const Bounds& box, double spacing, std::size_t padding) {
    const double lo[3] = {box.min.x, box.min.y, box.min.z};
    const double hi[3] = {box.max.x, box.max.y, box.max.z};
    orr_grid_spec g{};
    const orr_status st = orr_grid_around(lo, hi, spacing, padding, &g);
    if (st != ORR_OK) {
        raise(st);
    }
    GridSpec out;
    out.origin = {g.origin[0], g.origin[1], g.origin[2]};
    out.spacing = g.spacing;
    out.nx = g.nx;
    out.ny = g.ny;
    out.nz = g.nz;
    return out;
}

VoxelGrid voxelize(const TriangleMesh& mesh, const GridSpec& spec, double threshold) {
    const FlatMesh m(mesh);
    const orr_grid_spec g = spec_of(spec);
    VoxelGrid grid;
    grid.spec = spec;
    grid.solid.assign(output_cells(spec), 0);
    grid.winding.assign(output_cells(spec), 0.0);
    const orr_status st = orr_voxelize(&m.view, &g, threshold, device(), grid.solid.data(), grid.winding.data(),
                                       nullptr);
    if (st != ORR_OK) {
        raise(st);
    }
    return grid;
}

SignedDistanceField signed_distance_band(const TriangleMesh& mesh, const VoxelGrid& voxels, double band_cells) {
    const FlatMesh m(mesh);
    const orr_grid_spec g = spec_of(voxels.spec);
    SignedDistanceField sdf;
    sdf.spec = voxels.spec;
    const std::size_t n = voxels.solid.size();
    sdf.distance.assign(n, 0.0);
    sdf.in_band.assign(n, 0);
    const orr_status st = orr_signed_distance_band(&m.view, &g, voxels.solid.data(), n, band_cells, device(),
                                                   sdf.distance.data(), sdf.in_band.data(), &sdf.band, nullptr);
    if (st != ORR_OK) {
        raise(st);
    }
    return sdf;
}

} // namespace orrery::geom
