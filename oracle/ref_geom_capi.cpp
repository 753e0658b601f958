// C entry points over Orrery's own mesh voxelization (src/geom/voxel_grid.cpp,
// src/geom/winding_number.cpp) and its mesh builders (src/geom/primitives.cpp,
// src/geom/naca.cpp), compiled from the reference sources in place by
// oracle/Makefile into oracle/_ref/libref_lbm.so.
//
// TEST INFRASTRUCTURE ONLY.  This is the reference oracle of the geometry path:
// the golden fixtures, the checks of the restatement in oracle/voxel_oracle.py
// and the CPU baseline of the voxelization benchmark come from it.  The
// product never links or loads it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "orrery/geom/naca.h"
#include "orrery/geom/primitives.h"
#include "orrery/geom/voxel_grid.h"
#include "orrery/geom/winding_number.h"

namespace geom = orrery::geom;

namespace {

void copy_message(const std::string& text, char* message, size_t capacity) {
    if (message == nullptr || capacity == 0) {
        return;
    }
    const size_t n = text.size() < capacity - 1 ? text.size() : capacity - 1;
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

geom::TriangleMesh mesh_of(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt) {
    geom::TriangleMesh m;
    m.vertices.resize(nv);
    for (uint64_t i = 0; i < nv; ++i) {
        m.vertices[i] = {vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
    }
    m.triangles.resize(nt);
    for (uint64_t t = 0; t < nt; ++t) {
        m.triangles[t] = {triangles[3 * t], triangles[3 * t + 1], triangles[3 * t + 2]};
    }
    return m;
}

geom::GridSpec spec_of(const double origin[3], double spacing, uint64_t nx, uint64_t ny, uint64_t nz) {
    geom::GridSpec s;
    s.origin = {origin[0], origin[1], origin[2]};
    s.spacing = spacing;
    s.nx = nx;
    s.ny = ny;
    s.nz = nz;
    return s;
}

// Mesh built last by a ref_mesh_* call, read back by ref_mesh_copy.
geom::TriangleMesh g_mesh;

void keep(const geom::TriangleMesh& m, uint64_t* nv, uint64_t* nt) {
    g_mesh = m;
    *nv = g_mesh.vertices.size();
    *nt = g_mesh.triangles.size();
}

} // namespace

extern "C" {

// Mesh builders: each keeps its mesh and returns the vertex and triangle
// counts; ref_mesh_copy writes it out (3 doubles per vertex, 3 indices per
// triangle).  0 on success, -1 with the reference's message otherwise.
int ref_mesh_sphere(double radius, int around, double arc_step, uint64_t* nv, uint64_t* nt, char* message,
                    size_t capacity) {
    try {
        keep(geom::sphere_profile(radius).mesh(geom::RevolutionResolution{around, arc_step}), nv, nt);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

int ref_mesh_ellipsoid(double a, double b, double c, int around, double arc_step, uint64_t* nv, uint64_t* nt,
                       char* message, size_t capacity) {
    try {
        keep(geom::Ellipsoid{a, b, c}.mesh(geom::RevolutionResolution{around, arc_step}), nv, nt);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

int ref_mesh_cone(double radius, double height, int around, uint64_t* nv, uint64_t* nt, char* message,
                  size_t capacity) {
    try {
        keep(geom::cone_profile(radius, height).mesh(geom::RevolutionResolution{around, 0.05}), nv, nt);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

int ref_mesh_box(double lx, double ly, double lz, uint64_t* nv, uint64_t* nt, char* message, size_t capacity) {
    try {
        keep(geom::box_mesh(lx, ly, lz), nv, nt);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

int ref_mesh_naca_wing(const char* digits, double chord, double span, int n, int span_divisions, uint64_t* nv,
                       uint64_t* nt, char* message, size_t capacity) {
    try {
        const auto airfoil = geom::Naca4::from_designation(digits);
        if (!airfoil) {
            copy_message("not a NACA 4-digit designation", message, capacity);
            return -1;
        }
        keep(geom::naca_wing(*airfoil, chord, span, n, span_divisions).mesh, nv, nt);
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

void ref_mesh_copy(double* vertices, uint32_t* triangles) {
    for (size_t i = 0; i < g_mesh.vertices.size(); ++i) {
        vertices[3 * i] = g_mesh.vertices[i].x;
        vertices[3 * i + 1] = g_mesh.vertices[i].y;
        vertices[3 * i + 2] = g_mesh.vertices[i].z;
    }
    for (size_t t = 0; t < g_mesh.triangles.size(); ++t) {
        for (int k = 0; k < 3; ++k) {
            triangles[3 * t + k] = g_mesh.triangles[t][k];
        }
    }
}

// geom::grid_around: writes origin[3], spacing, n[3].
int ref_grid_around(const double lo[3], const double hi[3], double spacing, uint64_t padding, double origin[3],
                    uint64_t n[3], char* message, size_t capacity) {
    try {
        const geom::Bounds box{{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
        const geom::GridSpec g = geom::grid_around(box, spacing, padding);
        origin[0] = g.origin.x;
        origin[1] = g.origin.y;
        origin[2] = g.origin.z;
        n[0] = g.nx;
        n[1] = g.ny;
        n[2] = g.nz;
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// geom::voxelize: solid flags and winding numbers of every cell.
int ref_voxelize(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt,
                 const double origin[3], double spacing, uint64_t nx, uint64_t ny, uint64_t nz, double threshold,
                 uint8_t* solid, double* winding, char* message, size_t capacity) {
    try {
        const geom::TriangleMesh m = mesh_of(vertices, nv, triangles, nt);
        const geom::VoxelGrid g = geom::voxelize(m, spec_of(origin, spacing, nx, ny, nz), threshold);
        std::memcpy(solid, g.solid.data(), g.solid.size());
        std::memcpy(winding, g.winding.data(), g.winding.size() * sizeof(double));
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// geom::signed_distance_band on the given solid flags (a VoxelGrid of the
// spec); writes the distances, the in-band flags and the band width.
int ref_signed_distance_band(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt,
                             const double origin[3], double spacing, uint64_t nx, uint64_t ny, uint64_t nz,
                             const uint8_t* solid, uint64_t solid_count, double band_cells, double* distance,
                             uint8_t* in_band, double* band, char* message, size_t capacity) {
    try {
        const geom::TriangleMesh m = mesh_of(vertices, nv, triangles, nt);
        geom::VoxelGrid g;
        g.spec = spec_of(origin, spacing, nx, ny, nz);
        g.solid.assign(solid, solid + solid_count);
        const geom::SignedDistanceField f = geom::signed_distance_band(m, g, band_cells);
        std::memcpy(distance, f.distance.data(), f.distance.size() * sizeof(double));
        std::memcpy(in_band, f.in_band.data(), f.in_band.size());
        *band = f.band;
        return 0;
    } catch (const std::exception& e) {
        copy_message(e.what(), message, capacity);
        return -1;
    }
}

// Direct-sum winding number and tree queries at single points (known answers).
double ref_winding_direct(const double* vertices, uint64_t nv, const uint32_t* triangles, uint64_t nt,
                          const double p[3]) {
    const geom::TriangleMesh m = mesh_of(vertices, nv, triangles, nt);
    return geom::winding_number(m, {p[0], p[1], p[2]});
}

double ref_solid_angle(const double p[3], const double a[3], const double b[3], const double c[3]) {
    return geom::solid_angle({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
}

void ref_closest_point(const double p[3], const double a[3], const double b[3], const double c[3], double out[3]) {
    const geom::Vector3 q = geom::closest_point_on_triangle({p[0], p[1], p[2]}, {a[0], a[1], a[2]},
                                                           {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
    out[0] = q.x;
    out[1] = q.y;
    out[2] = q.z;
}

double ref_hypot3(double x, double y, double z) {
    return geom::norm({x, y, z});
}

} // extern "C"
