// Host-side planning and validation of D3Q19 and D2Q9 lattices.
#include "plan.h"

#include <algorithm>
#include <thread>
#include <cmath>
#include <iomanip>
#include <limits>
#include <sstream>

#include "lattice.h"

namespace orr {

namespace {

constexpr double kMaxLatticeMach = 0.1; // max_lattice_mach (lattice_units.h:22)

bool finite(double v) {
    return std::isfinite(v);
}

// Whether any of the n values is a NaN (the only value unequal to itself).
// Blocks of 4096 values are tested whole, which the compiler vectorises, and
// large arrays are split over host threads.
bool any_nan(const double* v, std::size_t n) {
    const auto scan = [v](std::size_t a, std::size_t b) {
        for (std::size_t k = a; k < b; k += 4096) {
            const std::size_t e = std::min(b, k + 4096);
            bool bad = false;
            for (std::size_t i = k; i < e; ++i) {
                bad |= v[i] != v[i];
            }
            if (bad) {
                return true;
            }
        }
        return false;
    };
    const std::size_t workers = n >= (std::size_t{1} << 20)
                                    ? std::min<std::size_t>(std::max(1u, std::thread::hardware_concurrency()), 16)
                                    : 1;
    if (workers == 1) {
        return scan(0, n);
    }
    std::vector<char> found(workers, 0);
    std::vector<std::thread> pool;
    for (std::size_t w = 0; w < workers; ++w) {
        pool.emplace_back([&, w] { found[w] = scan(n * w / workers, n * (w + 1) / workers) ? 1 : 0; });
    }
    for (std::thread& t : pool) t.join();
    return std::find(found.begin(), found.end(), 1) != found.end();
}

double lattice_mach(double speed) {
    // lattice_mach (src/aero/lbm/lattice_units.cpp:19-21): |u| / sqrt(c_s^2).
    return std::abs(speed) / std::sqrt(1.0 / 3.0);
}

// check_mach (lbm3d_common.cpp:21-30; lbm2d_common.cpp:18-27).
std::string check_mach(const char* family, const char* what, double speed) {
    if (!(lattice_mach(speed) < kMaxLatticeMach)) {
        std::ostringstream m;
        m << family << ": " << what << " " << speed << " has lattice Mach number "
          << lattice_mach(speed) << ", not below " << kMaxLatticeMach << " (APPROXIMATION A3)";
        return m.str();
    }
    return {};
}

// a * b without wrapping.
bool mul(std::size_t a, std::size_t b, std::size_t& out) {
    if (a != 0 && b > std::numeric_limits<std::size_t>::max() / a) {
        return false;
    }
    out = a * b;
    return true;
}

bool add(std::size_t a, std::size_t b, std::size_t& out) {
    if (b > std::numeric_limits<std::size_t>::max() - a) {
        return false;
    }
    out = a + b;
    return true;
}

// lattice_cells_3d (src/aero/lbm3d/solid_mask3d.cpp:22-36).
std::optional<std::size_t> cells3d(std::size_t nx, std::size_t ny, std::size_t nz) {
    std::size_t plane = 0, cells = 0;
    if (nx == 0 || ny == 0 || nz == 0 || !mul(nx, ny, plane) || !mul(plane, nz, cells) ||
        cells > kMaxGridCells) {
        return std::nullopt;
    }
    return cells;
}

bool binary32_storage(int32_t storage) {
    return storage != ORR_STORAGE_F64;
}

// The kernels see every real parameter rounded to binary32
// (check_binary32, lbm3d_gpu.cpp:91-127).
float to_float32(double v) {
    if (std::abs(v) > static_cast<double>(std::numeric_limits<float>::max())) {
        return v > 0.0 ? std::numeric_limits<float>::infinity()
                       : -std::numeric_limits<float>::infinity();
    }
    return static_cast<float>(v);
}

struct Param {
    const char* name;
    double value;
};

std::string binary32_problem(const char* family, const Param* params, std::size_t n, double tau) {
    for (std::size_t k = 0; k < n; ++k) {
        if (!std::isfinite(to_float32(params[k].value))) {
            std::ostringstream m;
            m << family << " gpu: " << params[k].name << " " << params[k].value
              << " is outside the binary32 range of the kernels";
            return m.str();
        }
    }
    if (!(static_cast<double>(to_float32(tau)) > 0.5)) {
        std::ostringstream m;
        m << std::setprecision(17) << family << " gpu: tau " << tau
          << " rounds to 1/2 in binary32 (zero viscosity in the kernels); tau - 1/2 must "
             "exceed 2^-25 (about 3e-8)";
        return m.str();
    }
    return {};
}

} // namespace

std::size_t storage_bytes(int32_t storage) {
    switch (storage) {
        case ORR_STORAGE_F16:
        case ORR_STORAGE_BF16:
            return 2;
        case ORR_STORAGE_F64:
            return 8;
        default:
            return 4;
    }
}

std::size_t arithmetic_bytes(int32_t storage) {
    return storage == ORR_STORAGE_F64 ? 8 : 4;
}

std::string mebibytes(std::size_t bytes) {
    std::ostringstream out;
    out << std::fixed << std::setprecision(1) << static_cast<double>(bytes) / (1024.0 * 1024.0)
        << " MiB";
    return out.str();
}

std::string problem3d(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance,
                      int32_t storage, bool allow_high_mach) {
    if (storage < ORR_STORAGE_F32 || storage > ORR_STORAGE_F64) {
        return "lbm3d gpu: unknown population storage";
    }
    if (c.nx < 3 || c.ny < 3 || c.nz < 3) {
        return "lbm3d: the lattice needs at least 3 nodes along each axis";
    }
    const auto cells = cells3d(c.nx, c.ny, c.nz);
    if (!cells) {
        return "lbm3d: more than geom::max_grid_cells nodes";
    }
    if (solid == nullptr) {
        return "lbm3d: the solid mask does not match the lattice size";
    }
    if (!finite(c.tau) || !(c.tau > 0.5)) {
        return "lbm3d: tau must be finite and above 1/2 (positive viscosity)";
    }
    for (const double v : {c.inlet_ux, c.inlet_uy, c.inlet_uz, c.body_force_x, c.body_force_y,
                           c.body_force_z, c.y_low.velocity_x, c.y_high.velocity_x,
                           c.z_low.velocity_x, c.z_high.velocity_x}) {
        if (!finite(v)) {
            return "lbm3d: velocities and body force must be finite";
        }
    }
    if (c.smagorinsky_enabled &&
        (!finite(c.smagorinsky_constant) || c.smagorinsky_constant < 0.0)) {
        return "lbm3d: the Smagorinsky constant must be finite and non-negative";
    }
    for (const orr_wall* w : {&c.y_low, &c.y_high, &c.z_low, &c.z_high}) {
        if (w->kind < ORR_WALL_PERIODIC || w->kind > ORR_WALL_NO_SLIP) {
            return "lbm3d: unknown wall kind";
        }
    }
    if ((c.y_low.kind == ORR_WALL_PERIODIC) != (c.y_high.kind == ORR_WALL_PERIODIC) ||
        (c.z_low.kind == ORR_WALL_PERIODIC) != (c.z_high.kind == ORR_WALL_PERIODIC)) {
        return "lbm3d: an axis is periodic on both sides or on neither";
    }
    if (!allow_high_mach) {
        const struct {
            const char* name;
            double speed;
        } sides[] = {{"y = 0 wall speed", c.y_low.velocity_x},
                     {"y = ny - 1 wall speed", c.y_high.velocity_x},
                     {"z = 0 wall speed", c.z_low.velocity_x},
                     {"z = nz - 1 wall speed", c.z_high.velocity_x}};
        for (const auto& s : sides) {
            if (std::string bad = check_mach("lbm3d", s.name, s.speed); !bad.empty()) {
                return bad;
            }
        }
    }
    if (!finite(c.sponge_strength) || c.sponge_strength < 0.0 || c.sponge_strength > 1.0) {
        return "lbm3d: the absorbing-layer strength must be in [0, 1]";
    }
    if (c.sponge_strength > 0.0 &&
        (c.x_boundary != ORR_X_INFLOW_OUTFLOW || c.sponge_inlet > c.nx || c.sponge_outlet > c.nx ||
         c.sponge_sides > std::min(c.ny, c.nz))) {
        return "lbm3d: absorbing layers need the inflow/outflow x boundary and must fit in the "
               "lattice";
    }
    if (c.solid_wall == ORR_SOLID_INTERPOLATED) {
        if (distance == nullptr) {
            return "lbm3d: the interpolated wall needs the mask's signed distance";
        }
        if (any_nan(distance, *cells)) {
            return "lbm3d: the mask's signed distance must not be NaN";
        }
    } else if (c.solid_wall != ORR_SOLID_HALFWAY) {
        return "lbm3d: unknown solid wall treatment";
    }
    if (c.x_boundary == ORR_X_INFLOW_OUTFLOW) {
        if (!allow_high_mach) {
            const double speed = std::sqrt(c.inlet_ux * c.inlet_ux + c.inlet_uy * c.inlet_uy +
                                           c.inlet_uz * c.inlet_uz);
            if (std::string bad = check_mach("lbm3d", "inlet speed", speed); !bad.empty()) {
                return bad;
            }
        }
        for (std::size_t z = 0; z < c.nz; ++z) {
            for (std::size_t y = 0; y < c.ny; ++y) {
                const std::size_t row = c.nx * (y + c.ny * z);
                if (solid[row] != 0 || solid[row + c.nx - 1] != 0) {
                    return "lbm3d: the inlet and outlet faces must be fluid";
                }
            }
        }
        if (c.outlet == ORR_OUTLET_CONVECTIVE && !(c.inlet_ux > 0.0)) {
            return "lbm3d: the convective outlet needs a positive inlet speed";
        }
    } else if (c.x_boundary != ORR_X_PERIODIC) {
        return "lbm3d: unknown x boundary";
    }
    // make_gpu_solver's bound on the kernels' 32-bit indices (lbm3d_gpu.cpp:492-497).
    if (*cells > std::numeric_limits<uint32_t>::max() / static_cast<std::size_t>(d3::Q)) {
        return "lbm3d gpu: lattice too large for 32-bit indices";
    }
    if (binary32_storage(storage)) {
        const double k = c.smagorinsky_enabled ? c.smagorinsky_constant : 0.0;
        const Param params[] = {{"tau", c.tau},
                                {"y = 0 wall speed", c.y_low.velocity_x},
                                {"y = ny - 1 wall speed", c.y_high.velocity_x},
                                {"z = 0 wall speed", c.z_low.velocity_x},
                                {"z = nz - 1 wall speed", c.z_high.velocity_x},
                                {"inlet x velocity", c.inlet_ux},
                                {"inlet y velocity", c.inlet_uy},
                                {"inlet z velocity", c.inlet_uz},
                                {"squared Smagorinsky constant", k * k},
                                {"body force x", c.body_force_x},
                                {"body force y", c.body_force_y},
                                {"body force z", c.body_force_z}};
        if (std::string bad =
                binary32_problem("lbm3d", params, sizeof(params) / sizeof(params[0]), c.tau);
            !bad.empty()) {
            return bad;
        }
    }
    return {};
}

std::string inlet_problem3d(const orr_lbm3d_config& c, const double v[3], bool allow_high_mach) {
    if (c.x_boundary != ORR_X_INFLOW_OUTFLOW) {
        return "lbm3d: a periodic lattice has no inlet";
    }
    if (!finite(v[0]) || !finite(v[1]) || !finite(v[2])) {
        return "lbm3d: the inlet velocity must be finite";
    }
    if (allow_high_mach) {
        return {};
    }
    return check_mach("lbm3d", "inlet speed", std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
}

namespace {

// Where population i of node (x, y, z) comes from, reduced to what planning
// needs: whether the source is a solid node inside the domain after the side
// rules (resolve_source, lbm3d_internal.h:87-130).
bool bounces3d(const orr_lbm3d_config& c, const uint8_t* solid, long x, long y, long z, int i) {
    const long nx = static_cast<long>(c.nx), ny = static_cast<long>(c.ny),
               nz = static_cast<long>(c.nz);
    long sx = x - d3::cx(i), sy = y - d3::cy(i), sz = z - d3::cz(i);
    const auto side = [](const orr_wall& lo, const orr_wall& hi, long& s, long n, long own) {
        if (s >= 0 && s < n) {
            return false;
        }
        const orr_wall& w = s < 0 ? lo : hi;
        if (w.kind == ORR_WALL_PERIODIC) {
            s = (s + n) % n;
            return false;
        }
        if (w.kind == ORR_WALL_SLIP) {
            s = own;
            return false;
        }
        return true; // no-slip domain wall: not a solid-node link
    };
    if (side(c.y_low, c.y_high, sy, ny, y) || side(c.z_low, c.z_high, sz, nz, z)) {
        return false;
    }
    if (sx < 0 || sx >= nx) {
        if (c.x_boundary != ORR_X_PERIODIC) {
            return false; // inlet or outlet
        }
        sx = (sx + nx) % nx;
    }
    return solid[static_cast<std::size_t>(sx + nx * (sy + ny * sz))] != 0;
}

// link_fraction (lbm3d_internal.h:132-179).
double link_fraction3d(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance,
                       long x, long y, long z, int i) {
    if (c.solid_wall != ORR_SOLID_INTERPOLATED || distance == nullptr) {
        return 0.5;
    }
    const long nx = static_cast<long>(c.nx), ny = static_cast<long>(c.ny),
               nz = static_cast<long>(c.nz);
    const auto inside = [&](long a, long b, long d) {
        return a >= 0 && b >= 0 && d >= 0 && a < nx && b < ny && d < nz;
    };
    const auto at = [&](long a, long b, long d) {
        return static_cast<std::size_t>(a + nx * (b + ny * d));
    };
    const long sx = x - d3::cx(i), sy = y - d3::cy(i), sz = z - d3::cz(i);
    if (!inside(sx, sy, sz)) {
        return 0.5;
    }
    const double df = distance[at(x, y, z)];
    const double ds = distance[at(sx, sy, sz)];
    if (!std::isfinite(df) || !std::isfinite(ds) || df < 0.0 || ds > 0.0 ||
        (df == 0.0 && ds == 0.0)) {
        return 0.5;
    }
    const double span = df - ds;
    const double ratio = std::isfinite(span) ? df / span : 0.5 * df / (0.5 * df - 0.5 * ds);
    const double q = std::min(ratio, 1.0);
    if (q < 0.5) {
        const long fx = x + d3::cx(i), fy = y + d3::cy(i), fz = z + d3::cz(i);
        if (!inside(fx, fy, fz) || solid[at(fx, fy, fz)] != 0) {
            return 0.5;
        }
    }
    return q;
}

} // namespace

Plan3D plan3d(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance) {
    Plan3D p;
    p.c = c;
    const long nx = static_cast<long>(c.nx), ny = static_cast<long>(c.ny),
               nz = static_cast<long>(c.nz);
    p.cells = static_cast<std::size_t>(nx * ny * nz);
    p.cls.resize(p.cells);              // filled slab by slab below
    const long plane = nx * ny;
    long off[d3::Q];
    for (int i = 0; i < d3::Q; ++i) {
        off[i] = -d3::cx(i) - nx * d3::cy(i) - plane * d3::cz(i);
    }
    // Classes for the step kernel's lanes (the result does not depend on
    // them): nodes with a solid source after the side rules are boundary
    // nodes (bounce-back mask per node); the other nodes of interior rows are
    // bulk (x-edges included) and those of the y and z face rows take the
    // face path.  Links are collected in scan order (cell, then direction),
    // the order of boundary_links.
    const bool interpolated = c.solid_wall == ORR_SOLID_INTERPOLATED;
    p.nmask.resize(p.cells);
    if (interpolated) {
        p.nslot.resize(p.cells);
    }
    // Large lattices are planned in z-slabs on several host threads; each slab
    // keeps its links and wall slots in scan order and the slabs are joined in
    // z order, which is the scan order of the whole lattice.
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const long workers = p.cells >= (std::size_t{1} << 20) ? std::min<long>({static_cast<long>(hw), 32L, nz}) : 1L;
    // Rows (y, z) holding a solid node.  A row whose source rows hold none
    // (`quiet` below) is classified whole: bulk from end to end inside, face
    // nodes on a y or z face, no link; the others node by node, in scan order.
    std::vector<uint8_t> row_solid(static_cast<std::size_t>(ny * nz), 0);
    const auto scan_rows = [&](long r0, long r1) {
        for (long r = r0; r < r1; ++r) {
            const uint8_t* row = solid + r * nx;
            row_solid[static_cast<std::size_t>(r)] =
                std::any_of(row, row + nx, [](uint8_t s) { return s != 0; }) ? 1 : 0;
        }
    };
    // The row a source index s of an axis of n rows reads after the side
    // rules of bounces3d (periodic wrap, free-slip mirror onto the node's
    // own row `own`), or -1 across a no-slip domain wall, which makes no link.
    const auto source_row = [](long s, long n, const orr_wall& lo, const orr_wall& hi, long own) -> long {
        if (s >= 0 && s < n) {
            return s;
        }
        const orr_wall& w = s < 0 ? lo : hi;
        if (w.kind == ORR_WALL_PERIODIC) {
            return (s + n) % n;
        }
        return w.kind == ORR_WALL_SLIP ? own : -1;
    };
    // A row none of whose source rows (y - c_y, z - c_z after the side rules;
    // x sources stay in those rows or leave through the inlet or outlet)
    // holds a solid node has no solid node and no link.
    const auto quiet = [&](long y, long z) {
        for (long dz = -1; dz <= 1; ++dz) {
            const long sz = source_row(z + dz, nz, c.z_low, c.z_high, z);
            if (sz < 0) {
                continue;
            }
            for (long dy = -1; dy <= 1; ++dy) {
                const long sy = source_row(y + dy, ny, c.y_low, c.y_high, y);
                if (sy >= 0 && row_solid[static_cast<std::size_t>(sy + ny * sz)] != 0) {
                    return false;
                }
            }
        }
        return true;
    };
    struct Slab {
        std::size_t fluid = 0, general = 0;
        std::vector<uint32_t> link_cell, link_dir;
        std::vector<double> link_q;
        std::vector<double> wall_q;        // 19 per local slot
        std::vector<std::size_t> slotted;  // cells given a local slot
    };
    const auto classify = [&](long z0, long z1, Slab& s) {
        const std::size_t c0 = static_cast<std::size_t>(plane * z0), c1 = static_cast<std::size_t>(plane * z1);
        std::fill(p.cls.begin() + c0, p.cls.begin() + c1, kBulk);
        std::fill(p.nmask.begin() + c0, p.nmask.begin() + c1, 0u);
        if (interpolated) {
            std::fill(p.nslot.begin() + c0, p.nslot.begin() + c1, -1);
        }
        for (long z = z0; z < z1; ++z) {
            for (long y = 0; y < ny; ++y) {
                if (quiet(y, z)) {
                    // Interior rows stay bulk from end to end; every node of a
                    // face row takes the face path.
                    s.fluid += static_cast<std::size_t>(nx);
                    if (y == 0 || z == 0 || y + 1 == ny || z + 1 == nz) {
                        const std::size_t r = static_cast<std::size_t>(nx * (y + ny * z));
                        std::fill(p.cls.begin() + r, p.cls.begin() + r + nx, kFace);
                        s.general += static_cast<std::size_t>(nx);
                    }
                    continue;
                }
                for (long x = 0; x < nx; ++x) {
                    const std::size_t h = static_cast<std::size_t>(x + nx * (y + ny * z));
                    if (solid[h] != 0) {
                        p.cls[h] = kSolid;
                        continue;
                    }
                    ++s.fluid;
                    const bool face_row = y == 0 || z == 0 || y + 1 == ny || z + 1 == nz;
                    const bool x_edge = x == 0 || x + 1 == nx;
                    if (!face_row && !x_edge) {
                        bool near = false;
                        for (int i = 1; i < d3::Q && !near; ++i) {
                            near = solid[static_cast<std::size_t>(static_cast<long>(h) + off[i])] != 0;
                        }
                        if (!near) {
                            continue; // kBulk
                        }
                    }
                    int32_t slot = -1;
                    bool linked = false;
                    uint32_t mask = 0;
                    for (int i = 1; i < d3::Q; ++i) {
                        if (!bounces3d(c, solid, x, y, z, i)) {
                            continue;
                        }
                        linked = true;
                        mask |= 1u << i;
                        const double q = link_fraction3d(c, solid, distance, x, y, z, i);
                        s.link_cell.push_back(static_cast<uint32_t>(h));
                        s.link_dir.push_back(static_cast<uint32_t>(i));
                        s.link_q.push_back(q);
                        if (interpolated) {
                            if (slot < 0) {
                                slot = static_cast<int32_t>(s.wall_q.size() / d3::Q);
                                s.wall_q.insert(s.wall_q.end(), d3::Q, 0.5);
                            }
                            s.wall_q[static_cast<std::size_t>(slot) * d3::Q + static_cast<std::size_t>(i)] = q;
                        }
                    }
                    if (!linked) {
                        if (face_row) {
                            p.cls[h] = kFace;
                            ++s.general;
                        }
                        continue; // interior-row x-edge node: bulk
                    }
                    p.cls[h] = kBoundary;
                    ++s.general;
                    p.nmask[h] = mask;
                    if (interpolated) {
                        p.nslot[h] = slot;
                        s.slotted.push_back(h);
                    }
                }
            }
        }
    };
    std::vector<Slab> slabs(static_cast<std::size_t>(workers));
    const auto slab_z = [&](long w) { return nz * w / workers; };
    if (workers == 1) {
        scan_rows(0, ny * nz);
        classify(0, nz, slabs[0]);
    } else {
        std::vector<std::thread> pool;
        for (long w = 0; w < workers; ++w) {
            pool.emplace_back([&, w] { scan_rows(ny * slab_z(w), ny * slab_z(w + 1)); });
        }
        for (std::thread& t : pool) t.join();
        pool.clear();
        for (long w = 0; w < workers; ++w) {
            pool.emplace_back([&, w] { classify(slab_z(w), slab_z(w + 1), slabs[static_cast<std::size_t>(w)]); });
        }
        for (std::thread& t : pool) t.join();
    }
    for (Slab& s : slabs) {
        const int32_t first_slot = static_cast<int32_t>(p.wall_q.size() / d3::Q);
        for (const std::size_t h : s.slotted) {
            p.nslot[h] += first_slot;
        }
        p.fluid += s.fluid;
        p.general += s.general;
        p.link_cell.insert(p.link_cell.end(), s.link_cell.begin(), s.link_cell.end());
        p.link_dir.insert(p.link_dir.end(), s.link_dir.begin(), s.link_dir.end());
        p.link_q.insert(p.link_q.end(), s.link_q.begin(), s.link_q.end());
        p.wall_q.insert(p.wall_q.end(), s.wall_q.begin(), s.wall_q.end());
    }
    return p;
}

std::optional<std::size_t> memory3d(const orr_lbm3d_config& c, std::size_t links,
                                    std::size_t wall_slots, int32_t storage) {
    const auto cells = cells3d(c.nx, c.ny, c.nz);
    if (!cells) {
        return std::nullopt;
    }
    const std::size_t s = storage_bytes(storage), a = arithmetic_bytes(storage);
    std::size_t total = 0, t = 0;
    // Two population buffers.
    if (!mul(*cells, d3::Q * s * 2, t) || !add(total, t, total)) return std::nullopt;
    // Node classes (one byte), bounce-back masks, wall slots and four moment planes.
    const std::size_t slot_bytes = c.solid_wall == ORR_SOLID_INTERPOLATED ? 4 : 0;
    if (!mul(*cells, 1 + 4 + slot_bytes + 4 * a, t) || !add(total, t, total)) return std::nullopt;
    // Outlet history.
    std::size_t face = 0;
    if (!mul(c.ny, c.nz, face) || !mul(face, d3::kOutletSlots * a, t) || !add(total, t, total))
        return std::nullopt;
    // Wall fractions.
    if (!mul(std::max<std::size_t>(wall_slots, 1), d3::Q * a, t) || !add(total, t, total))
        return std::nullopt;
    // Links: cell, direction, fraction.
    if (!mul(links, 16, t) || !add(total, t, total)) return std::nullopt;
    // Force, mass and inlet buffers; slack of the staged step; table entry.
    if (!add(total, 256 + 4 * kPopPad * s + kClassPad + kTableBytes, total)) return std::nullopt;
    return total;
}

// ---- D2Q9 ----

std::string problem2d(const orr_lbm2d_config& c, const uint8_t* solid, int32_t storage,
                      bool allow_high_mach) {
    if (storage < ORR_STORAGE_F32 || storage > ORR_STORAGE_F64) {
        return "lbm2d gpu: unknown population storage";
    }
    if (c.nx < 3 || c.ny < 3) {
        return "lbm2d: the lattice needs at least 3 x 3 nodes";
    }
    if (c.nx > kMaxGridCells / c.ny) {
        return "lbm2d: more than geom::max_grid_cells nodes";
    }
    if (solid == nullptr) {
        return "lbm2d: the solid mask does not match the lattice size";
    }
    if (!finite(c.tau) || !(c.tau > 0.5)) {
        return "lbm2d: tau must be finite and above 1/2 (positive viscosity)";
    }
    if (!finite(c.inlet_ux) || !finite(c.inlet_uy) || !finite(c.body_force_x) ||
        !finite(c.body_force_y) || !finite(c.bottom.velocity_x) || !finite(c.top.velocity_x)) {
        return "lbm2d: velocities and body force must be finite";
    }
    if (c.smagorinsky_enabled &&
        (!finite(c.smagorinsky_constant) || c.smagorinsky_constant < 0.0)) {
        return "lbm2d: the Smagorinsky constant must be finite and non-negative";
    }
    for (const orr_wall* w : {&c.bottom, &c.top}) {
        if (w->kind < ORR_WALL_PERIODIC || w->kind > ORR_WALL_NO_SLIP) {
            return "lbm2d: unknown wall kind";
        }
    }
    if ((c.bottom.kind == ORR_WALL_PERIODIC) != (c.top.kind == ORR_WALL_PERIODIC)) {
        return "lbm2d: y is periodic on both sides or on neither";
    }
    if (!allow_high_mach) {
        if (std::string bad = check_mach("lbm2d", "bottom wall speed", c.bottom.velocity_x);
            !bad.empty()) {
            return bad;
        }
        if (std::string bad = check_mach("lbm2d", "top wall speed", c.top.velocity_x);
            !bad.empty()) {
            return bad;
        }
    }
    if (c.x_boundary == ORR_X_INFLOW_OUTFLOW) {
        if (!allow_high_mach) {
            if (std::string bad =
                    check_mach("lbm2d", "inlet speed", std::hypot(c.inlet_ux, c.inlet_uy));
                !bad.empty()) {
                return bad;
            }
        }
        for (std::size_t y = 0; y < c.ny; ++y) {
            if (solid[c.nx * y] != 0 || solid[c.nx - 1 + c.nx * y] != 0) {
                return "lbm2d: the inlet and outlet columns must be fluid";
            }
        }
        if (c.outlet == ORR_OUTLET_CONVECTIVE && !(c.inlet_ux > 0.0)) {
            return "lbm2d: the convective outlet needs a positive inlet speed";
        }
    } else if (c.x_boundary != ORR_X_PERIODIC) {
        return "lbm2d: unknown x boundary";
    }
    if (binary32_storage(storage)) {
        const double k = c.smagorinsky_enabled ? c.smagorinsky_constant : 0.0;
        const Param params[] = {{"tau", c.tau},
                                {"bottom wall speed", c.bottom.velocity_x},
                                {"top wall speed", c.top.velocity_x},
                                {"inlet x velocity", c.inlet_ux},
                                {"inlet y velocity", c.inlet_uy},
                                {"squared Smagorinsky constant", k * k},
                                {"body force x", c.body_force_x},
                                {"body force y", c.body_force_y}};
        if (std::string bad =
                binary32_problem("lbm2d", params, sizeof(params) / sizeof(params[0]), c.tau);
            !bad.empty()) {
            return bad;
        }
    }
    return {};
}

Plan2D plan2d(const orr_lbm2d_config& c, const uint8_t* solid) {
    Plan2D p;
    p.c = c;
    const long nx = static_cast<long>(c.nx), ny = static_cast<long>(c.ny);
    p.cells = static_cast<std::size_t>(nx * ny);
    p.cls.assign(p.cells, kBulk);
    long off[d2::Q];
    for (int i = 0; i < d2::Q; ++i) {
        off[i] = -d2::cx(i) - nx * d2::cy(i);
    }
    p.nmask.assign(p.cells, 0u);
    // Classes as in plan3d: nodes with a solid source are boundary nodes,
    // other interior-row nodes bulk, other bottom/top-row nodes face nodes;
    // links (boundary_links, lbm2d_common.cpp:79-97) in scan order.
    for (long y = 0; y < ny; ++y) {
        for (long x = 0; x < nx; ++x) {
            const std::size_t h = static_cast<std::size_t>(x + nx * y);
            if (solid[h] != 0) {
                p.cls[h] = kSolid;
                continue;
            }
            ++p.fluid;
            const bool face_row = y == 0 || y + 1 == ny;
            const bool x_edge = x == 0 || x + 1 == nx;
            if (!face_row && !x_edge) {
                bool near = false;
                for (int i = 1; i < d2::Q && !near; ++i) {
                    near = solid[static_cast<std::size_t>(static_cast<long>(h) + off[i])] != 0;
                }
                if (!near) {
                    continue; // kBulk
                }
            }
            uint32_t mask = 0;
            for (int i = 1; i < d2::Q; ++i) {
                long sx = x - d2::cx(i), sy = y - d2::cy(i);
                if (sy < 0 || sy >= ny) {
                    const orr_wall& w = sy < 0 ? c.bottom : c.top;
                    if (w.kind == ORR_WALL_NO_SLIP) {
                        continue;
                    }
                    sy = w.kind == ORR_WALL_PERIODIC ? (sy + ny) % ny : y;
                }
                if (sx < 0 || sx >= nx) {
                    if (c.x_boundary != ORR_X_PERIODIC) {
                        continue;
                    }
                    sx = (sx + nx) % nx;
                }
                if (solid[static_cast<std::size_t>(sx + nx * sy)] != 0) {
                    mask |= 1u << i;
                    p.link_cell.push_back(static_cast<uint32_t>(h));
                    p.link_dir.push_back(static_cast<uint32_t>(i));
                }
            }
            if (mask != 0u) {
                p.cls[h] = kBoundary;
                p.nmask[h] = mask;
                ++p.general;
            } else if (face_row) {
                p.cls[h] = kFace;
                ++p.general;
            }
        }
    }
    return p;
}

std::optional<std::size_t> memory2d(const orr_lbm2d_config& c, std::size_t links,
                                    int32_t storage) {
    if (c.nx == 0 || c.ny == 0 || c.nx > kMaxGridCells / c.ny) {
        return std::nullopt;
    }
    const std::size_t cells = c.nx * c.ny;
    const std::size_t s = storage_bytes(storage), a = arithmetic_bytes(storage);
    return cells * (d2::Q * s * 2 + 1 + 3 * a) + c.ny * d2::kOutletSlots * a +
           cells * 4 + links * 8 + 256;
}

} // namespace orr
