// Host-side planning of a lattice before anything touches the device:
// validation with the reference's refusal rules and messages, node classes,
// the compact boundary-node list the step kernel's general path walks, the
// boundary links of the force, and the interpolated-wall table.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "orrery_lbm.h"

namespace orr {

inline constexpr std::size_t kMaxGridCells = std::size_t{1} << 27; // geom::max_grid_cells

// Slack of the D3Q19 device arrays for the staged step: elements before and
// after each population buffer and bytes after the class array (a staged row
// segment may reach one tile plus its halo past either end; those values are
// never used), and the device bytes of the solver's lattice-table entry.
inline constexpr std::size_t kPopPad = 1024;
inline constexpr std::size_t kClassPad = 1024;
inline constexpr std::size_t kTableBytes = 512;

// Refusal text of validate() for a D3Q19 lattice (empty when accepted):
// problem_of (src/aero/lbm3d/lbm3d_common.cpp:74-155), the 32-bit index
// bound and check_binary32 of make_gpu_solver (lbm3d_gpu.cpp:94-127, 492-500;
// binary32 only for the binary32-arithmetic storages).  `allow_high_mach`
// skips the lattice Mach checks (an explicit opt-in).
std::string problem3d(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance,
                      int32_t storage, bool allow_high_mach);

// check_inlet_velocity (lbm3d_common.cpp:163-174).
std::string inlet_problem3d(const orr_lbm3d_config& c, const double velocity[3],
                            bool allow_high_mach);

// Allocator whose value-less construction leaves the element uninitialised:
// a per-cell table sized with resize() is then written once, by the planner
// threads that own its slabs, instead of being zeroed first on one thread.
template <class T> struct UninitAllocator : std::allocator<T> {
    using value_type = T;
    template <class U> struct rebind {
        using other = UninitAllocator<U>;
    };
    UninitAllocator() = default;
    template <class U> UninitAllocator(const UninitAllocator<U>&) noexcept {}
    template <class U, class... Args> void construct(U* p, Args&&... args) {
        if constexpr (sizeof...(Args) == 0) {
            ::new (static_cast<void*>(p)) U;
        } else {
            ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
        }
    }
};
template <class T> using CellTable = std::vector<T, UninitAllocator<T>>;

struct Plan3D {
    orr_lbm3d_config c{};
    std::size_t cells = 0;
    std::size_t fluid = 0;
    CellTable<uint8_t> cls;             // kSolid / kBulk / kBoundary / kFace per cell
    CellTable<uint32_t> nmask;          // per cell, bit i: direction i bounces back
    CellTable<int32_t> nslot;           // per cell wall slot (interpolated wall only), -1 none
    std::size_t general = 0;            // nodes on the general gather (face + boundary)
    std::vector<double> wall_q;         // 19 fractions per slot
    std::vector<uint32_t> link_cell;    // boundary links, scan order
    std::vector<uint32_t> link_dir;
    std::vector<double> link_q;
};

// Builds the plan of an accepted configuration (classify_nodes,
// boundary_links, link_fraction, wall_table: lbm3d_internal.h:132-310,
// lbm3d_common.cpp:176-198).
Plan3D plan3d(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance);

// Bytes the device solver allocates for a lattice: populations twice (with
// their slack), node classes and bounce-back masks (and wall slots for the
// interpolated wall), moments, outlet history, wall table, links, the
// lattice-table entry and the small reduction buffers.
// Empty on overflow.
std::optional<std::size_t> memory3d(const orr_lbm3d_config& c, std::size_t links,
                                    std::size_t wall_slots, int32_t storage);

// ---- D2Q9 ----

// validate (src/aero/lbm/lbm2d_common.cpp:31-77) plus the binary32 checks of
// the 2D make_gpu_solver (lbm2d.h:205-212).
std::string problem2d(const orr_lbm2d_config& c, const uint8_t* solid, int32_t storage,
                      bool allow_high_mach);

struct Plan2D {
    orr_lbm2d_config c{};
    std::size_t cells = 0;
    std::size_t fluid = 0;
    std::size_t general = 0;            // nodes on the general gather
    std::vector<uint8_t> cls;
    std::vector<uint32_t> nmask;        // per cell, bit i: direction i bounces back
    std::vector<uint32_t> link_cell;
    std::vector<uint32_t> link_dir;
};

Plan2D plan2d(const orr_lbm2d_config& c, const uint8_t* solid);

std::optional<std::size_t> memory2d(const orr_lbm2d_config& c, std::size_t links,
                                    int32_t storage);

std::size_t storage_bytes(int32_t storage);
std::size_t arithmetic_bytes(int32_t storage);
std::string mebibytes(std::size_t bytes);

} // namespace orr
