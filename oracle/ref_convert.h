// Conversions between the C ABI's records and the reference's types, shared
// by the oracle's C entry points.  TEST INFRASTRUCTURE ONLY.
#pragma once

#include <cstdint>
#include <cstring>
#include <string>

#include "orrery/aero/lbm/lbm2d.h"
#include "orrery/aero/lbm3d/lbm3d.h"
#include "orrery/aero/lbm3d/solid_mask3d.h"
#include "orrery_lbm.h"

namespace ref_convert {

namespace lbm = orrery::aero::lbm;

inline void copy_message(const std::string& text, char* message, size_t capacity) {
    if (message == nullptr || capacity == 0) {
        return;
    }
    const size_t n = text.size() < capacity - 1 ? text.size() : capacity - 1;
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

inline lbm::Wall wall_of(const orr_wall& w) {
    lbm::Wall out;
    out.kind = static_cast<lbm::WallKind>(w.kind);
    out.velocity_x = w.velocity_x;
    return out;
}

inline lbm::Lbm3DConfig config3d_of(const orr_lbm3d_config& c) {
    lbm::Lbm3DConfig out;
    out.nx = c.nx;
    out.ny = c.ny;
    out.nz = c.nz;
    out.tau = c.tau;
    out.x_boundary = static_cast<lbm::XBoundary>(c.x_boundary);
    out.outlet = static_cast<lbm::Outlet>(c.outlet);
    out.y_low = wall_of(c.y_low);
    out.y_high = wall_of(c.y_high);
    out.z_low = wall_of(c.z_low);
    out.z_high = wall_of(c.z_high);
    out.inlet_ux = c.inlet_ux;
    out.inlet_uy = c.inlet_uy;
    out.inlet_uz = c.inlet_uz;
    out.body_force_x = c.body_force_x;
    out.body_force_y = c.body_force_y;
    out.body_force_z = c.body_force_z;
    out.smagorinsky.enabled = c.smagorinsky_enabled != 0;
    out.smagorinsky.constant = c.smagorinsky_constant;
    out.sponge.strength = c.sponge_strength;
    out.sponge.inlet = c.sponge_inlet;
    out.sponge.outlet = c.sponge_outlet;
    out.sponge.sides = c.sponge_sides;
    out.solid_wall = static_cast<lbm::SolidWall>(c.solid_wall);
    return out;
}

inline lbm::Lbm2DConfig config2d_of(const orr_lbm2d_config& c) {
    lbm::Lbm2DConfig out;
    out.nx = c.nx;
    out.ny = c.ny;
    out.tau = c.tau;
    out.x_boundary = static_cast<lbm::XBoundary>(c.x_boundary);
    out.outlet = static_cast<lbm::Outlet>(c.outlet);
    out.bottom = wall_of(c.bottom);
    out.top = wall_of(c.top);
    out.inlet_ux = c.inlet_ux;
    out.inlet_uy = c.inlet_uy;
    out.body_force_x = c.body_force_x;
    out.body_force_y = c.body_force_y;
    out.smagorinsky.enabled = c.smagorinsky_enabled != 0;
    out.smagorinsky.constant = c.smagorinsky_constant;
    return out;
}

inline lbm::SolidMask3D mask3d_of(const orr_lbm3d_config& c, const uint8_t* solid, const double* distance) {
    lbm::SolidMask3D mask;
    mask.nx = c.nx;
    mask.ny = c.ny;
    mask.nz = c.nz;
    const size_t cells = c.nx * c.ny * c.nz;
    mask.solid.assign(solid, solid + cells);
    if (distance != nullptr) {
        mask.distance.assign(distance, distance + cells);
    }
    return mask;
}

} // namespace ref_convert
