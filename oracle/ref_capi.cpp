// C entry points over Orrery's own double-precision CPU LBM solvers
// (src/aero/lbm3d/lbm3d_cpu.cpp, src/aero/lbm/lbm2d_cpu.cpp), compiled from
// the reference sources in place by oracle/Makefile into oracle/_ref.
//
// TEST INFRASTRUCTURE ONLY.  This is the reference oracle: the checker that
// the restatement in oracle/lbm_oracle.c and the CUDA path are compared with,
// and the CPU baseline of the benchmark.  The product never links or loads it.
#include <array>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "orrery/aero/lbm/lbm2d.h"
#include "orrery/aero/lbm/solid_mask.h"
#include "orrery/aero/lbm3d/lbm3d.h"
#include "orrery/aero/lbm3d/solid_mask3d.h"
#include "tbb/parallel_for.h"

#include "orrery_lbm.h"
#include "ref_convert.h"

namespace lbm = orrery::aero::lbm;

namespace {

using ref_convert::config2d_of;
using ref_convert::config3d_of;
using ref_convert::copy_message;
using ref_convert::mask3d_of;
using ref_convert::wall_of;

struct Ref3D {
    std::unique_ptr<lbm::Lbm3DSolver> solver;
    size_t cells = 0;
};

struct Ref2D {
    std::unique_ptr<lbm::Lbm2DSolver> solver;
    size_t cells = 0;
};

} // namespace

extern "C" {

void ref_set_threads(int threads) {
    tbb_shim::Pool::instance().set_threads(threads);
}

int ref_threads(void) {
    return tbb_shim::Pool::instance().threads();
}

int ref3d_validate(const orr_lbm3d_config* config, const uint8_t* solid, const double* distance,
                   char* message, size_t capacity) {
    const auto problem = lbm::validate(config3d_of(*config), mask3d_of(*config, solid, distance));
    copy_message(problem ? *problem : std::string(), message, capacity);
    return problem ? 1 : 0;
}

void* ref3d_create(const orr_lbm3d_config* config, const uint8_t* solid, const double* distance,
                   char* message, size_t capacity) {
    auto made = lbm::make_cpu_solver(config3d_of(*config), mask3d_of(*config, solid, distance));
    if (!made) {
        copy_message(made.error(), message, capacity);
        return nullptr;
    }
    auto* ref = new Ref3D;
    ref->solver = std::move(made).value();
    ref->cells = config->nx * config->ny * config->nz;
    copy_message(std::string(), message, capacity);
    return ref;
}

void ref3d_destroy(void* handle) {
    delete static_cast<Ref3D*>(handle);
}

int ref3d_initialize(void* handle, const double* rho, const double* ux, const double* uy,
                     const double* uz) {
    auto* ref = static_cast<Ref3D*>(handle);
    const lbm::Lbm3DConfig& config = ref->solver->config();
    if (rho == nullptr) {
        return ref->solver->initialize(lbm::uniform_inlet_state(config)) ? 0 : 1;
    }
    const size_t nx = config.nx;
    const size_t ny = config.ny;
    const auto state = [=](size_t x, size_t y, size_t z) {
        const size_t c = x + nx * (y + ny * z);
        return lbm::d3q19::Moments{rho[c], ux[c], uy[c], uz[c]};
    };
    return ref->solver->initialize(state) ? 0 : 1;
}

int ref3d_step(void* handle, uint64_t count) {
    return static_cast<Ref3D*>(handle)->solver->step(count) ? 0 : 1;
}

int ref3d_set_inlet(void* handle, const double* velocity, char* message, size_t capacity) {
    auto done = static_cast<Ref3D*>(handle)->solver->set_inlet_velocity(
        {velocity[0], velocity[1], velocity[2]});
    copy_message(done ? std::string() : done.error(), message, capacity);
    return done ? 0 : 1;
}

int ref3d_populations(void* handle, double* out) {
    auto* ref = static_cast<Ref3D*>(handle);
    auto f = ref->solver->populations();
    if (!f) {
        return 1;
    }
    std::memcpy(out, f.value().data(), f.value().size() * sizeof(double));
    return 0;
}

int ref3d_force(void* handle, double* out) {
    auto f = static_cast<Ref3D*>(handle)->solver->force();
    if (!f) {
        return 1;
    }
    for (int a = 0; a < 3; ++a) {
        out[a] = f.value().force[a];
        out[3 + a] = f.value().moment[a];
    }
    return 0;
}

int ref3d_macroscopic(void* handle, double* rho, double* ux, double* uy, double* uz) {
    auto* ref = static_cast<Ref3D*>(handle);
    auto m = ref->solver->macroscopic();
    if (!m) {
        return 1;
    }
    const size_t bytes = ref->cells * sizeof(double);
    std::memcpy(rho, m.value().density.data(), bytes);
    std::memcpy(ux, m.value().velocity_x.data(), bytes);
    std::memcpy(uy, m.value().velocity_y.data(), bytes);
    std::memcpy(uz, m.value().velocity_z.data(), bytes);
    return 0;
}

int ref3d_mass(void* handle, double* out) {
    auto m = static_cast<Ref3D*>(handle)->solver->mass();
    if (!m) {
        return 1;
    }
    *out = m.value();
    return 0;
}

uint64_t ref3d_link_count(void* handle) {
    return static_cast<Ref3D*>(handle)->solver->links().size();
}

void ref3d_links(void* handle, uint32_t* cell, uint32_t* direction, double* q) {
    const auto& links = static_cast<Ref3D*>(handle)->solver->links();
    for (size_t k = 0; k < links.size(); ++k) {
        cell[k] = links[k].cell;
        direction[k] = links[k].direction;
        q[k] = links[k].q;
    }
}

uint64_t ref3d_steps(void* handle) {
    return static_cast<Ref3D*>(handle)->solver->steps();
}

// sphere_mask (src/aero/lbm3d/solid_mask3d.cpp:77-85): solid flags and the
// signed distance, for checking the package's own mask generators.
void ref3d_sphere_mask(uint64_t nx, uint64_t ny, uint64_t nz, const double* centre, double radius,
                       uint8_t* solid, double* distance) {
    const lbm::SolidMask3D mask =
        lbm::sphere_mask(nx, ny, nz, {centre[0], centre[1], centre[2]}, radius);
    std::memcpy(solid, mask.solid.data(), mask.solid.size());
    std::memcpy(distance, mask.distance.data(), mask.distance.size() * sizeof(double));
}

// box_mask (src/aero/lbm3d/solid_mask3d.cpp:87-102).
void ref3d_box_mask(uint64_t nx, uint64_t ny, uint64_t nz, const double* lo, const double* hi,
                    uint8_t* solid, double* distance) {
    const lbm::SolidMask3D mask =
        lbm::box_mask(nx, ny, nz, {lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]});
    std::memcpy(solid, mask.solid.data(), mask.solid.size());
    std::memcpy(distance, mask.distance.data(), mask.distance.size() * sizeof(double));
}

// gpu_memory_bytes / cpu_memory_bytes (src/aero/lbm3d/lbm3d_common.cpp:272-307).
int ref3d_memory(const orr_lbm3d_config* config, uint64_t links, uint64_t wall_slots,
                 uint64_t* gpu_base, uint64_t* gpu_total, uint64_t* cpu) {
    const lbm::Lbm3DConfig c = config3d_of(*config);
    const auto base = lbm::gpu_memory_bytes(c);
    const auto total = lbm::gpu_memory_bytes(c, links, wall_slots);
    const auto host = lbm::cpu_memory_bytes(c);
    if (!base || !total || !host) {
        return 1;
    }
    *gpu_base = *base;
    *gpu_total = *total;
    *cpu = *host;
    return 0;
}

// ---- D2Q9 ----

int ref2d_validate(const orr_lbm2d_config* config, const uint8_t* solid, char* message,
                   size_t capacity) {
    lbm::SolidMask2D mask;
    mask.nx = config->nx;
    mask.ny = config->ny;
    mask.solid.assign(solid, solid + config->nx * config->ny);
    const auto problem = lbm::validate(config2d_of(*config), mask);
    copy_message(problem ? *problem : std::string(), message, capacity);
    return problem ? 1 : 0;
}

void* ref2d_create(const orr_lbm2d_config* config, const uint8_t* solid, char* message,
                   size_t capacity) {
    lbm::SolidMask2D mask;
    mask.nx = config->nx;
    mask.ny = config->ny;
    mask.solid.assign(solid, solid + config->nx * config->ny);
    auto made = lbm::make_cpu_solver(config2d_of(*config), std::move(mask));
    if (!made) {
        copy_message(made.error(), message, capacity);
        return nullptr;
    }
    auto* ref = new Ref2D;
    ref->solver = std::move(made).value();
    ref->cells = config->nx * config->ny;
    copy_message(std::string(), message, capacity);
    return ref;
}

void ref2d_destroy(void* handle) {
    delete static_cast<Ref2D*>(handle);
}

int ref2d_initialize(void* handle, const double* rho, const double* ux, const double* uy) {
    auto* ref = static_cast<Ref2D*>(handle);
    const lbm::Lbm2DConfig& config = ref->solver->config();
    if (rho == nullptr) {
        return ref->solver->initialize(lbm::uniform_inlet_state(config)) ? 0 : 1;
    }
    const size_t nx = config.nx;
    const auto state = [=](size_t x, size_t y) {
        const size_t c = x + nx * y;
        return lbm::d2q9::Moments{rho[c], ux[c], uy[c]};
    };
    return ref->solver->initialize(state) ? 0 : 1;
}

int ref2d_step(void* handle, uint64_t count) {
    return static_cast<Ref2D*>(handle)->solver->step(count) ? 0 : 1;
}

int ref2d_populations(void* handle, double* out) {
    auto f = static_cast<Ref2D*>(handle)->solver->populations();
    if (!f) {
        return 1;
    }
    std::memcpy(out, f.value().data(), f.value().size() * sizeof(double));
    return 0;
}

int ref2d_force(void* handle, double* out) {
    auto f = static_cast<Ref2D*>(handle)->solver->force();
    if (!f) {
        return 1;
    }
    out[0] = f.value().x;
    out[1] = f.value().y;
    out[2] = f.value().moment;
    return 0;
}

int ref2d_macroscopic(void* handle, double* rho, double* ux, double* uy) {
    auto* ref = static_cast<Ref2D*>(handle);
    auto m = ref->solver->macroscopic();
    if (!m) {
        return 1;
    }
    const size_t bytes = ref->cells * sizeof(double);
    std::memcpy(rho, m.value().density.data(), bytes);
    std::memcpy(ux, m.value().velocity_x.data(), bytes);
    std::memcpy(uy, m.value().velocity_y.data(), bytes);
    return 0;
}

int ref2d_mass(void* handle, double* out) {
    auto m = static_cast<Ref2D*>(handle)->solver->mass();
    if (!m) {
        return 1;
    }
    *out = m.value();
    return 0;
}

// circle_mask (src/aero/lbm/solid_mask.cpp:39-43).
void ref2d_circle_mask(uint64_t nx, uint64_t ny, double cx, double cy, double radius,
                       uint8_t* solid) {
    const lbm::SolidMask2D mask = lbm::circle_mask(nx, ny, cx, cy, radius);
    std::memcpy(solid, mask.solid.data(), mask.solid.size());
}

} // extern "C"
