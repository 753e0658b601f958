// The three D3Q19 kernels of the reference's GPU driver, GpuLbm3D
// (src/aero/lbm3d/lbm3d_gpu.cpp), on CUDA: lbm_d3q19_step, lbm_d3q19_moments
// and lbm_d3q19_force with the driver's buffers, bindings and uniforms
// (lbm3d_gpu.cpp:37-44, 158-189, 333-436), for an IComputeBackend that runs
// them (orrery_b200/adapter/compute_backend_cuda.cpp).
//
// The driver's buffers are binary32: populations shifted by their weights
// (f - w, structure of arrays, the layout of this library's binary32 form),
// node codes (0 solid, 1 bulk, 2 boundary, 3 + wall slot), 19 wall fractions
// per slot, the convective-outlet history (slot * ny * nz + y + ny z, the
// layout of this library's), the moments (rho - 1, ux, uy, uz planes) and the
// links (cell, direction pairs).  The step and moments kernels are this
// library's binary32 ones, run on those buffers; what they need beyond them
// (this library's node classes and bounce-back masks, the wall slots, the
// inlet velocity in device memory) is derived once from the node codes, on
// the host by the planner, when the tables are created.  The force kernel
// writes, per link, the shifted sum f*_o(x) + f_j(x, t+1) the driver adds up
// in binary64 (lbm_d3q19_force.comp.glsl).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "kernels3d.cuh"
#include "lattice.h"
#include "ops3d.h"
#include "plan.h"
#include "trace.h"

using namespace orr;

struct orr_gl3d {
    int device = 0;
    orr_gl3d_params dims{};   // the parameters the tables were built for
    Geom3D g{};
    bool interpolated = false;
    uint8_t* cls = nullptr;
    uint32_t* nmask = nullptr;
    int32_t* nslot = nullptr;
    float* inlet = nullptr;   // device: the imposed inlet velocity
    float inlet_host[3] = {0.0f, 0.0f, 0.0f};
    bool inlet_set = false;
    std::string error;

    ~orr_gl3d() {
        cudaSetDevice(device);
        for (void* p : {static_cast<void*>(cls), static_cast<void*>(nmask), static_cast<void*>(nslot),
                        static_cast<void*>(inlet)}) {
            if (p) cudaFree(p);
        }
    }
};

namespace {

int32_t wall_kind(uint32_t code) {
    // the driver's wall codes (wall_code, lbm3d_gpu.cpp:64-74)
    return code == 0u ? ORR_WALL_PERIODIC : (code == 1u ? ORR_WALL_SLIP : ORR_WALL_NO_SLIP);
}

// The configuration the driver's uniforms describe (the wall kind of the
// solid walls follows from the node codes: slots mean the interpolated wall).
orr_lbm3d_config config_of(const orr_gl3d_params& p, bool interpolated) {
    orr_lbm3d_config c{};
    c.nx = p.nx;
    c.ny = p.ny;
    c.nz = p.nz;
    c.tau = p.tau;
    c.x_boundary = p.x_mode != 0u ? ORR_X_INFLOW_OUTFLOW : ORR_X_PERIODIC;
    c.outlet = p.outlet_mode != 0u ? ORR_OUTLET_EXTRAPOLATION : ORR_OUTLET_CONVECTIVE;
    orr_wall* walls[4] = {&c.y_low, &c.y_high, &c.z_low, &c.z_high};
    for (int k = 0; k < 4; ++k) {
        walls[k]->kind = wall_kind(p.wall_kind[k]);
        walls[k]->velocity_x = p.wall_ux[k];
    }
    c.inlet_ux = p.inlet[0];
    c.inlet_uy = p.inlet[1];
    c.inlet_uz = p.inlet[2];
    c.body_force_x = p.force[0];
    c.body_force_y = p.force[1];
    c.body_force_z = p.force[2];
    c.smagorinsky_enabled = p.smagorinsky_c2 > 0.0f ? 1 : 0;
    c.smagorinsky_constant = std::sqrt(static_cast<double>(p.smagorinsky_c2));
    c.sponge_strength = p.sponge_strength;
    c.sponge_inlet = p.sponge_inlet;
    c.sponge_outlet = p.sponge_outlet;
    c.sponge_sides = p.sponge_sides;
    c.solid_wall = interpolated ? ORR_SOLID_INTERPOLATED : ORR_SOLID_HALFWAY;
    return c;
}

Phys3D<float> phys_of(const orr_gl3d_params& p) {
    Phys3D<float> q{};
    q.tau = p.tau;
    q.smag_c = std::sqrt(p.smagorinsky_c2);
    q.smag_c2 = p.smagorinsky_c2;
    q.fx = p.force[0];
    q.fy = p.force[1];
    q.fz = p.force[2];
    for (int k = 0; k < 4; ++k) q.wall_ux[k] = p.wall_ux[k];
    q.outlet_speed = p.outlet_speed;
    q.sponge_strength = p.sponge_strength;
    return q;
}

orr_gl3d* tables_of(orr_gl3d* t) {
    if (t == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "gl3d: null tables"};
    }
    check(cudaSetDevice(t->device), "cudaSetDevice");
    return t;
}

void require_same_lattice(const orr_gl3d* t, const orr_gl3d_params* p) {
    if (p == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "gl3d: null parameters"};
    }
    if (p->nx != t->dims.nx || p->ny != t->dims.ny || p->nz != t->dims.nz || p->x_mode != t->dims.x_mode ||
        p->outlet_mode != t->dims.outlet_mode ||
        !std::equal(std::begin(p->wall_kind), std::end(p->wall_kind), std::begin(t->dims.wall_kind))) {
        throw Refusal{ORR_ERR_INVALID, "gl3d: the dispatch's lattice differs from the node-code tables'"};
    }
}

// The driver's force kernel: per link (cell, direction j) the shifted sum of
// the population leaving towards the wall and the one reflected back, in
// binary32 (lbm_d3q19_force.comp.glsl; the reflection of lbm3_reflected with
// the link's wall fraction, 1/2 without a slot).  A link outside the lattice
// writes 0.
__global__ void gl_link_force_kernel(Geom3D g, const float* __restrict__ f, const uint32_t* __restrict__ links,
                                     const int32_t* __restrict__ nslot, const float* __restrict__ wall,
                                     uint32_t count, float* __restrict__ out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint64_t h = links[2u * k];
        const int j = static_cast<int>(links[2u * k + 1u]);
        if (h >= g.cells || j < 1 || j >= d3::Q) {
            out[k] = 0.0f;
            continue;
        }
        const int o = opposite_rt(j);
        int jx, jy, jz;
        c_rt(j, jx, jy, jz);
        const int32_t slot = nslot != nullptr ? nslot[h] : -1;
        float q = slot >= 0 ? wall[static_cast<uint64_t>(slot) * d3::Q + j] : 0.5f;
        const float leaving = f[static_cast<uint64_t>(o) * g.cells + h];
        const int64_t farther = static_cast<int64_t>(h) + jx + static_cast<int64_t>(g.nx) * jy +
                                static_cast<int64_t>(g.plane) * jz;
        if (q < 0.5f && (farther < 0 || static_cast<uint64_t>(farther) >= g.cells)) {
            q = 0.5f;
        }
        float back;
        if (q == 0.5f) {
            back = leaving;
        } else if (q < 0.5f) {
            const float t = lk_mul(2.0f, q);
            back = lk_fma(t, leaving, lk_mul(lk_sub(1.0f, t), f[static_cast<uint64_t>(o) * g.cells + farther]));
        } else {
            const float t = lk_mul(2.0f, q);
            back = r_div(lk_fma(lk_sub(t, 1.0f), f[static_cast<uint64_t>(j) * g.cells + h], leaving), t);
        }
        out[k] = r_add(leaving, back);
    }
}

// Uploads the inlet velocity when it changed since the last dispatch.
void sync_inlet(orr_gl3d* t, const orr_gl3d_params& p, cudaStream_t s) {
    if (t->inlet_set && std::memcmp(t->inlet_host, p.inlet, sizeof t->inlet_host) == 0) {
        return;
    }
    std::memcpy(t->inlet_host, p.inlet, sizeof t->inlet_host);
    // From pageable memory: the call returns once the values are staged.
    check(cudaMemcpyAsync(t->inlet, p.inlet, sizeof t->inlet_host, cudaMemcpyHostToDevice, s), "gl3d inlet");
    t->inlet_set = true;
}

} // namespace

extern "C" {

uint64_t orr_gl3d_buffer_slack(void) {
    return static_cast<uint64_t>(kPopPad) * sizeof(float);
}

orr_status orr_gl3d_create(const orr_gl3d_params* params, const uint32_t* class_codes, int32_t device,
                           orr_gl3d** out) {
    orr::Zone zone("lbm_gl3d_create");
    if (out == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output handle");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (params == nullptr || class_codes == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl3d: null parameters or node codes"};
        }
        const orr_gl3d_params& p = *params;
        if (p.nx < 1 || p.ny < 1 || p.nz < 1) {
            throw Refusal{ORR_ERR_INVALID, "gl3d: empty lattice"};
        }
        const std::size_t cells = static_cast<std::size_t>(p.nx) * p.ny * p.nz;
        std::vector<uint8_t> solid(cells);
        std::vector<int32_t> slot(cells);
        bool interpolated = false;
        for (std::size_t c = 0; c < cells; ++c) {
            solid[c] = class_codes[c] == 0u ? 1u : 0u;
            slot[c] = class_codes[c] >= 3u ? static_cast<int32_t>(class_codes[c] - 3u) : -1;
            interpolated = interpolated || class_codes[c] >= 3u;
        }
        // Node classes and bounce-back masks from the solid nodes (the
        // halfway plan: both depend on the mask and the sides only).
        orr_lbm3d_config c = config_of(p, false);
        // The dispatch's inlet velocity is the instantaneous one (the adapter
        // ramps it up from rest); the lattice is validated with the
        // configured speed, which the driver passes as u_outlet_speed.
        c.inlet_ux = p.outlet_speed;
        if (std::string problem = problem3d(c, solid.data(), nullptr, ORR_STORAGE_F32, true); !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        const Plan3D plan = plan3d(c, solid.data(), nullptr);
        require_device(device);
        check(cudaSetDevice(device), "cudaSetDevice");
        auto t = std::make_unique<orr_gl3d>();
        t->device = device;
        t->dims = p;
        t->interpolated = interpolated;
        c = config_of(p, interpolated);
        Geom3D& g = t->g;
        g.nx = p.nx;
        g.ny = p.ny;
        g.nz = p.nz;
        g.plane = p.nx * p.ny;
        g.cells = cells;
        g.x_mode = c.x_boundary;
        g.outlet_mode = c.outlet;
        g.y_lo = c.y_low.kind;
        g.y_hi = c.y_high.kind;
        g.z_lo = c.z_low.kind;
        g.z_hi = c.z_high.kind;
        g.forced = p.force[0] != 0.0f || p.force[1] != 0.0f || p.force[2] != 0.0f;
        g.sponge = p.sponge_strength > 0.0f && c.x_boundary == ORR_X_INFLOW_OUTFLOW;
        g.sponge_inlet = p.sponge_inlet;
        g.sponge_outlet = p.sponge_outlet;
        g.sponge_sides = p.sponge_sides;
        const auto open_side = [](const orr_wall& w) {
            return w.kind == ORR_WALL_PERIODIC || w.kind == ORR_WALL_SLIP;
        };
        g.flat = open_side(c.y_low) && open_side(c.y_high) && open_side(c.z_low) && open_side(c.z_high) &&
                 !interpolated;
        check(cudaMalloc(reinterpret_cast<void**>(&t->cls), cells + kClassPad), "gl3d class table");
        check(cudaMemsetAsync(t->cls, 0, cells + kClassPad, nullptr), "gl3d class table");
        check(cudaMalloc(reinterpret_cast<void**>(&t->nmask), cells * 4), "gl3d mask table");
        check(cudaMalloc(reinterpret_cast<void**>(&t->inlet), 4 * sizeof(float)), "gl3d inlet");
        check(cudaMemcpy(t->cls, plan.cls.data(), cells, cudaMemcpyHostToDevice), "gl3d class upload");
        check(cudaMemcpy(t->nmask, plan.nmask.data(), cells * 4, cudaMemcpyHostToDevice), "gl3d mask upload");
        if (interpolated) {
            check(cudaMalloc(reinterpret_cast<void**>(&t->nslot), cells * 4), "gl3d slot table");
            check(cudaMemcpy(t->nslot, slot.data(), cells * 4, cudaMemcpyHostToDevice), "gl3d slot upload");
        }
        // The clear and the uploads ran on the legacy stream, and a copy from
        // pageable memory may return before its data lands: wait for them
        // here, since the kernels run on the caller's stream, which need not
        // synchronise with the legacy one.
        check(cudaStreamSynchronize(nullptr), "gl3d table upload");
        *out = t.release();
        return ORR_OK;
    });
}

void orr_gl3d_destroy(orr_gl3d* tables) {
    delete tables;
}

const char* orr_gl3d_last_error(const orr_gl3d* tables) {
    return tables ? tables->error.c_str() : orr_last_error();
}

orr_status orr_gl3d_step(orr_gl3d* tables, const orr_gl3d_params* params, const float* src, float* dst,
                         float* outlet, const float* wall, void* stream) {
    orr::Zone zone("lbm_step");
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        orr_gl3d* t = tables_of(tables);
        require_same_lattice(t, params);
        if (src == nullptr || dst == nullptr || outlet == nullptr || (t->interpolated && wall == nullptr)) {
            throw Refusal{ORR_ERR_INVALID, "gl3d step: null buffer"};
        }
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        sync_inlet(t, *params, s);
        const Phys3D<float> phys = phys_of(*params);
        StepBuffers3D b{};
        b.cls = t->cls;
        b.nmask = t->nmask;
        b.nslot = t->nslot;
        b.wall_q = wall;
        b.hist = outlet;
        b.inlet = t->inlet;
        const bool smag = params->smagorinsky_c2 > 0.0f;
        const uint32_t block = params->nx % 256 == 0 ? 256u : 128u;
        check(ops3d_f32().step(t->g, &phys, src, dst, b, smag, block, 1, s), "gl3d step kernel");
        return ORR_OK;
    });
}

orr_status orr_gl3d_moments(orr_gl3d* tables, const orr_gl3d_params* params, const float* src, float* moments,
                            void* stream) {
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        orr_gl3d* t = tables_of(tables);
        require_same_lattice(t, params);
        if (src == nullptr || moments == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl3d moments: null buffer"};
        }
        const Phys3D<float> phys = phys_of(*params);
        check(ops3d_f32().moments(t->g, &phys, t->cls, src, moments, static_cast<cudaStream_t>(stream)),
              "gl3d moments kernel");
        return ORR_OK;
    });
}

orr_status orr_gl3d_link_force(orr_gl3d* tables, const orr_gl3d_params* params, const float* src,
                               const uint32_t* links, float* link_force, const float* wall, void* stream) {
    orr::Zone zone("lbm_force");
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        orr_gl3d* t = tables_of(tables);
        require_same_lattice(t, params);
        const uint32_t count = params->link_count;
        if (count == 0) {
            return ORR_OK;
        }
        if (src == nullptr || links == nullptr || link_force == nullptr || (t->interpolated && wall == nullptr)) {
            throw Refusal{ORR_ERR_INVALID, "gl3d force: null buffer"};
        }
        const unsigned blocks = std::min<unsigned>((count + 255u) / 256u, 1184u);
        gl_link_force_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
            t->g, src, links, t->nslot, wall, count, link_force);
        check(cudaGetLastError(), "gl3d force kernel");
        return ORR_OK;
    });
}

} // extern "C"
