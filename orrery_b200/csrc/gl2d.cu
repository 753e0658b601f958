// The three D2Q9 kernels of the reference's GPU driver, GpuLbm2D
// (src/aero/lbm/lbm2d_gpu.cpp): lbm_d2q9_step, lbm_d2q9_moments and
// lbm_d2q9_force with the driver's buffers, bindings and uniforms
// (lbm2d_gpu.cpp:36-44, 104-124, 220-300), for an IComputeBackend that runs
// them (orrery_b200/adapter/compute_backend_cuda.cpp).  The 2D twin of
// gl3d.cu.
//
// The driver's buffers are binary32: populations shifted by their weights
// (f - w, structure of arrays, the layout of this library's binary32 D2Q9
// form), solid flags (1 solid, 0 fluid), the convective-outlet history
// (slot * ny + y for directions 3, 6, 7, the layout of this library's), the
// moments (rho - 1, ux, uy planes) and the links (cell, direction pairs).
// The step and moments kernels are this library's binary32 ones, run on
// those buffers; the node classes and bounce-back masks they need are
// derived once from the solid flags by the planner when the tables are
// created.  The force kernel writes, per link, the two components of
// 2 c_o fs_o that the driver turns into the link's force in binary64
// (lbm_d2q9_force.comp.glsl; GpuLbm2D::force, lbm2d_gpu.cpp:284-310).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "kernels2d.cuh"
#include "lattice.h"
#include "ops2d.h"
#include "plan.h"
#include "trace.h"

using namespace orr;

struct orr_gl2d {
    int device = 0;
    orr_gl2d_params dims{};   // the parameters the tables were built for
    Geom2D g{};
    uint8_t* cls = nullptr;
    uint32_t* nmask = nullptr;
    std::string error;

    ~orr_gl2d() {
        cudaSetDevice(device);
        if (cls) cudaFree(cls);
        if (nmask) cudaFree(nmask);
    }
};

namespace {

int32_t wall_kind2(uint32_t code) {
    // the driver's wall codes (wall_code, lbm2d_gpu.cpp:46-56)
    return code == 0u ? ORR_WALL_PERIODIC : (code == 1u ? ORR_WALL_SLIP : ORR_WALL_NO_SLIP);
}

// The configuration the driver's uniforms describe.
orr_lbm2d_config config_of2(const orr_gl2d_params& p) {
    orr_lbm2d_config c{};
    c.nx = p.nx;
    c.ny = p.ny;
    c.tau = p.tau;
    c.x_boundary = p.x_mode != 0u ? ORR_X_INFLOW_OUTFLOW : ORR_X_PERIODIC;
    c.outlet = p.outlet_mode != 0u ? ORR_OUTLET_EXTRAPOLATION : ORR_OUTLET_CONVECTIVE;
    c.bottom.kind = wall_kind2(p.bottom_kind);
    c.bottom.velocity_x = p.bottom_ux;
    c.top.kind = wall_kind2(p.top_kind);
    c.top.velocity_x = p.top_ux;
    c.inlet_ux = p.inlet[0];
    c.inlet_uy = p.inlet[1];
    c.body_force_x = p.force[0];
    c.body_force_y = p.force[1];
    c.smagorinsky_enabled = p.smagorinsky_c2 > 0.0f ? 1 : 0;
    c.smagorinsky_constant = std::sqrt(static_cast<double>(p.smagorinsky_c2));
    return c;
}

Phys2D<float> phys_of2(const orr_gl2d_params& p) {
    Phys2D<float> q{};
    q.tau = p.tau;
    q.smag_c = std::sqrt(p.smagorinsky_c2);
    q.smag_c2 = p.smagorinsky_c2;
    q.fx = p.force[0];
    q.fy = p.force[1];
    q.wall_ux[0] = p.bottom_ux;
    q.wall_ux[1] = p.top_ux;
    q.outlet_speed = p.outlet_speed;
    q.inlet_ux = p.inlet[0];
    q.inlet_uy = p.inlet[1];
    return q;
}

orr_gl2d* tables2_of(orr_gl2d* t) {
    if (t == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "gl2d: null tables"};
    }
    check(cudaSetDevice(t->device), "cudaSetDevice");
    return t;
}

void require_same_lattice2(const orr_gl2d* t, const orr_gl2d_params* p) {
    if (p == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "gl2d: null parameters"};
    }
    if (p->nx != t->dims.nx || p->ny != t->dims.ny || p->x_mode != t->dims.x_mode ||
        p->outlet_mode != t->dims.outlet_mode || p->bottom_kind != t->dims.bottom_kind ||
        p->top_kind != t->dims.top_kind) {
        throw Refusal{ORR_ERR_INVALID, "gl2d: the dispatch's lattice differs from the solid-flag tables'"};
    }
}

// Per link (cell, direction j): the population leaving towards the wall,
// o = opposite(j), as the two components of 2 c_o fs_o
// (lbm_d2q9_force.comp.glsl).  A link outside the lattice writes 0.
__global__ void gl2_link_force_kernel(Geom2D g, const float* __restrict__ f, const uint32_t* __restrict__ links,
                                      uint32_t count, float* __restrict__ out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint64_t h = links[2u * k];
        const int j = static_cast<int>(links[2u * k + 1u]);
        if (h >= g.cells || j < 1 || j >= d2::Q) {
            out[2u * k] = 0.0f;
            out[2u * k + 1u] = 0.0f;
            continue;
        }
        const int o = opposite2_rt(j);
        int ox, oy;
        c2_rt(o, ox, oy);
        const float fs = f[static_cast<uint64_t>(o) * g.cells + h];
        out[2u * k] = __fmul_rn(2.0f * static_cast<float>(ox), fs);
        out[2u * k + 1u] = __fmul_rn(2.0f * static_cast<float>(oy), fs);
    }
}

} // namespace

extern "C" {

orr_status orr_gl2d_create(const orr_gl2d_params* params, const uint32_t* solid_flags, int32_t device,
                           orr_gl2d** out) {
    orr::Zone zone("lbm_gl2d_create");
    if (out == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output handle");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (params == nullptr || solid_flags == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl2d: null parameters or solid flags"};
        }
        const orr_gl2d_params& p = *params;
        if (p.nx < 1 || p.ny < 1) {
            throw Refusal{ORR_ERR_INVALID, "gl2d: empty lattice"};
        }
        const std::size_t cells = static_cast<std::size_t>(p.nx) * p.ny;
        std::vector<uint8_t> solid(cells);
        for (std::size_t c = 0; c < cells; ++c) {
            solid[c] = solid_flags[c] != 0u ? 1u : 0u;
        }
        orr_lbm2d_config c = config_of2(p);
        // Validated with the configured inlet speed (u_outlet_speed), not the
        // instantaneous one of the dispatch.
        c.inlet_ux = p.outlet_speed;
        if (std::string problem = problem2d(c, solid.data(), ORR_STORAGE_F32, true); !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        const Plan2D plan = plan2d(c, solid.data());
        require_device(device);
        check(cudaSetDevice(device), "cudaSetDevice");
        auto t = std::make_unique<orr_gl2d>();
        t->device = device;
        t->dims = p;
        Geom2D& g = t->g;
        g.nx = p.nx;
        g.ny = p.ny;
        g.cells = cells;
        g.x_mode = c.x_boundary;
        g.outlet_mode = c.outlet;
        g.bottom = c.bottom.kind;
        g.top = c.top.kind;
        g.forced = p.force[0] != 0.0f || p.force[1] != 0.0f;
        check(cudaMalloc(reinterpret_cast<void**>(&t->cls), cells), "gl2d class table");
        check(cudaMalloc(reinterpret_cast<void**>(&t->nmask), cells * 4), "gl2d mask table");
        check(cudaMemcpy(t->cls, plan.cls.data(), cells, cudaMemcpyHostToDevice), "gl2d class upload");
        check(cudaMemcpy(t->nmask, plan.nmask.data(), cells * 4, cudaMemcpyHostToDevice), "gl2d mask upload");
        // Landed before any kernel on the caller's stream reads them (copies
        // from pageable memory may return before their data lands).
        check(cudaStreamSynchronize(nullptr), "gl2d table upload");
        *out = t.release();
        return ORR_OK;
    });
}

void orr_gl2d_destroy(orr_gl2d* tables) {
    delete tables;
}

const char* orr_gl2d_last_error(const orr_gl2d* tables) {
    return tables ? tables->error.c_str() : orr_last_error();
}

orr_status orr_gl2d_step(orr_gl2d* tables, const orr_gl2d_params* params, const float* src, float* dst,
                         float* outlet, void* stream) {
    orr::Zone zone("lbm_step");
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        orr_gl2d* t = tables2_of(tables);
        require_same_lattice2(t, params);
        if (src == nullptr || dst == nullptr || outlet == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl2d step: null buffer"};
        }
        const Phys2D<float> phys = phys_of2(*params);
        const StepBuffers2D b{t->cls, t->nmask, outlet};
        const bool smag = params->smagorinsky_c2 > 0.0f;
        check(ops2d_f32().step(t->g, &phys, src, dst, b, smag, 128u, static_cast<cudaStream_t>(stream)),
              "gl2d step kernel");
        return ORR_OK;
    });
}

orr_status orr_gl2d_moments(orr_gl2d* tables, const orr_gl2d_params* params, const float* src, float* moments,
                            void* stream) {
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        orr_gl2d* t = tables2_of(tables);
        require_same_lattice2(t, params);
        if (src == nullptr || moments == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl2d moments: null buffer"};
        }
        const Phys2D<float> phys = phys_of2(*params);
        check(ops2d_f32().moments(t->g, &phys, t->cls, src, moments, static_cast<cudaStream_t>(stream)),
              "gl2d moments kernel");
        return ORR_OK;
    });
}

orr_status orr_gl2d_link_force(orr_gl2d* tables, const orr_gl2d_params* params, const float* src,
                               const uint32_t* links, float* link_force, void* stream) {
    orr::Zone zone("lbm_force");
    return orr::guarded(tables ? &tables->error : nullptr, [&]() -> orr_status {
        if (params == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl2d: null parameters"};
        }
        // The kernel needs the lattice's size only: without tables it runs on
        // the current device with the size of `params`.
        Geom2D g{};
        if (tables != nullptr) {
            orr_gl2d* t = tables2_of(tables);
            require_same_lattice2(t, params);
            g = t->g;
        } else {
            g.nx = params->nx;
            g.ny = params->ny;
            g.cells = static_cast<uint64_t>(params->nx) * params->ny;
        }
        const uint32_t count = params->link_count;
        if (count == 0) {
            return ORR_OK;
        }
        if (src == nullptr || links == nullptr || link_force == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "gl2d force: null buffer"};
        }
        const unsigned blocks = std::min<unsigned>((count + 255u) / 256u, 1184u);
        gl2_link_force_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(g, src, links, count,
                                                                                      link_force);
        check(cudaGetLastError(), "gl2d force kernel");
        return ORR_OK;
    });
}

} // extern "C"
