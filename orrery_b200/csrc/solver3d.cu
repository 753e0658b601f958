// The D3Q19 device solver behind the C ABI: the counterpart of the
// reference's GpuLbm3D (src/aero/lbm3d/lbm3d_gpu.cpp:151-483) and
// make_gpu_solver (:487-513), on CUDA instead of an IComputeBackend.  The
// handle's state and device layout are in solver3d_state.cuh.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "trace.h"
#include "host_copy.h"
#include "kernels3d.cuh"
#include "lattice.h"
#include "lattice_table.cuh"
#include "ops3d.h"
#include "plan.h"
#include "solver3d_state.cuh"

using namespace orr;

namespace {

orr_lbm3d* handle_of(orr_lbm3d* h) {
    if (h == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "null solver handle"};
    }
    check(cudaSetDevice(h->device), "cudaSetDevice");
    return h;
}

template <class P> void fill_phys(P& p, const orr_lbm3d_config& c, bool binary32) {
    using A = decltype(p.tau);
    const auto cv = [binary32](double v) -> A {
        return binary32 ? static_cast<A>(static_cast<float>(v)) : static_cast<A>(v);
    };
    const double k = c.smagorinsky_enabled ? c.smagorinsky_constant : 0.0;
    p.tau = cv(c.tau);
    p.smag_c = cv(k);
    p.smag_c2 = cv(k * k);
    p.fx = cv(c.body_force_x);
    p.fy = cv(c.body_force_y);
    p.fz = cv(c.body_force_z);
    p.wall_ux[0] = cv(c.y_low.velocity_x);
    p.wall_ux[1] = cv(c.y_high.velocity_x);
    p.wall_ux[2] = cv(c.z_low.velocity_x);
    p.wall_ux[3] = cv(c.z_high.velocity_x);
    p.outlet_speed = cv(c.inlet_ux);
    p.sponge_strength = cv(c.sponge_strength);
}

orr_solver_options options_or_default(const orr_solver_options* o) {
    orr_solver_options d{};
    d.storage = ORR_STORAGE_F32;
    d.allow_high_mach = 0;
    d.device = 0;
    d.block_x = 0;
    return o ? *o : d;
}

void copy_message(const std::string& text, char* message, size_t capacity) {
    if (message == nullptr || capacity == 0) {
        return;
    }
    const size_t n = std::min(text.size(), capacity - 1);
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

void initialize_state(orr_lbm3d* h, const double* rho, const double* ux, const double* uy,
                      const double* uz, bool at_rest = false) {
    const auto& c = h->plan.c;
    const std::size_t cells = h->plan.cells;
    double* staged[4] = {nullptr, nullptr, nullptr, nullptr};
    if (rho != nullptr) {
        // Stage the four fields in the other population buffer: 32 bytes per
        // node fit in 19 storage values of at least 2 bytes.
        double* base = static_cast<double*>(h->f[1]);
        const double* src[4] = {rho, ux, uy, uz};
        orr::HostSpan spans[4];
        for (int k = 0; k < 4; ++k) {
            staged[k] = base + static_cast<std::size_t>(k) * cells;
            spans[k] = {const_cast<double*>(src[k]), staged[k], cells * sizeof(double)};
        }
        orr::copy_to_device(spans, 4, h->stream, h->device);
    }
    const bool inflow = c.x_boundary == ORR_X_INFLOW_OUTFLOW && !at_rest;
    check(h->ops->init(h->g, h->cls, staged[0], staged[1], staged[2], staged[3], 1.0,
                       inflow ? c.inlet_ux : 0.0, inflow ? c.inlet_uy : 0.0,
                       inflow ? c.inlet_uz : 0.0, h->f[0], h->stream),
          "init kernel");
    check(cudaMemcpyAsync(h->f[1], h->f[0], d3::Q * cells * h->sbytes, cudaMemcpyDeviceToDevice,
                          h->stream),
          "population copy");
    check(h->ops->history(h->g, h->f[0], h->hist, h->stream), "history kernel");
    // The status word and the stall-request word after it.
    check(cudaMemsetAsync(h->status(), 0, 2 * sizeof(uint32_t), h->stream), "status reset");
    ++h->epoch;
    h->launches += 2;
    h->cur = 0;
    h->steps = 0;
    const double v[3] = {at_rest ? 0.0 : c.inlet_ux, at_rest ? 0.0 : c.inlet_uy, at_rest ? 0.0 : c.inlet_uz};
    h->upload_inlet(v);
}

// Unshifted binary64 populations of directions [i0, i0 + gridDim.y) from a
// shifted storage (value + w_i, the host's decode), written direction-major
// where the host copies them from.
template <class S>
__global__ void widen_populations_kernel(const S* __restrict__ f, double* __restrict__ out, uint64_t cells, int i0) {
    const int i = i0 + static_cast<int>(blockIdx.y);
    const double w = d3::w(i);
    const S* src = f + static_cast<uint64_t>(i) * cells;
    double* dst = out + static_cast<uint64_t>(blockIdx.y) * cells;
    for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < cells;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        dst[c] = static_cast<double>(Storage<S>::value(src[c])) + w;
    }
}

} // namespace

void orr::initialize_at_rest(orr_lbm3d* h) {
    check(cudaSetDevice(h->device), "cudaSetDevice");
    initialize_state(h, nullptr, nullptr, nullptr, nullptr, true);
    check(cudaStreamSynchronize(h->stream), "initialize");
}

extern "C" {

orr_status orr_lbm3d_validate(const orr_lbm3d_config* config, const uint8_t* solid,
                              const double* distance, const orr_solver_options* options,
                              char* message, size_t capacity) {
    if (config == nullptr) {
        copy_message("null configuration", message, capacity);
        return orr::fail(ORR_ERR_INVALID, "null configuration");
    }
    const orr_solver_options o = options_or_default(options);
    const std::string problem =
        orr::problem3d(*config, solid, distance, o.storage, o.allow_high_mach != 0);
    copy_message(problem, message, capacity);
    if (!problem.empty()) {
        return orr::fail(ORR_ERR_INVALID, problem);
    }
    return ORR_OK;
}

orr_status orr_lbm3d_memory_bytes(const orr_lbm3d_config* config, uint64_t links,
                                  uint64_t boundary_nodes, int32_t storage, uint64_t* bytes) {
    if (config == nullptr || bytes == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    const auto m = orr::memory3d(*config, links,
                                 config->solid_wall == ORR_SOLID_INTERPOLATED ? boundary_nodes : 0,
                                 storage);
    if (!m) {
        return orr::fail(ORR_ERR_INVALID, "lbm3d gpu: the device memory of the lattice overflows std::size_t");
    }
    *bytes = *m;
    return ORR_OK;
}

orr_status orr_lbm3d_plan(const orr_lbm3d_config* config, const uint8_t* solid,
                          const double* distance, uint64_t* links, uint64_t* fluid,
                          uint64_t* boundary_nodes, uint32_t* cell, uint32_t* direction,
                          double* q) {
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (config == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null configuration"};
        }
        if (std::string problem = problem3d(*config, solid, distance, ORR_STORAGE_F64, true);
            !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        const Plan3D p = plan3d(*config, solid, distance);
        const std::size_t n = p.link_cell.size();
        if (links) *links = n;
        if (fluid) *fluid = p.fluid;
        if (boundary_nodes) *boundary_nodes = p.general;
        if (cell) std::memcpy(cell, p.link_cell.data(), n * 4);
        if (direction) std::memcpy(direction, p.link_dir.data(), n * 4);
        if (q) std::memcpy(q, p.link_q.data(), n * 8);
        return ORR_OK;
    });
}

orr_status orr_lbm3d_create(const orr_lbm3d_config* config, const uint8_t* solid,
                            const double* distance, const orr_solver_options* options,
                            orr_lbm3d** out) {
    orr::Zone zone("lbm_create");
    if (out == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output handle");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (config == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null configuration"};
        }
        const orr_solver_options o = options_or_default(options);
        // validate() and the binary32 checks, before anything is allocated.
        if (std::string problem =
                problem3d(*config, solid, distance, o.storage, o.allow_high_mach != 0);
            !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        const bool tiled_block = o.kernel == ORR_KERNEL_TILED && (o.block_x == 256 || o.block_x == 512);
        if (!tiled_block && (o.block_x < 0 || o.block_x > 256 || (o.block_x % 32) != 0)) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: block_x must be 0 or a multiple of 32 up to 256 "
                                           "(256 or 512 consumer threads for the tiled step)"};
        }
        if (o.kernel < ORR_KERNEL_AUTO || o.kernel > ORR_KERNEL_TILED) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: unknown step kernel"};
        }
        if (o.kernel == ORR_KERNEL_STAGED && o.block_x != 0 && o.block_x != 128 && o.block_x != 256) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the staged step takes block_x 128 or 256"};
        }
        if (o.stages < 0 || o.stages > static_cast<int32_t>(kMaxStages)) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: stages must be 0 (tuned) or 1 to 8"};
        }
        if (o.nodes_per_thread < 0 || o.nodes_per_thread > 2) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: nodes_per_thread must be 0 (default), 1 or 2"};
        }
        require_device(o.device);
        auto h = std::make_unique<orr_lbm3d>();
        h->device = o.device;
        h->storage = o.storage;
        h->allow_high_mach = o.allow_high_mach != 0;
        // Default row tile: 256 nodes for binary32 storage when they divide
        // the rows (the row step is memory bound there and longer tiles read
        // a little faster), else 128.
        h->block = o.block_x > 0 && o.block_x <= 256 ? static_cast<uint32_t>(o.block_x)
                   : (o.storage == ORR_STORAGE_F32 && config->nx % 256 == 0) ? 256u
                                                                              : kDefaultBlock;
        h->ops = &ops_for(o.storage);
        h->sbytes = storage_bytes(o.storage);
        h->abytes = arithmetic_bytes(o.storage);
        // A helper thread reads the free device memory (a query that has
        // taken milliseconds) and, when the part of the memory check that
        // follows from the configuration alone fits, allocates those buffers,
        // while this thread plans the lattice; the full check, with the plan's
        // links and wall slots, follows against the free memory it read.
        const std::size_t cells = static_cast<std::size_t>(config->nx) * config->ny * config->nz;
        const bool interpolated = config->solid_wall == ORR_SOLID_INTERPOLATED;
        orr_lbm3d* hp = h.get();
        const auto allocate_fixed = [hp, cells, interpolated, config]() {
            check(cudaSetDevice(hp->device), "cudaSetDevice");
            check(cudaStreamCreateWithFlags(&hp->stream, cudaStreamNonBlocking), "stream");
            for (int k = 0; k < 2; ++k) {
                const std::size_t bytes = (d3::Q * cells + 2 * kPopPad) * hp->sbytes;
                check(cudaMalloc(&hp->fbase[k], bytes), "population buffer");
                check(cudaMemsetAsync(hp->fbase[k], 0, bytes, hp->stream), "population buffer");
                hp->f[k] = static_cast<char*>(hp->fbase[k]) + kPopPad * hp->sbytes;
            }
            hp->cls = device_alloc<uint8_t>(cells + kClassPad, "node class buffer");
            check(cudaMemsetAsync(hp->cls + cells, 0, kClassPad, hp->stream), "node class buffer");
            hp->nmask = device_alloc<uint32_t>(cells, "bounce-back mask buffer");
            if (interpolated) {
                hp->nslot = device_alloc<int32_t>(cells, "wall slot buffer");
            }
            check(cudaMalloc(&hp->hist,
                             static_cast<std::size_t>(d3::kOutletSlots) * config->ny * config->nz * hp->abytes),
                  "outlet buffer");
            check(cudaMalloc(&hp->moments, 4 * cells * hp->abytes), "moment buffer");
            check(cudaMalloc(&hp->small, 256), "small buffer");
            check(cudaMemsetAsync(hp->small, 0, 256, hp->stream), "small buffer");
            check(cudaMallocHost(reinterpret_cast<void**>(&hp->host_small), 256), "pinned buffer");
            check(cudaMalloc(&hp->table, kTableBytes), "lattice table");
        };
        std::size_t free_bytes = 0, total_bytes = 0;
        {
            const auto fixed = memory3d(*config, 0, 0, o.storage);
            std::exception_ptr failed;
            std::thread helper([&] {
                try {
                    check(cudaSetDevice(hp->device), "cudaSetDevice");
                    check(cudaMemGetInfo(&free_bytes, &total_bytes), "cudaMemGetInfo");
                    if (fixed && *fixed <= free_bytes) {
                        allocate_fixed();
                    }
                } catch (...) {
                    failed = std::current_exception();
                }
            });
            try {
                h->plan = plan3d(*config, solid, distance);
            } catch (...) {
                helper.join();
                throw;
            }
            helper.join();
            if (failed) {
                std::rethrow_exception(failed);
            }
        }
        const Plan3D& p = h->plan;
        // The memory check counts every table the solver allocates
        // (check_memory, lbm3d_gpu.cpp:129-149).
        const std::size_t slots = p.wall_q.size() / d3::Q;
        const auto need = memory3d(*config, p.link_cell.size(), slots, o.storage);
        if (!need) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the device memory of the lattice overflows std::size_t"};
        }
        if (*need > free_bytes) {
            throw Refusal{ORR_ERR_MEMORY, "lbm3d gpu: the lattice needs " + mebibytes(*need) +
                                              " of device memory, " + mebibytes(free_bytes) +
                                              " are available; use fewer cells"};
        }
        // Geometry and parameters.
        Geom3D& g = h->g;
        g.nx = static_cast<uint32_t>(config->nx);
        g.ny = static_cast<uint32_t>(config->ny);
        g.nz = static_cast<uint32_t>(config->nz);
        g.plane = g.nx * g.ny;
        g.cells = p.cells;
        g.x_mode = config->x_boundary;
        g.outlet_mode = config->outlet;
        g.y_lo = config->y_low.kind;
        g.y_hi = config->y_high.kind;
        g.z_lo = config->z_low.kind;
        g.z_hi = config->z_high.kind;
        g.forced = config->body_force_x != 0.0 || config->body_force_y != 0.0 ||
                   config->body_force_z != 0.0;
        g.sponge = config->sponge_strength > 0.0 && config->x_boundary == ORR_X_INFLOW_OUTFLOW;
        g.sponge_inlet = static_cast<uint32_t>(config->sponge_inlet);
        g.sponge_outlet = static_cast<uint32_t>(config->sponge_outlet);
        g.sponge_sides = static_cast<uint32_t>(config->sponge_sides);
        const auto open_side = [](const orr_wall& w) {
            return w.kind == ORR_WALL_PERIODIC || w.kind == ORR_WALL_SLIP;
        };
        g.flat = open_side(config->y_low) && open_side(config->y_high) && open_side(config->z_low) &&
                 open_side(config->z_high) && config->solid_wall == ORR_SOLID_HALFWAY;
        const bool binary32 = o.storage != ORR_STORAGE_F64;
        if (binary32) {
            g.forced = to_f32(config->body_force_x) != 0.0f || to_f32(config->body_force_y) != 0.0f ||
                       to_f32(config->body_force_z) != 0.0f;
        }
        fill_phys(h->phys32, *config, true);
        fill_phys(h->phys64, *config, false);
        h->smag = config->smagorinsky_enabled != 0 &&
                  (binary32 ? h->phys32.smag_c2 > 0.0f : true);
        // Streams and device tables (the plan-sized ones here; the others
        // unless the helper made them).
        if (h->stream == nullptr) {
            allocate_fixed();
        }
        check(cudaMalloc(&h->wall_q, std::max<std::size_t>(slots, 1) * d3::Q * h->abytes), "wall buffer");
        h->lcell = device_alloc<uint32_t>(p.link_cell.size(), "link buffer");
        h->ldir = device_alloc<uint32_t>(p.link_cell.size(), "link buffer");
        h->lq = device_alloc<double>(p.link_cell.size(), "link buffer");
        // Uploads.
        cudaStream_t s = h->stream;
        {
            orr::HostSpan tables[3] = {
                {const_cast<uint8_t*>(p.cls.data()), h->cls, cells},
                {const_cast<uint32_t*>(p.nmask.data()), h->nmask, cells * 4},
                {const_cast<int32_t*>(p.nslot.data()), h->nslot, p.nslot.empty() ? 0 : cells * 4}};
            orr::copy_to_device(tables, 3, s, h->device);
        }
        {
            std::vector<double> q = p.wall_q;
            if (q.empty()) {
                q.assign(d3::Q, 0.5);
            }
            if (binary32) {
                std::vector<float> qf(q.begin(), q.end());
                check(cudaMemcpyAsync(h->wall_q, qf.data(), qf.size() * 4, cudaMemcpyHostToDevice, s),
                      "wall upload");
                check(cudaStreamSynchronize(s), "wall upload");
            } else {
                check(cudaMemcpyAsync(h->wall_q, q.data(), q.size() * 8, cudaMemcpyHostToDevice, s),
                      "wall upload");
                check(cudaStreamSynchronize(s), "wall upload");
            }
        }
        if (!p.link_cell.empty()) {
            const std::size_t n = p.link_cell.size();
            check(cudaMemcpyAsync(h->lcell, p.link_cell.data(), n * 4, cudaMemcpyHostToDevice, s), "link upload");
            check(cudaMemcpyAsync(h->ldir, p.link_dir.data(), n * 4, cudaMemcpyHostToDevice, s), "link upload");
            check(cudaMemcpyAsync(h->lq, p.link_q.data(), n * 8, cudaMemcpyHostToDevice, s), "link upload");
        }
        // Step kernel: the row-tile step, or the persistent staged or tiled
        // step when asked for.
        if (o.kernel == ORR_KERNEL_STAGED && !g.flat) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the staged step needs periodic or free-slip sides "
                                           "and halfway walls"};
        }
        if (o.kernel == ORR_KERNEL_TILED && !tileable(g)) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the tiled step needs periodic or free-slip sides, "
                                           "halfway walls and rows of a multiple of 16 nodes"};
        }
        // The tiled step: when asked for (512 consumer threads and tiles of
        // 8 rows, or 256 and 4).
        if (o.kernel == ORR_KERNEL_TILED) {
            const uint32_t tblock = o.block_x == 256 ? 256u : 512u;
            // Rows per tile: two nodes per consumer thread (the default), or
            // one with nodes_per_thread 1.
            const uint32_t rows = tblock * (o.nodes_per_thread == 1 ? 1u : 2u) / kTileW;
            h->shape = tiled_shape(*h->ops, h->smag, rows, tblock, static_cast<uint32_t>(o.stages), o.device);
            if (h->shape.per_sm <= 0) {
                throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the tiled step cannot launch with " +
                                                   std::to_string(h->shape.stages) + " stages"};
            }
            if (std::string why = encode_tile_maps(h->tmaps, g, h->f[0], h->f[1], h->cls, h->sbytes, rows);
                !why.empty()) {
                throw Refusal{ORR_ERR_CUDA, "lbm3d gpu: " + why};
            }
            h->tiled = true;
            h->tile_rows = rows;
            if (binary32) {
                h->upload_table(h->phys32);
            } else {
                h->upload_table(h->phys64);
            }
            h->tgrid = tile_grid(g, rows, tblock);
            const uint64_t most = std::max<uint64_t>({h->tgrid.tiles, h->tgrid.direct, 1});
            h->shape.grid = static_cast<uint32_t>(std::min<uint64_t>(h->shape.grid, most));
        }
        // The automatic choice is the row kernel for every storage: at 40
        // registers it runs the 2-byte forms faster than the staged kernel
        // (47.4 against 45.0 GLUPS for binary16 on the 256 x 128 x 128 sphere)
        // with no pipeline to wait on.
        const bool want = !h->tiled && o.kernel == ORR_KERNEL_STAGED;
        if (want) {
            const uint32_t sblock = o.block_x == 128 ? 128u : 256u;
            const uint32_t npt = o.nodes_per_thread > 0 ? static_cast<uint32_t>(o.nodes_per_thread)
                                                        : default_npt(o.storage);
            h->shape = staged_shape(*h->ops, h->smag, sblock, npt, static_cast<uint32_t>(o.stages), o.device);
            if (h->shape.per_sm <= 0) {
                if (o.kernel == ORR_KERNEL_STAGED) {
                    throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: the staged step cannot launch with " +
                                                       std::to_string(h->shape.stages) + " stages"};
                }
            } else {
                h->persistent = true;
                if (binary32) {
                    h->upload_table(h->phys32);
                } else {
                    h->upload_table(h->phys64);
                }
                // No more CTAs than items.
                const uint64_t most = std::max<uint64_t>({h->items.staged, h->items.direct, 1});
                h->shape.grid = static_cast<uint32_t>(std::min<uint64_t>(h->shape.grid, most));
            }
        }
        if (!h->persistent && !h->tiled && o.nodes_per_thread == 2) {
            // Row-tile step with two neighbouring nodes per thread.
            if (!h->ops->pairs_ok(g, h->block)) {
                throw Refusal{ORR_ERR_INVALID, "lbm3d gpu: two nodes per thread of the row step need 2-byte "
                                               "storage, periodic or free-slip sides, halfway walls, an even nx "
                                               "and blocks of at most 128 threads"};
            }
            h->row_npt = 2;
        }
        initialize_state(h.get(), nullptr, nullptr, nullptr, nullptr);
        // Capture the step graph now, so that no step() call, the first
        // included, does host capture or instantiation work between its
        // launches.
        h->build_graph();
        check(cudaStreamSynchronize(s), "create");
        // The per-node tables are on the device now; keep the links.
        h->plan.cls.clear();
        h->plan.cls.shrink_to_fit();
        h->plan.nmask.clear();
        h->plan.nmask.shrink_to_fit();
        h->plan.nslot.clear();
        h->plan.nslot.shrink_to_fit();
        *out = h.release();
        return ORR_OK;
    });
}

void orr_lbm3d_destroy(orr_lbm3d* solver) {
    if (solver != nullptr && solver->batch != nullptr) {
        orr_batch3d_forget(solver->batch, solver);
    }
    delete solver;
}

const char* orr_lbm3d_last_error(const orr_lbm3d* solver) {
    return solver ? solver->error.c_str() : orr_last_error();
}

orr_status orr_lbm3d_initialize(orr_lbm3d* solver, const double* rho, const double* ux,
                                const double* uy, const double* uz) {
    orr::Zone zone("lbm_initialize");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        const bool any = rho || ux || uy || uz;
        const bool all = rho && ux && uy && uz;
        if (any && !all) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d: initialize needs all four fields or none"};
        }
        initialize_state(h, rho, ux, uy, uz);
        check(cudaStreamSynchronize(h->stream), "initialize");
        return ORR_OK;
    });
}

orr_status orr_lbm3d_step(orr_lbm3d* solver, uint64_t count) {
    orr::Zone zone("lbm_step");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (h->batch != nullptr) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d: the solver belongs to a batch; step the batch"};
        }
        h->run(count);
        return ORR_OK;
    });
}

orr_status orr_lbm3d_steps(const orr_lbm3d* solver, uint64_t* steps) {
    if (solver == nullptr || steps == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *steps = solver->steps;
    return ORR_OK;
}

orr_status orr_lbm3d_set_inlet_velocity(orr_lbm3d* solver, const double velocity[3]) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (velocity == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null velocity"};
        }
        if (std::string problem = inlet_problem3d(h->plan.c, velocity, h->allow_high_mach);
            !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        h->upload_inlet(velocity);
        return ORR_OK;
    });
}

orr_status orr_lbm3d_inlet_velocity(const orr_lbm3d* solver, double velocity[3]) {
    if (solver == nullptr || velocity == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    std::memcpy(velocity, solver->inlet, 3 * sizeof(double));
    return ORR_OK;
}

orr_status orr_lbm3d_force(orr_lbm3d* solver, double force_moment[6]) {
    orr::Zone zone("lbm_force");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (force_moment == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        const std::size_t links = h->plan.link_cell.size();
        check(h->ops->force(h->g, h->f[h->cur], h->lcell, h->ldir, h->lq, links, h->acc(), h->stream),
              "force kernel");
        if (links > 0) {
            ++h->launches;
        }
        // One read-back: the six sums (64 bytes into the small buffer) and,
        // for the persistent step, its status word (kStatusOffset).
        static_assert(kStatusOffset >= 64 + 6 * sizeof(double) && kStatusOffset + 4 <= 64 + 192);
        const bool watched = h->persistent || h->tiled;
        const std::size_t bytes = watched ? kStatusOffset + 4 - 64 : 6 * sizeof(double);
        check(cudaMemcpyAsync(h->host_small + 8, h->acc(), bytes, cudaMemcpyDeviceToHost, h->stream),
              "force read-back");
        check(cudaStreamSynchronize(h->stream), "force read-back");
        if (watched) {
            uint32_t word = 0;
            std::memcpy(&word, reinterpret_cast<const char*>(h->host_small + 8) + (kStatusOffset - 64), 4);
            orr_lbm3d::raise_status(word);
        }
        std::memcpy(force_moment, h->host_small + 8, 6 * sizeof(double));
        return ORR_OK;
    });
}

orr_status orr_lbm3d_macroscopic(orr_lbm3d* solver, double* rho, double* ux, double* uy,
                                 double* uz) {
    orr::Zone zone("lbm_macroscopic");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        h->check_status();
        const std::size_t cells = h->plan.cells;
        check(h->ops->moments(h->g, h->phys(), h->cls, h->f[h->cur], h->moments, h->stream),
              "moments kernel");
        ++h->launches;
        double* outs[4] = {rho, ux, uy, uz};
        // The binary32 planes of the shifted forms (rho - 1, ux, uy, uz) cross
        // the bus as binary32 and are widened to binary64 by the host threads
        // of the staged copy, rho with 1 added back (exact: rho - 1 has 24
        // significant bits and 1 + (rho - 1) fits in 53); binary64 planes are
        // copied as they are.
        const bool narrow = h->storage != ORR_STORAGE_F64;
        orr::HostSpan spans[4];
        int count = 0;
        for (int k = 0; k < 4; ++k) {
            if (outs[k] == nullptr) {
                continue;
            }
            if (narrow) {
                spans[count++] = {outs[k], static_cast<float*>(h->moments) + k * cells, cells * 4, true,
                                  k == 0 ? 1.0 : 0.0};
            } else {
                spans[count++] = {outs[k], static_cast<double*>(h->moments) + k * cells, cells * 8};
            }
        }
        orr::copy_to_host(spans, count, h->stream, h->device);
        return ORR_OK;
    });
}

orr_status orr_lbm3d_populations(orr_lbm3d* solver, double* f) {
    orr::Zone zone("lbm_populations");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (f == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        h->check_status();
        const std::size_t cells = h->plan.cells;
        const std::size_t n = d3::Q * cells;
        if (h->storage == ORR_STORAGE_F64) {
            const orr::HostSpan all{f, h->f[h->cur], n * 8};
            orr::copy_to_host(&all, 1, h->stream, h->device);
            return ORR_OK;
        }
        // The shifted values are widened on the device into the idle
        // population buffer (which the next step overwrites whole), as many
        // directions at a time as it holds in binary64, and each pass is
        // copied straight into the caller's array.
        const int per_pass = static_cast<int>(d3::Q * h->sbytes / 8);
        double* wide = static_cast<double*>(h->f[1 - h->cur]);
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((cells + 255) / 256, 1184));
        for (int i0 = 0; i0 < d3::Q; i0 += per_pass) {
            const int count = std::min(per_pass, d3::Q - i0);
            const dim3 grid(blocks, static_cast<unsigned>(count));
            if (h->storage == ORR_STORAGE_F32) {
                widen_populations_kernel<<<grid, 256, 0, h->stream>>>(static_cast<const float*>(h->f[h->cur]), wide,
                                                                      cells, i0);
            } else if (h->storage == ORR_STORAGE_F16) {
                widen_populations_kernel<<<grid, 256, 0, h->stream>>>(static_cast<const __half*>(h->f[h->cur]),
                                                                      wide, cells, i0);
            } else {
                widen_populations_kernel<<<grid, 256, 0, h->stream>>>(
                    static_cast<const __nv_bfloat16*>(h->f[h->cur]), wide, cells, i0);
            }
            check(cudaGetLastError(), "population widening");
            ++h->launches;
            const orr::HostSpan part{f + static_cast<std::size_t>(i0) * cells, wide,
                                     static_cast<std::size_t>(count) * cells * 8};
            orr::copy_to_host(&part, 1, h->stream, h->device);
        }
        return ORR_OK;
    });
}

orr_status orr_lbm3d_mass(orr_lbm3d* solver, double* mass) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (mass == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        check(h->ops->mass(h->g, h->cls, h->f[h->cur], h->acc() + 6, h->stream), "mass kernel");
        ++h->launches;
        check(cudaMemcpyAsync(h->host_small + 16, h->acc() + 6, sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream),
              "mass read-back");
        check(cudaStreamSynchronize(h->stream), "mass read-back");
        h->check_status();
        double m = h->host_small[16];
        if (h->storage != ORR_STORAGE_F64) {
            m += static_cast<double>(h->plan.fluid); // the weights of each fluid node add up to 1
        }
        *mass = m;
        return ORR_OK;
    });
}

orr_status orr_lbm3d_link_count(const orr_lbm3d* solver, uint64_t* count) {
    if (solver == nullptr || count == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *count = solver->plan.link_cell.size();
    return ORR_OK;
}

orr_status orr_lbm3d_links(const orr_lbm3d* solver, uint32_t* cell, uint32_t* direction,
                           double* q) {
    if (solver == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    const Plan3D& p = solver->plan;
    const std::size_t n = p.link_cell.size();
    if (cell) std::memcpy(cell, p.link_cell.data(), n * 4);
    if (direction) std::memcpy(direction, p.link_dir.data(), n * 4);
    if (q) std::memcpy(q, p.link_q.data(), n * 8);
    return ORR_OK;
}

orr_status orr_lbm3d_node_counts(const orr_lbm3d* solver, uint64_t* fluid, uint64_t* boundary) {
    if (solver == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    if (fluid) *fluid = solver->plan.fluid;
    if (boundary) *boundary = solver->plan.general;
    return ORR_OK;
}

orr_status orr_lbm3d_stream(const orr_lbm3d* solver, void** stream) {
    if (solver == nullptr || stream == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *stream = solver->stream;
    return ORR_OK;
}

orr_status orr_lbm3d_kernel_info(const orr_lbm3d* solver, orr_kernel_info* info) {
    if (solver == nullptr || info == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    return orr::guarded(nullptr, [&]() -> orr_status {
        check(cudaSetDevice(solver->device), "cudaSetDevice");
        orr_kernel_info k{};
        if (solver->tiled) {
            k.kernel = ORR_KERNEL_TILED;
            k.block = solver->shape.block;
            k.stages = solver->shape.stages;
            k.grid = solver->shape.grid;
            k.ctas_per_sm = solver->shape.per_sm;
            k.registers = solver->ops->tiled_registers(solver->smag, solver->tile_rows, solver->shape.block);
            k.shared_bytes = 0;
            k.nodes_per_thread = solver->shape.npt;
            k.staged_items = solver->tgrid.tiles;
            k.direct_items = solver->tgrid.direct;
        } else if (solver->persistent) {
            k.kernel = ORR_KERNEL_STAGED;
            k.block = solver->shape.block;
            k.stages = solver->shape.stages;
            k.grid = solver->shape.grid;
            k.ctas_per_sm = solver->shape.per_sm;
            k.registers = solver->ops->staged_registers(solver->smag, solver->shape.block, solver->shape.npt);
            k.shared_bytes = solver->ops->staged_smem(solver->shape.block, solver->shape.npt, solver->shape.stages);
            k.nodes_per_thread = solver->shape.npt;
            k.staged_items = solver->items.staged;
            k.direct_items = solver->items.direct;
        } else {
            k.kernel = ORR_KERNEL_ROWS;
            k.block = solver->block;
            const uint32_t span = solver->block * solver->row_npt;
            k.nodes_per_thread = solver->row_npt;
            k.grid = ((solver->g.nx + span - 1) / span) * solver->g.ny * solver->g.nz;
            k.registers = solver->ops->step_registers(solver->smag, solver->row_npt);
        }
        *info = k;
        return ORR_OK;
    });
}

orr_status orr_lbm3d_launch_count(const orr_lbm3d* solver, uint64_t* launches) {
    if (solver == nullptr || launches == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *launches = solver->launches;
    return ORR_OK;
}

orr_status orr_lbm3d_request_stall(orr_lbm3d* solver, uint32_t cta) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm3d* h = handle_of(solver);
        if (!h->persistent && !h->tiled) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d: a stall request needs the staged or tiled step"};
        }
        const uint64_t ctas = std::min<uint64_t>(h->shape.grid, h->tiled ? h->tgrid.tiles : h->items.staged);
        if (cta >= ctas) {
            throw Refusal{ORR_ERR_INVALID, "lbm3d: the stall request names a CTA without staged spans"};
        }
        uint32_t* word = reinterpret_cast<uint32_t*>(h->host_small + 31);
        *word = cta + 1u;
        check(cudaMemcpyAsync(h->status() + 1, word, sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream),
              "stall request");
        check(cudaStreamSynchronize(h->stream), "stall request");
        return ORR_OK;
    });
}

} // extern "C"
