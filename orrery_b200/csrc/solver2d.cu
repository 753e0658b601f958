// The D2Q9 device solver behind the C ABI: the counterpart of the
// reference's GpuLbm2D (src/aero/lbm/lbm2d_gpu.cpp) and the 2D make_gpu_solver
// (src/aero/lbm/include/orrery/aero/lbm/lbm2d.h:205-212).  Same layout and
// execution as the D3Q19 solver: ping-pong SoA populations and one all-rows
// step kernel per step, replayed as CUDA graphs.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "trace.h"
#include "kernels2d.cuh"
#include "lattice.h"
#include "ops2d.h"
#include "plan.h"

namespace {

using namespace orr;

constexpr uint32_t kGraphSteps2 = 16;
constexpr uint32_t kDefaultBlock2 = 128;

const Ops2D& ops2_for(int32_t storage) {
    switch (storage) {
        case ORR_STORAGE_F16:
            return ops2d_f16();
        case ORR_STORAGE_BF16:
            return ops2d_bf16();
        case ORR_STORAGE_F64:
            return ops2d_f64();
        default:
            return ops2d_f32();
    }
}

} // namespace

struct orr_lbm2d {
    Plan2D plan;
    int32_t storage = ORR_STORAGE_F32;
    int device = 0;
    uint32_t block = kDefaultBlock2;
    const Ops2D* ops = nullptr;
    Geom2D g{};
    Phys2D<float> phys32{};
    Phys2D<double> phys64{};
    bool smag = false;
    std::size_t sbytes = 4, abytes = 4;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    uint8_t* cls = nullptr;
    uint32_t* nmask = nullptr;
    void* hist = nullptr;
    void* moments = nullptr;
    uint32_t* lcell = nullptr;
    uint32_t* ldir = nullptr;
    double* acc = nullptr;
    double* host_acc = nullptr;
    uint64_t steps = 0, launches = 0;
    std::string error;

    const void* phys() const {
        return storage == ORR_STORAGE_F64 ? static_cast<const void*>(&phys64)
                                          : static_cast<const void*>(&phys32);
    }
    StepBuffers2D buffers() const { return StepBuffers2D{cls, nmask, hist}; }

    ~orr_lbm2d() {
        cudaSetDevice(device);
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : {f[0], f[1], static_cast<void*>(cls), static_cast<void*>(nmask), hist, moments,
                        static_cast<void*>(lcell), static_cast<void*>(ldir), static_cast<void*>(acc)}) {
            if (p) cudaFree(p);
        }
        if (host_acc) cudaFreeHost(host_acc);
        if (stream) cudaStreamDestroy(stream);
    }

    void launch_step(int from) {
        const StepBuffers2D b = buffers();
        check(ops->step(g, phys(), f[from], f[1 - from], b, smag, block, stream), "step kernel");
        ++launches;
    }

    // Captures kGraphSteps2 steps (buffer 0 -> 1 -> ... -> 0) as one graph.
    void build_graph() {
        cudaGraph_t captured = nullptr;
        const uint64_t before = launches;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        try {
            for (uint32_t k = 0; k < kGraphSteps2; ++k) {
                launch_step(static_cast<int>(k & 1u));
            }
        } catch (...) {
            cudaStreamEndCapture(stream, &captured);
            if (captured) cudaGraphDestroy(captured);
            launches = before;
            throw;
        }
        launches = before;
        check(cudaStreamEndCapture(stream, &captured), "graph capture");
        const cudaError_t e = cudaGraphInstantiate(&graph, captured, 0);
        cudaGraphDestroy(captured);
        check(e, "graph instantiate");
    }

    void run(uint64_t count) {
        uint64_t left = count;
        if (left >= kGraphSteps2) {
            if (cur != 0) {
                launch_step(cur);
                cur = 1 - cur;
                --left;
            }
            if (!graph) {
                build_graph();
            }
            while (left >= kGraphSteps2) {
                check(cudaGraphLaunch(graph, stream), "graph launch");
                launches += kGraphSteps2;
                left -= kGraphSteps2;
            }
        }
        for (; left > 0; --left) {
            launch_step(cur);
            cur = 1 - cur;
        }
        steps += count;
    }
};

namespace {

orr_lbm2d* handle2_of(orr_lbm2d* h) {
    if (h == nullptr) {
        throw Refusal{ORR_ERR_INVALID, "null solver handle"};
    }
    check(cudaSetDevice(h->device), "cudaSetDevice");
    return h;
}

template <class P> void fill_phys2(P& p, const orr_lbm2d_config& c, bool binary32) {
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
    p.wall_ux[0] = cv(c.bottom.velocity_x);
    p.wall_ux[1] = cv(c.top.velocity_x);
    p.outlet_speed = cv(c.inlet_ux);
    p.inlet_ux = cv(c.inlet_ux);
    p.inlet_uy = cv(c.inlet_uy);
}

void initialize2(orr_lbm2d* h, const double* rho, const double* ux, const double* uy) {
    const auto& c = h->plan.c;
    const std::size_t cells = h->plan.cells;
    double* staged[3] = {nullptr, nullptr, nullptr};
    if (rho != nullptr) {
        double* base = static_cast<double*>(h->f[1]);
        const double* src[3] = {rho, ux, uy};
        for (int k = 0; k < 3; ++k) {
            staged[k] = base + static_cast<std::size_t>(k) * cells;
            check(cudaMemcpyAsync(staged[k], src[k], cells * 8, cudaMemcpyHostToDevice, h->stream),
                  "initial state upload");
        }
    }
    const bool inflow = c.x_boundary == ORR_X_INFLOW_OUTFLOW;
    check(h->ops->init(h->g, h->cls, staged[0], staged[1], staged[2], inflow ? c.inlet_ux : 0.0,
                       inflow ? c.inlet_uy : 0.0, h->f[0], h->stream),
          "init kernel");
    check(cudaMemcpyAsync(h->f[1], h->f[0], d2::Q * cells * h->sbytes, cudaMemcpyDeviceToDevice, h->stream),
          "population copy");
    check(h->ops->history(h->g, h->f[0], h->hist, h->stream), "history kernel");
    h->launches += 2;
    h->cur = 0;
    h->steps = 0;
    check(cudaStreamSynchronize(h->stream), "initialize");
}

void copy_message2(const std::string& text, char* message, size_t capacity) {
    if (message == nullptr || capacity == 0) {
        return;
    }
    const size_t n = std::min(text.size(), capacity - 1);
    std::memcpy(message, text.data(), n);
    message[n] = '\0';
}

} // namespace

extern "C" {

orr_status orr_lbm2d_validate(const orr_lbm2d_config* config, const uint8_t* solid,
                              const orr_solver_options* options, char* message, size_t capacity) {
    if (config == nullptr) {
        copy_message2("null configuration", message, capacity);
        return orr::fail(ORR_ERR_INVALID, "null configuration");
    }
    const int32_t storage = options ? options->storage : ORR_STORAGE_F32;
    const bool high = options ? options->allow_high_mach != 0 : false;
    const std::string problem = orr::problem2d(*config, solid, storage, high);
    copy_message2(problem, message, capacity);
    if (!problem.empty()) {
        return orr::fail(ORR_ERR_INVALID, problem);
    }
    return ORR_OK;
}

orr_status orr_lbm2d_create(const orr_lbm2d_config* config, const uint8_t* solid,
                            const orr_solver_options* options, orr_lbm2d** out) {
    if (out == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output handle");
    }
    *out = nullptr;
    return orr::guarded(nullptr, [&]() -> orr_status {
        if (config == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null configuration"};
        }
        orr_solver_options o{};
        if (options) o = *options;
        if (std::string problem = problem2d(*config, solid, o.storage, o.allow_high_mach != 0);
            !problem.empty()) {
            throw Refusal{ORR_ERR_INVALID, problem};
        }
        if (o.block_x < 0 || o.block_x > 256 || (o.block_x % 32) != 0) {
            throw Refusal{ORR_ERR_INVALID, "lbm2d gpu: block_x must be 0 or a multiple of 32 up to 256"};
        }
        require_device(o.device);
        auto h = std::make_unique<orr_lbm2d>();
        h->device = o.device;
        h->storage = o.storage;
        h->block = o.block_x > 0 ? static_cast<uint32_t>(o.block_x) : kDefaultBlock2;
        h->ops = &ops2_for(o.storage);
        h->sbytes = storage_bytes(o.storage);
        h->abytes = arithmetic_bytes(o.storage);
        h->plan = plan2d(*config, solid);
        const Plan2D& p = h->plan;
        const auto need = memory2d(*config, p.link_cell.size(), o.storage);
        std::size_t free_bytes = 0, total_bytes = 0;
        check(cudaMemGetInfo(&free_bytes, &total_bytes), "cudaMemGetInfo");
        if (!need || *need > free_bytes) {
            throw Refusal{ORR_ERR_MEMORY, "lbm2d gpu: the lattice needs " + mebibytes(need ? *need : 0) +
                                              " of device memory, " + mebibytes(free_bytes) +
                                              " are available; use fewer cells"};
        }
        Geom2D& g = h->g;
        g.nx = static_cast<uint32_t>(config->nx);
        g.ny = static_cast<uint32_t>(config->ny);
        g.cells = p.cells;
        g.x_mode = config->x_boundary;
        g.outlet_mode = config->outlet;
        g.bottom = config->bottom.kind;
        g.top = config->top.kind;
        const bool binary32 = o.storage != ORR_STORAGE_F64;
        g.forced = binary32 ? (static_cast<float>(config->body_force_x) != 0.0f ||
                               static_cast<float>(config->body_force_y) != 0.0f)
                            : (config->body_force_x != 0.0 || config->body_force_y != 0.0);
        fill_phys2(h->phys32, *config, true);
        fill_phys2(h->phys64, *config, false);
        h->smag = config->smagorinsky_enabled != 0 && (binary32 ? h->phys32.smag_c2 > 0.0f : true);
        check(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
        const std::size_t cells = p.cells;
        for (int k = 0; k < 2; ++k) {
            check(cudaMalloc(&h->f[k], d2::Q * cells * h->sbytes), "population buffer");
        }
        check(cudaMalloc(reinterpret_cast<void**>(&h->cls), cells), "node class buffer");
        check(cudaMalloc(reinterpret_cast<void**>(&h->nmask), cells * 4), "bounce-back mask buffer");
        check(cudaMalloc(&h->hist, static_cast<std::size_t>(d2::kOutletSlots) * config->ny * h->abytes),
              "outlet buffer");
        check(cudaMalloc(&h->moments, 3 * cells * h->abytes), "moment buffer");
        check(cudaMalloc(reinterpret_cast<void**>(&h->lcell), std::max<std::size_t>(p.link_cell.size(), 1) * 4),
              "link buffer");
        check(cudaMalloc(reinterpret_cast<void**>(&h->ldir), std::max<std::size_t>(p.link_cell.size(), 1) * 4),
              "link buffer");
        check(cudaMalloc(reinterpret_cast<void**>(&h->acc), 8 * sizeof(double)), "accumulator");
        check(cudaMallocHost(reinterpret_cast<void**>(&h->host_acc), 8 * sizeof(double)), "pinned buffer");
        cudaStream_t s = h->stream;
        check(cudaMemcpyAsync(h->cls, p.cls.data(), cells, cudaMemcpyHostToDevice, s), "class upload");
        check(cudaMemcpyAsync(h->nmask, p.nmask.data(), cells * 4, cudaMemcpyHostToDevice, s), "mask upload");
        if (!p.link_cell.empty()) {
            check(cudaMemcpyAsync(h->lcell, p.link_cell.data(), p.link_cell.size() * 4, cudaMemcpyHostToDevice, s),
                  "link upload");
            check(cudaMemcpyAsync(h->ldir, p.link_dir.data(), p.link_dir.size() * 4, cudaMemcpyHostToDevice, s),
                  "link upload");
        }
        initialize2(h.get(), nullptr, nullptr, nullptr);
        // The step graph is captured here, not inside a later step() call.
        h->build_graph();
        h->plan.cls.clear();
        h->plan.cls.shrink_to_fit();
        *out = h.release();
        return ORR_OK;
    });
}

void orr_lbm2d_destroy(orr_lbm2d* solver) {
    delete solver;
}

const char* orr_lbm2d_last_error(const orr_lbm2d* solver) {
    return solver ? solver->error.c_str() : orr_last_error();
}

orr_status orr_lbm2d_initialize(orr_lbm2d* solver, const double* rho, const double* ux,
                                const double* uy) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm2d* h = handle2_of(solver);
        const bool any = rho || ux || uy, all = rho && ux && uy;
        if (any && !all) {
            throw Refusal{ORR_ERR_INVALID, "lbm2d: initialize needs all three fields or none"};
        }
        initialize2(h, rho, ux, uy);
        return ORR_OK;
    });
}

orr_status orr_lbm2d_step(orr_lbm2d* solver, uint64_t count) {
    orr::Zone zone("lbm_step");
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        handle2_of(solver)->run(count);
        return ORR_OK;
    });
}

orr_status orr_lbm2d_steps(const orr_lbm2d* solver, uint64_t* steps) {
    if (solver == nullptr || steps == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *steps = solver->steps;
    return ORR_OK;
}

orr_status orr_lbm2d_force(orr_lbm2d* solver, double force_moment[3]) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm2d* h = handle2_of(solver);
        if (force_moment == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        const std::size_t links = h->plan.link_cell.size();
        check(h->ops->force(h->g, h->f[h->cur], h->lcell, h->ldir, links, h->acc, h->stream), "force kernel");
        if (links > 0) ++h->launches;
        check(cudaMemcpyAsync(h->host_acc, h->acc, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
              "force read-back");
        check(cudaStreamSynchronize(h->stream), "force read-back");
        std::memcpy(force_moment, h->host_acc, 3 * sizeof(double));
        return ORR_OK;
    });
}

orr_status orr_lbm2d_macroscopic(orr_lbm2d* solver, double* rho, double* ux, double* uy) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm2d* h = handle2_of(solver);
        const std::size_t cells = h->plan.cells;
        check(h->ops->moments(h->g, h->phys(), h->cls, h->f[h->cur], h->moments, h->stream), "moments kernel");
        ++h->launches;
        double* outs[3] = {rho, ux, uy};
        const bool shifted = h->storage != ORR_STORAGE_F64;
        std::vector<float> tmp(shifted ? cells : 0);
        for (int k = 0; k < 3; ++k) {
            if (outs[k] == nullptr) continue;
            const char* plane = static_cast<const char*>(h->moments) + k * cells * h->abytes;
            if (shifted) {
                check(cudaMemcpyAsync(tmp.data(), plane, cells * 4, cudaMemcpyDeviceToHost, h->stream),
                      "moment read-back");
                check(cudaStreamSynchronize(h->stream), "moment read-back");
                for (std::size_t c = 0; c < cells; ++c) {
                    outs[k][c] = static_cast<double>(tmp[c]) + (k == 0 ? 1.0 : 0.0);
                }
            } else {
                check(cudaMemcpyAsync(outs[k], plane, cells * 8, cudaMemcpyDeviceToHost, h->stream),
                      "moment read-back");
                check(cudaStreamSynchronize(h->stream), "moment read-back");
            }
        }
        return ORR_OK;
    });
}

orr_status orr_lbm2d_populations(orr_lbm2d* solver, double* f) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm2d* h = handle2_of(solver);
        if (f == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        const std::size_t cells = h->plan.cells, n = d2::Q * cells;
        if (h->storage == ORR_STORAGE_F64) {
            check(cudaMemcpyAsync(f, h->f[h->cur], n * 8, cudaMemcpyDeviceToHost, h->stream), "population read-back");
            check(cudaStreamSynchronize(h->stream), "population read-back");
            return ORR_OK;
        }
        std::vector<unsigned char> raw(n * h->sbytes);
        check(cudaMemcpyAsync(raw.data(), h->f[h->cur], raw.size(), cudaMemcpyDeviceToHost, h->stream),
              "population read-back");
        check(cudaStreamSynchronize(h->stream), "population read-back");
        for (int i = 0; i < d2::Q; ++i) {
            const double w = d2::w(i);
            for (std::size_t c = 0; c < cells; ++c) {
                const std::size_t k = static_cast<std::size_t>(i) * cells + c;
                double v;
                if (h->storage == ORR_STORAGE_F32) {
                    float x;
                    std::memcpy(&x, raw.data() + 4 * k, 4);
                    v = x;
                } else if (h->storage == ORR_STORAGE_F16) {
                    __half x;
                    std::memcpy(&x, raw.data() + 2 * k, 2);
                    v = static_cast<double>(__half2float(x));
                } else {
                    __nv_bfloat16 x;
                    std::memcpy(&x, raw.data() + 2 * k, 2);
                    v = static_cast<double>(__bfloat162float(x));
                }
                f[k] = v + w;
            }
        }
        return ORR_OK;
    });
}

orr_status orr_lbm2d_mass(orr_lbm2d* solver, double* mass) {
    return orr::guarded(solver ? &solver->error : nullptr, [&]() -> orr_status {
        orr_lbm2d* h = handle2_of(solver);
        if (mass == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "null output"};
        }
        check(h->ops->mass(h->g, h->cls, h->f[h->cur], h->acc + 4, h->stream), "mass kernel");
        ++h->launches;
        check(cudaMemcpyAsync(h->host_acc + 4, h->acc + 4, sizeof(double), cudaMemcpyDeviceToHost, h->stream),
              "mass read-back");
        check(cudaStreamSynchronize(h->stream), "mass read-back");
        double m = h->host_acc[4];
        if (h->storage != ORR_STORAGE_F64) {
            m += static_cast<double>(h->plan.fluid);
        }
        *mass = m;
        return ORR_OK;
    });
}

orr_status orr_lbm2d_link_count(const orr_lbm2d* solver, uint64_t* count) {
    if (solver == nullptr || count == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *count = solver->plan.link_cell.size();
    return ORR_OK;
}

orr_status orr_lbm2d_links(const orr_lbm2d* solver, uint32_t* cell, uint32_t* direction) {
    if (solver == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    const std::size_t n = solver->plan.link_cell.size();
    if (cell) std::memcpy(cell, solver->plan.link_cell.data(), n * 4);
    if (direction) std::memcpy(direction, solver->plan.link_dir.data(), n * 4);
    return ORR_OK;
}

orr_status orr_lbm2d_stream(const orr_lbm2d* solver, void** stream) {
    if (solver == nullptr || stream == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *stream = solver->stream;
    return ORR_OK;
}

orr_status orr_lbm2d_launch_count(const orr_lbm2d* solver, uint64_t* launches) {
    if (solver == nullptr || launches == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null argument");
    }
    *launches = solver->launches;
    return ORR_OK;
}

} // extern "C"
