// State of a D3Q19 device solver (the handle behind orr_lbm3d_*), shared by
// the solver's entry points and the batch that steps several solvers with
// one persistent launch.
//
// Device layout (one allocation per table):
//   populations   two buffers of 19 * cells storage values, structure of
//                 arrays f[i * cells + x + nx (y + ny z)]; ping-pong (A-B),
//                 with kPopPad elements of slack on both sides
//   classes       one byte per node (solid / bulk / face / boundary), slack after
//   masks         per node, the directions that bounce back (solid source)
//   slots         per node, the wall-table slot (interpolated wall only)
//   wall table    19 fractions per slot (interpolated wall)
//   links         cell, direction and fraction of every boundary link
//   moments       4 planes (rho or rho - 1, ux, uy, uz) for read-back
//   history       5 * ny * nz convective-outlet values
//   small         inlet velocity (3), force/moment (6) and mass accumulators,
//                 the persistent step's status word
//   table         the lattice-table entry of the persistent step
// Steps run as CUDA graphs of kGraphSteps steps, one kernel launch each:
// the persistent staged step (staged3d.cuh) when the lattice qualifies, else
// the row-tile step.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "common.h"
#include "kernels3d.cuh"
#include "lattice.h"
#include "lattice_table.cuh"
#include "ops3d.h"
#include "plan.h"

struct orr_batch3d;
struct orr_lbm3d;

// Drops a member from its batch (orr_lbm3d_destroy of a member).
void orr_batch3d_forget(orr_batch3d* batch, orr_lbm3d* solver) noexcept;

namespace orr {
// Initialises the solver at rest (rho 1, u 0 at every node) with a zero inlet
// velocity: the start of a ramped solve (the reference adapter's gradual
// start initialises the same state, lbm_aero_solver3d.cpp:320-329).
void initialize_at_rest(orr_lbm3d* h);
} // namespace orr

namespace orr {

constexpr uint32_t kGraphSteps = 16; // even: a graph returns to the buffer it started on
constexpr uint32_t kDefaultBlock = 128;
constexpr std::size_t kStatusOffset = 128; // bytes into the small buffer

template <class T> T* device_alloc(std::size_t count, const char* what) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<std::size_t>(count, 1) * sizeof(T)), what);
    return static_cast<T*>(p);
}

inline const Ops3D& ops_for(int32_t storage) {
    switch (storage) {
        case ORR_STORAGE_F16:
            return ops3d_f16();
        case ORR_STORAGE_BF16:
            return ops3d_bf16();
        case ORR_STORAGE_F64:
            return ops3d_f64();
        default:
            return ops3d_f32();
    }
}

// Nodes per consumer thread of a staged span when the caller leaves it open.
inline uint32_t default_npt(int32_t storage) {
    (void)storage;
    return 1u;
}

inline float to_f32(double v) {
    return static_cast<float>(v);
}

} // namespace orr

// (A private header of this library: the handle is a global C type.)
using namespace orr;

struct orr_lbm3d {
    // Set while a batch steps this solver (its own step() is refused then).
    orr_batch3d* batch = nullptr;
    // Bumped by initialize(): a batch rebuilds its table when it changes.
    uint64_t epoch = 0;

    Plan3D plan;
    int32_t storage = ORR_STORAGE_F32;
    bool allow_high_mach = false;
    int device = 0;
    uint32_t block = kDefaultBlock;
    uint32_t row_npt = 1;  // nodes per thread of the row-tile step (2: the pair step)
    const Ops3D* ops = nullptr;
    Geom3D g{};
    Phys3D<float> phys32{};
    Phys3D<double> phys64{};
    bool smag = false;
    std::size_t sbytes = 4;
    std::size_t abytes = 4;

    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;

    void* fbase[2] = {nullptr, nullptr}; // allocations; f[k] = fbase[k] + kPopPad values
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    bool persistent = false;  // the staged persistent step runs the steps
    bool tiled = false;       // the tiled step runs the steps (shape as the staged one's)
    TileMaps tmaps{};
    TileGrid tgrid{};
    uint32_t tile_rows = 8;
    StagedShape shape{};
    ItemCounts items{};
    void* table = nullptr;
    alignas(16) unsigned char host_table[kTableBytes] = {}; // host copy of the table entry
    uint8_t* cls = nullptr;
    uint32_t* nmask = nullptr;
    int32_t* nslot = nullptr;
    void* wall_q = nullptr;
    void* hist = nullptr;
    void* moments = nullptr;
    uint32_t* lcell = nullptr;
    uint32_t* ldir = nullptr;
    double* lq = nullptr;
    void* small = nullptr;   // inlet (3 x arithmetic) at 0, accumulators at 64
    double* host_small = nullptr; // pinned: inlet staging + results

    uint64_t steps = 0;
    uint64_t launches = 0;
    double inlet[3] = {0.0, 0.0, 0.0};
    std::string error;

    const void* phys() const {
        return storage == ORR_STORAGE_F64 ? static_cast<const void*>(&phys64)
                                          : static_cast<const void*>(&phys32);
    }
    void* inlet_dev() const { return small; }
    uint32_t* status() const {
        return reinterpret_cast<uint32_t*>(static_cast<char*>(small) + kStatusOffset);
    }
    double* acc() const { return reinterpret_cast<double*>(static_cast<char*>(small) + 64); }

    StepBuffers3D buffers() const {
        StepBuffers3D b{};
        b.cls = cls;
        b.nmask = nmask;
        b.nslot = nslot;
        b.wall_q = wall_q;
        b.hist = hist;
        b.inlet = small;
        return b;
    }

    ~orr_lbm3d() { release(); }

    void release() noexcept {
        if (device >= 0) {
            cudaSetDevice(device);
        }
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : {fbase[0], fbase[1], static_cast<void*>(cls), static_cast<void*>(nmask),
                        static_cast<void*>(nslot), wall_q, hist, moments,
                        static_cast<void*>(lcell), static_cast<void*>(ldir),
                        static_cast<void*>(lq), small, table}) {
            if (p) cudaFree(p);
        }
        if (host_small) cudaFreeHost(host_small);
        if (stream) cudaStreamDestroy(stream);
        graph = nullptr;
        fbase[0] = fbase[1] = nullptr;
        f[0] = f[1] = nullptr;
        table = nullptr;
        cls = nullptr;
        nmask = nullptr;
        nslot = nullptr;
        wall_q = hist = moments = small = nullptr;
        lcell = ldir = nullptr;
        lq = nullptr;
        host_small = nullptr;
        stream = nullptr;
    }

    // Uploads the imposed inlet velocity in the arithmetic type.
    void upload_inlet(const double v[3]) {
        inlet[0] = v[0];
        inlet[1] = v[1];
        inlet[2] = v[2];
        check(cudaStreamSynchronize(stream), "inlet upload");
        if (storage == ORR_STORAGE_F64) {
            std::memcpy(host_small, v, 3 * sizeof(double));
        } else {
            float* h = reinterpret_cast<float*>(host_small);
            h[0] = to_f32(v[0]);
            h[1] = to_f32(v[1]);
            h[2] = to_f32(v[2]);
        }
        check(cudaMemcpyAsync(small, host_small, 3 * abytes, cudaMemcpyHostToDevice, stream),
              "inlet upload");
        check(cudaStreamSynchronize(stream), "inlet upload");
    }

    // One step src -> dst on `stream` (one kernel launch).
    void launch_step(int from) {
        if (tiled) {
            check(ops->tiled(host_table, tmaps, tgrid, static_cast<uint32_t>(from), shape.stages, smag, tile_rows,
                             shape.block, shape.grid, status(), stream),
                  "step kernel");
        } else if (persistent) {
            check(ops->staged(host_table, table, 1, items.staged, items.direct, static_cast<uint32_t>(from),
                              shape.stages, smag, shape.block, shape.npt, shape.grid, status(), stream),
                  "step kernel");
        } else {
            check(ops->step(g, phys(), f[from], f[1 - from], buffers(), smag, block, row_npt, stream),
                  "step kernel");
        }
        ++launches;
    }

    // The persistent step's status word (a wait that timed out makes the
    // populations invalid until the next initialize).
    void check_status() {
        if (!persistent && !tiled) {
            return;
        }
        uint32_t* word = reinterpret_cast<uint32_t*>(host_small + 30);
        check(cudaMemcpyAsync(word, status(), sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
              "status read-back");
        check(cudaStreamSynchronize(stream), "status read-back");
        raise_status(*word);
    }
    static void raise_status(uint32_t word) {
        if (word != 0u) {
            throw Refusal{ORR_ERR_TIMEOUT, "lbm3d gpu: a staged step gave up waiting for its row copies; "
                                        "the populations are invalid until initialize"};
        }
    }

    // Builds the lattice-table entry of the persistent step.
    template <class A> void upload_table(const Phys3D<A>& p) {
        Lattice3D<A> L{};
        L.g = g;
        L.p = p;
        L.b = buffers();
        L.f[0] = f[0];
        L.f[1] = f[1];
        L.parity = 0;
        L.staged = stageable(g) ? 1u : 0u;
        items = number_items(&L, 1, shape.block, shape.npt);
        static_assert(sizeof(Lattice3D<A>) <= kTableBytes, "table entry");
        std::memcpy(host_table, &L, sizeof(L));
        check(cudaMemcpyAsync(table, &L, sizeof(L), cudaMemcpyHostToDevice, stream), "table upload");
        check(cudaStreamSynchronize(stream), "table upload");
    }

    void build_graph() {
        cudaGraph_t captured = nullptr;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        const uint64_t before = launches;
        try {
            for (uint32_t k = 0; k < kGraphSteps; ++k) {
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
        if (left >= kGraphSteps) {
            if (cur != 0) {
                launch_step(cur);
                cur = 1 - cur;
                --left;
            }
            if (!graph) {
                build_graph();
            }
            while (left >= kGraphSteps) {
                check(cudaGraphLaunch(graph, stream), "graph launch");
                launches += kGraphSteps;
                left -= kGraphSteps;
            }
        }
        for (; left > 0; --left) {
            launch_step(cur);
            cur = 1 - cur;
        }
        steps += count;
    }
};

