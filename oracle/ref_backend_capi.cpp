// The reference's own GPU driver, GpuLbm3D (src/aero/lbm3d/lbm3d_gpu.cpp,
// make_gpu_solver), compiled unmodified from the reference sources in place
// by oracle/Makefile into oracle/_ref/libref_backend.so, running its
// lbm_d3q19_* dispatches on the CUDA compute backend of
// orrery_b200/adapter/compute_backend_cuda.cpp: the backend seam
// (IComputeBackend, src/aero/compute/include/orrery/aero/compute/
// compute_backend.h:94-129) end to end on the B200 library.
//
// TEST INFRASTRUCTURE ONLY: the check of the backend seam (the reference's
// "GPU and CPU D3Q19 agree" comparisons, tests/aero/lbm3d/test_lbm3d_gpu.cpp,
// with the CUDA backend in place of the GL one).  The product never links or
// loads it.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "compute_backend_cuda.h"
#include "lbm2d_cuda.h"
#include "orrery/aero/lbm/lbm2d.h"
#include "orrery/aero/lbm/lbm_aero_solver.h"
#include "orrery/aero/lbm3d/lbm3d.h"
#include "orrery/aero/lbm3d/lbm_aero_solver3d.h"
#include "orrery/geom/primitives.h"
#include "orrery_lbm.h"
#include "ref_convert.h"

namespace lbm = orrery::aero::lbm;
namespace compute = orrery::aero::compute;

extern "C" {

// One solve of the reference's D3Q19 GPU driver on the CUDA backend: make_gpu_solver
// on (config, solid, distance), initialise from the four fields (or the
// uniform inlet state when rho is null), `steps` steps, then the read-backs
// whose outputs are not null: populations (19 cells, unshifted), moments
// (density, ux, uy, uz planes of cells each) and force (force, moment).
// meta (4): dispatches the backend served, node-code tables it built, and
// whether it executes kernels; the driver's lattice step count.  0 on
// success; -1 with the error's text.
int ref_backend_solve(const orr_lbm3d_config* config, const uint8_t* solid, const double* distance,
                      const double* rho, const double* ux, const double* uy, const double* uz, uint64_t steps,
                      double* populations, double* moments, double* force, double* meta, char* message,
                      size_t capacity) {
    try {
        compute::CudaComputeBackend backend(0);
        const lbm::Lbm3DConfig c = ref_convert::config3d_of(*config);
        auto made = lbm::make_gpu_solver(backend, c, ref_convert::mask3d_of(*config, solid, distance));
        if (!made) {
            ref_convert::copy_message(made.error(), message, capacity);
            return -1;
        }
        std::unique_ptr<lbm::Lbm3DSolver> solver = std::move(made).value();
        if (rho != nullptr) {
            const std::size_t nx = c.nx, ny = c.ny;
            const auto state = [=](std::size_t x, std::size_t y, std::size_t z) {
                const std::size_t k = x + nx * (y + ny * z);
                return lbm::d3q19::Moments{rho[k], ux[k], uy[k], uz[k]};
            };
            if (auto done = solver->initialize(state); !done) {
                ref_convert::copy_message(done.error(), message, capacity);
                return -1;
            }
        }
        if (auto done = solver->step(steps); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
        const std::size_t cells = c.nx * c.ny * c.nz;
        if (populations != nullptr) {
            auto f = solver->populations();
            if (!f) {
                ref_convert::copy_message(f.error(), message, capacity);
                return -1;
            }
            std::memcpy(populations, f.value().data(), f.value().size() * sizeof(double));
        }
        if (moments != nullptr) {
            auto m = solver->macroscopic();
            if (!m) {
                ref_convert::copy_message(m.error(), message, capacity);
                return -1;
            }
            const lbm::MacroFields3D& v = m.value();
            std::memcpy(moments, v.density.data(), cells * sizeof(double));
            std::memcpy(moments + cells, v.velocity_x.data(), cells * sizeof(double));
            std::memcpy(moments + 2 * cells, v.velocity_y.data(), cells * sizeof(double));
            std::memcpy(moments + 3 * cells, v.velocity_z.data(), cells * sizeof(double));
        }
        if (force != nullptr) {
            auto f = solver->force();
            if (!f) {
                ref_convert::copy_message(f.error(), message, capacity);
                return -1;
            }
            for (int k = 0; k < 3; ++k) {
                force[k] = f.value().force[k];
                force[3 + k] = f.value().moment[k];
            }
        }
        if (meta != nullptr) {
            meta[0] = static_cast<double>(backend.dispatches());
            meta[1] = static_cast<double>(backend.tables_built());
            meta[2] = backend.info().executes_kernels ? 1.0 : 0.0;
            meta[3] = static_cast<double>(solver->steps());
        }
        solver.reset();
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

namespace {

// Initial fields (or none), `steps` steps and the read-backs of one D2Q9
// solver: populations (9 cells, unshifted), moments (density, ux, uy planes)
// and force (x, y, moment about the origin), whichever outputs are not null.
int run2d(lbm::Lbm2DSolver& solver, const lbm::Lbm2DConfig& c, const double* rho, const double* ux,
          const double* uy, uint64_t steps, double* populations, double* moments, double* force, char* message,
          size_t capacity) {
    if (rho != nullptr) {
        const std::size_t nx = c.nx;
        const auto state = [=](std::size_t x, std::size_t y) {
            const std::size_t k = x + nx * y;
            return lbm::d2q9::Moments{rho[k], ux[k], uy[k]};
        };
        if (auto done = solver.initialize(state); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
    }
    if (auto done = solver.step(steps); !done) {
        ref_convert::copy_message(done.error(), message, capacity);
        return -1;
    }
    const std::size_t cells = c.nx * c.ny;
    if (populations != nullptr) {
        auto f = solver.populations();
        if (!f) {
            ref_convert::copy_message(f.error(), message, capacity);
            return -1;
        }
        std::memcpy(populations, f.value().data(), f.value().size() * sizeof(double));
    }
    if (moments != nullptr) {
        auto m = solver.macroscopic();
        if (!m) {
            ref_convert::copy_message(m.error(), message, capacity);
            return -1;
        }
        const lbm::MacroFields2D& v = m.value();
        std::memcpy(moments, v.density.data(), cells * sizeof(double));
        std::memcpy(moments + cells, v.velocity_x.data(), cells * sizeof(double));
        std::memcpy(moments + 2 * cells, v.velocity_y.data(), cells * sizeof(double));
    }
    if (force != nullptr) {
        auto f = solver.force();
        if (!f) {
            ref_convert::copy_message(f.error(), message, capacity);
            return -1;
        }
        force[0] = f.value().x;
        force[1] = f.value().y;
        force[2] = f.value().moment;
    }
    return 0;
}

lbm::SolidMask2D mask2d_of(const lbm::Lbm2DConfig& c, const uint8_t* solid) {
    lbm::SolidMask2D mask;
    mask.nx = c.nx;
    mask.ny = c.ny;
    mask.solid.assign(solid, solid + c.nx * c.ny);
    return mask;
}

} // namespace

// The same for the reference's D2Q9 driver, GpuLbm2D (src/aero/lbm/
// lbm2d_gpu.cpp, its make_gpu_solver), on the CUDA backend: initial fields
// (rho, ux, uy) or the uniform inlet state; the outputs of run2d.  meta (4):
// dispatches, solid-flag tables built, executes kernels, steps.
int ref_backend_solve2d(const orr_lbm2d_config* config, const uint8_t* solid, const double* rho,
                        const double* ux, const double* uy, uint64_t steps, double* populations, double* moments,
                        double* force, double* meta, char* message, size_t capacity) {
    try {
        compute::CudaComputeBackend backend(0);
        const lbm::Lbm2DConfig c = ref_convert::config2d_of(*config);
        auto made = lbm::make_gpu_solver(backend, c, mask2d_of(c, solid));
        if (!made) {
            ref_convert::copy_message(made.error(), message, capacity);
            return -1;
        }
        std::unique_ptr<lbm::Lbm2DSolver> solver = std::move(made).value();
        if (run2d(*solver, c, rho, ux, uy, steps, populations, moments, force, message, capacity) != 0) {
            return -1;
        }
        if (meta != nullptr) {
            meta[0] = static_cast<double>(backend.dispatches());
            meta[1] = static_cast<double>(backend.tables_built());
            meta[2] = backend.info().executes_kernels ? 1.0 : 0.0;
            meta[3] = static_cast<double>(solver->steps());
        }
        solver.reset();
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The same through the Lbm2DSolver seam: make_cuda_solver of
// orrery_b200/adapter/lbm2d_cuda.cpp (binary32 storage).  meta (1): steps.
int ref_cuda2d_solve(const orr_lbm2d_config* config, const uint8_t* solid, const double* rho, const double* ux,
                     const double* uy, uint64_t steps, double* populations, double* moments, double* force,
                     double* meta, char* message, size_t capacity) {
    try {
        const lbm::Lbm2DConfig c = ref_convert::config2d_of(*config);
        auto made = lbm::make_cuda_solver(c, mask2d_of(c, solid));
        if (!made) {
            ref_convert::copy_message(made.error(), message, capacity);
            return -1;
        }
        std::unique_ptr<lbm::Lbm2DSolver> solver = std::move(made).value();
        if (run2d(*solver, c, rho, ux, uy, steps, populations, moments, force, message, capacity) != 0) {
            return -1;
        }
        if (meta != nullptr) {
            meta[0] = static_cast<double>(solver->steps());
        }
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The reference's 2D adapter, LbmAeroSolver2D (src/aero/lbm/lbm_aero_solver.cpp),
// on its CPU solver and on GpuLbm2D over the CUDA backend: the case of
// "The IAeroSolver adapter runs on the GPU backend" (tests/aero/lbm/
// test_lbm_gpu.cpp:278-311; a circle of 96 points, radius 0.01, speed 0.1,
// density 1000, Re 100, 10 cells per length, u_lat 0.05, duration 10, 2000
// steps per call).  out (6): Cd CPU, Cd GPU, iterations CPU, iterations GPU,
// surface Cp samples CPU, GPU.  0 on success; -1 with the error's text.
int ref_backend_adapter2d(double* out, char* message, size_t capacity) {
    try {
        namespace aero = orrery::aero;
        compute::CudaComputeBackend backend(0);
        aero::AeroGeometry geometry;
        for (int k = 0; k < 96; ++k) {
            const double a = 2.0 * std::numbers::pi * static_cast<double>(k) / 96.0;
            geometry.section.push_back({0.01 * std::cos(a), 0.01 * std::sin(a)});
        }
        geometry.reference.length = 0.02;
        geometry.reference.area = 0.02;
        aero::FlowConditions conditions;
        conditions.speed = 0.1;
        conditions.density = 1000.0;
        conditions.viscosity = 1000.0 * 0.1 * 0.02 / 100.0;
        lbm::LbmSolverOptions options;
        options.resolution = lbm::LatticeResolution{10.0, 0.05};
        options.duration = 10.0;
        options.steps_per_call = 2000;
        lbm::LbmAeroSolver2D cpu(options);
        options.backend = &backend;
        lbm::LbmAeroSolver2D gpu(options);
        cpu.setup(geometry, conditions);
        gpu.setup(geometry, conditions);
        while (!cpu.step()) {
        }
        while (!gpu.step()) {
        }
        out[0] = cpu.result().cd;
        out[1] = gpu.result().cd;
        out[2] = static_cast<double>(cpu.result().iterations);
        out[3] = static_cast<double>(gpu.result().iterations);
        out[4] = static_cast<double>(cpu.result().surface.cp.size());
        out[5] = static_cast<double>(gpu.result().surface.cp.size());
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The reference's 3D adapter, LbmAeroSolver3D (src/aero/lbm3d/
// lbm_aero_solver3d.cpp), unmodified, on its CPU solver and on the reference's
// GPU driver over the CUDA backend (LbmSolver3DOptions::backend): the case of
// "The 3D IAeroSolver adapter runs on the GPU backend" (tests/aero/lbm3d/
// test_lbm3d_gpu.cpp:291-324; a 2 cm sphere of 32 segments, speed 0.1,
// density 1000, Re 50, 10 cells per length, u_lat 0.05, upstream 2,
// downstream 4, width 4, duration 5, window 2, 1000 steps per call).  out
// (4): Cd CPU, Cd GPU, iterations CPU, iterations GPU.
int ref_backend_adapter3d(double* out, char* message, size_t capacity) {
    try {
        namespace aero = orrery::aero;
        namespace geom = orrery::geom;
        compute::CudaComputeBackend backend(0);
        aero::AeroGeometry geometry;
        geometry.mesh = geom::sphere_profile(0.01).mesh({32, 0.1});
        geometry.reference.length = 0.02;
        geometry.reference.area = 0.25 * std::numbers::pi * 0.02 * 0.02;
        aero::FlowConditions conditions;
        conditions.speed = 0.1;
        conditions.density = 1000.0;
        conditions.viscosity = 1000.0 * 0.1 * 0.02 / 50.0;
        lbm::LbmSolver3DOptions options;
        options.resolution = lbm::LatticeResolution{10.0, 0.05};
        options.upstream = 2.0;
        options.downstream = 4.0;
        options.width = 4.0;
        options.duration = 5.0;
        options.average_window = 2.0;
        options.steps_per_call = 1000;
        lbm::LbmAeroSolver3D cpu(options);
        cpu.setup(geometry, conditions);
        while (!cpu.step()) {
        }
        options.backend = &backend;
        lbm::LbmAeroSolver3D gpu(options);
        gpu.setup(geometry, conditions);
        while (!gpu.step()) {
        }
        out[0] = cpu.result().cd;
        out[1] = gpu.result().cd;
        out[2] = static_cast<double>(cpu.result().iterations);
        out[3] = static_cast<double>(gpu.result().iterations);
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The rate of the reference's own benchmark (tests/bench/aero/
// bench_lbm_gpu.cpp: gpu_steps_per_second) with its GPU driver on the CUDA
// backend: make_gpu_solver, `warmup` steps, a drain, then `count` steps
// timed by the host clock up to the drain after them.  seconds: the timed
// span.  The 3D and 2D drivers.
int ref_backend_rate3d(const orr_lbm3d_config* config, const uint8_t* solid, uint64_t warmup, uint64_t count,
                       double* seconds, char* message, size_t capacity) {
    try {
        compute::CudaComputeBackend backend(0);
        const lbm::Lbm3DConfig c = ref_convert::config3d_of(*config);
        auto made = lbm::make_gpu_solver(backend, c, ref_convert::mask3d_of(*config, solid, nullptr));
        if (!made) {
            ref_convert::copy_message(made.error(), message, capacity);
            return -1;
        }
        auto solver = std::move(made).value();
        if (auto done = solver->step(warmup); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
        backend.finish();
        const auto t0 = std::chrono::steady_clock::now();
        if (auto done = solver->step(count); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
        backend.finish();
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

int ref_backend_rate2d(const orr_lbm2d_config* config, const uint8_t* solid, uint64_t warmup, uint64_t count,
                       double* seconds, char* message, size_t capacity) {
    try {
        compute::CudaComputeBackend backend(0);
        const lbm::Lbm2DConfig c = ref_convert::config2d_of(*config);
        auto made = lbm::make_gpu_solver(backend, c, mask2d_of(c, solid));
        if (!made) {
            ref_convert::copy_message(made.error(), message, capacity);
            return -1;
        }
        auto solver = std::move(made).value();
        if (auto done = solver->step(warmup); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
        backend.finish();
        const auto t0 = std::chrono::steady_clock::now();
        if (auto done = solver->step(count); !done) {
            ref_convert::copy_message(done.error(), message, capacity);
            return -1;
        }
        backend.finish();
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    } catch (const std::exception& e) {
        ref_convert::copy_message(e.what(), message, capacity);
        return -1;
    }
}

// The backend's refusals through the seam, for the tests of its contract:
// an unknown kernel, an empty dispatch, a uniform of the wrong type, an
// unknown buffer, an upload outside a buffer.  Returns how many of the five
// were refused (each must be), with the last refusal's text.
int ref_backend_refusals(char* message, size_t capacity) {
    compute::CudaComputeBackend backend(0);
    int refused = 0;
    std::string last;
    const auto note = [&](const compute::Status& s) {
        if (!s) {
            ++refused;
            last = s.error();
        }
    };
    auto made = backend.create_buffer(64);
    if (!made) {
        ref_convert::copy_message(made.error(), message, capacity);
        return -1;
    }
    const compute::BufferId id = made.value();
    note(backend.dispatch({"lbm_d3q19_missing", {1, 1, 1}, {}, {}}));
    note(backend.dispatch({"lbm_d3q19_step", {0, 1, 1}, {}, {}}));
    const compute::Uniform wrong{"u_tau", std::uint32_t{1}};
    note(backend.dispatch({"lbm_d3q19_step", {1, 1, 1}, std::span<const compute::Uniform>(&wrong, 1), {}}));
    const compute::BufferBinding unknown{0, compute::BufferId{9999}};
    note(backend.dispatch({"lbm_d3q19_step", {1, 1, 1}, {}, std::span<const compute::BufferBinding>(&unknown, 1)}));
    std::vector<std::byte> bytes(65);
    note(backend.upload(id, 0, bytes));
    backend.release_buffer(id);
    ref_convert::copy_message(last, message, capacity);
    return refused;
}

} // extern "C"
