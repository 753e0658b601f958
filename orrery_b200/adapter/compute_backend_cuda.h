// IComputeBackend on the B200 library: the file a maintainer adds beside the
// reference's OpenGL backend (src/render/compute/gl_compute_backend.cpp) so
// that the reference's GPU driver, GpuLbm3D (src/aero/lbm3d/lbm3d_gpu.cpp,
// make_gpu_solver), and anything else written against the backend seam
// (src/aero/compute/include/orrery/aero/compute/compute_backend.h:94-129) run
// their D3Q19 kernels on CUDA.  Compiled against the reference's headers and
// linked with orrery_b200/_native/liborrery_lbm.so and the CUDA runtime.
//
// Buffers are device allocations (zero-initialised, each with the slack the
// library's step reads past a lattice's edges); upload and readback are
// ordered after every earlier dispatch on the backend's one stream, so
// barrier() has nothing to do.  dispatch() serves the three kernels the
// D3Q19 driver binds (lbm_d3q19_step, lbm_d3q19_moments, lbm_d3q19_force)
// through the library's orr_gl3d_* entry points, and the three of the D2Q9
// driver, GpuLbm2D (src/aero/lbm/lbm2d_gpu.cpp: lbm_d2q9_step, _moments,
// _force), through orr_gl2d_*, with the drivers' binding points and
// uniforms: the tables the library derives from a node-code (or solid-flag)
// buffer are built at the first dispatch that binds it and kept until that
// buffer is written again or released.  Like the reference's backends, one
// thread uses a backend.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <string_view>

#include "orrery/aero/compute/compute_backend.h"
#include "orrery_lbm.h"

namespace orrery::aero::compute {

class CudaComputeBackend final : public IComputeBackend {
public:
    explicit CudaComputeBackend(int device = 0);
    ~CudaComputeBackend() override;

    [[nodiscard]] ComputeBackendInfo info() const override;
    [[nodiscard]] bool has_kernel(std::string_view name) const override;
    // The free device memory; CUDA has no binding limit below it.
    [[nodiscard]] DeviceMemory memory() const override;

    [[nodiscard]] core::Result<BufferId, std::string> create_buffer(std::size_t bytes) override;
    void release_buffer(BufferId buffer) noexcept override;
    [[nodiscard]] std::size_t buffer_size(BufferId buffer) const noexcept override;
    [[nodiscard]] Status upload(BufferId buffer, std::size_t offset, std::span<const std::byte> bytes) override;
    [[nodiscard]] Status readback(BufferId buffer, std::size_t offset, std::span<std::byte> bytes) override;
    [[nodiscard]] Status dispatch(const DispatchCommand& command) override;
    void barrier() override {}
    // Waits until every upload, dispatch and read-back so far has completed
    // (the GL backend's finish(), which the reference's benchmarks call
    // around their timed steps).
    void finish();

    // Dispatches served so far (by all three kernels), and node-code tables
    // built: for tests of the caching.
    [[nodiscard]] std::uint64_t dispatches() const noexcept { return dispatches_; }
    [[nodiscard]] std::uint64_t tables_built() const noexcept { return tables_built_; }

private:
    struct Buffer {
        void* base = nullptr;      // the allocation
        std::byte* data = nullptr; // base + slack
        std::size_t bytes = 0;
    };
    struct Tables {
        orr_gl3d* handle = nullptr;    // D3Q19: from a node-code buffer
        orr_gl3d_params lattice{};
        std::size_t wall_values = 0;   // wall fractions the node codes' slots address
        orr_gl2d* handle2 = nullptr;   // D2Q9: from a solid-flag buffer
        orr_gl2d_params lattice2{};
    };

    [[nodiscard]] Status tables_for(BufferId classes, const orr_gl3d_params& params, Tables*& out);
    [[nodiscard]] Status tables2_for(BufferId solid, const orr_gl2d_params& params, Tables*& out);
    [[nodiscard]] Status dispatch2(const DispatchCommand& command);
    void drop_tables(BufferId buffer) noexcept;

    int device_ = 0;
    void* stream_ = nullptr;       // cudaStream_t
    std::size_t slack_ = 0;
    std::uint32_t next_id_ = 1;
    std::map<std::uint32_t, Buffer> buffers_;
    std::map<std::uint32_t, Tables> tables_; // by node-code buffer
    std::uint64_t dispatches_ = 0;
    std::uint64_t tables_built_ = 0;
};

} // namespace orrery::aero::compute
