// IComputeBackend on the B200 library (see compute_backend_cuda.h).
#include "compute_backend_cuda.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <optional>
#include <variant>
#include <vector>

namespace orrery::aero::compute {

namespace {

// Binding points of the driver's kernels (lbm3d_gpu.cpp:37-44).
constexpr std::uint32_t kBindSource = 0;
constexpr std::uint32_t kBindClass = 1;
constexpr std::uint32_t kBindDestination = 2;
constexpr std::uint32_t kBindMoments = 3;
constexpr std::uint32_t kBindLinks = 4;
constexpr std::uint32_t kBindLinkForce = 5;
constexpr std::uint32_t kBindOutlet = 6;
constexpr std::uint32_t kBindWall = 7;

constexpr std::string_view kStep = "lbm_d3q19_step";
constexpr std::string_view kMoments = "lbm_d3q19_moments";
constexpr std::string_view kForce = "lbm_d3q19_force";
// The D2Q9 driver's kernels (lbm2d_gpu.cpp; binding points 0..6 as above,
// binding 1 the solid flags).
constexpr std::string_view kStep2 = "lbm_d2q9_step";
constexpr std::string_view kMoments2 = "lbm_d2q9_moments";
constexpr std::string_view kForce2 = "lbm_d2q9_force";

Status failure(std::string text) {
    return core::failure(std::move(text));
}

std::string cuda_text(const char* what, cudaError_t e) {
    return std::string("cuda backend: ") + what + ": " + cudaGetErrorString(e);
}

// The driver's uniforms (lbm3d_gpu.cpp:158-189) into the library's record:
// integer uniforms unchanged, binary32 uniforms rounded once; a known name
// of the wrong type is an error, unknown names are ignored.
std::optional<std::string> read_uniforms(std::span<const Uniform> uniforms, orr_gl3d_params& p) {
    struct U32 {
        std::string_view name;
        std::uint32_t* at;
    };
    struct F32 {
        std::string_view name;
        float* at;
    };
    const std::array<U32, 15> u32{{{"u_nx", &p.nx},
                                   {"u_ny", &p.ny},
                                   {"u_nz", &p.nz},
                                   {"u_x_mode", &p.x_mode},
                                   {"u_y_low_kind", &p.wall_kind[0]},
                                   {"u_y_high_kind", &p.wall_kind[1]},
                                   {"u_z_low_kind", &p.wall_kind[2]},
                                   {"u_z_high_kind", &p.wall_kind[3]},
                                   {"u_link_count", &p.link_count},
                                   {"u_outlet_mode", &p.outlet_mode},
                                   {"u_sponge_inlet", &p.sponge_inlet},
                                   {"u_sponge_outlet", &p.sponge_outlet},
                                   {"u_sponge_sides", &p.sponge_sides},
                                   {"u_link_row", nullptr},
                                   {"", nullptr}}};
    const std::array<F32, 15> f32{{{"u_y_low_ux", &p.wall_ux[0]},
                                   {"u_y_high_ux", &p.wall_ux[1]},
                                   {"u_z_low_ux", &p.wall_ux[2]},
                                   {"u_z_high_ux", &p.wall_ux[3]},
                                   {"u_inlet_ux", &p.inlet[0]},
                                   {"u_inlet_uy", &p.inlet[1]},
                                   {"u_inlet_uz", &p.inlet[2]},
                                   {"u_tau", &p.tau},
                                   {"u_smagorinsky_c2", &p.smagorinsky_c2},
                                   {"u_force_x", &p.force[0]},
                                   {"u_force_y", &p.force[1]},
                                   {"u_force_z", &p.force[2]},
                                   {"u_outlet_speed", &p.outlet_speed},
                                   {"u_sponge_strength", &p.sponge_strength},
                                   {"", nullptr}}};
    for (const Uniform& u : uniforms) {
        bool known = false;
        for (const U32& k : u32) {
            if (!k.name.empty() && k.name == u.name) {
                known = true;
                if (!std::holds_alternative<std::uint32_t>(u.value)) {
                    return "cuda backend: uniform " + std::string(u.name) + " must be an unsigned integer";
                }
                if (k.at) *k.at = std::get<std::uint32_t>(u.value);
            }
        }
        for (const F32& k : f32) {
            if (!k.name.empty() && k.name == u.name) {
                known = true;
                if (!std::holds_alternative<Float32Uniform>(u.value)) {
                    return "cuda backend: uniform " + std::string(u.name) + " must be a binary32 value";
                }
                *k.at = static_cast<float>(std::get<Float32Uniform>(u.value).value);
            }
        }
        (void)known; // names no kernel here declares are ignored, as a GL program ignores them
    }
    return std::nullopt;
}

// The D2Q9 driver's uniforms (lbm2d_gpu.cpp:104-124), by the same rules.
std::optional<std::string> read_uniforms2(std::span<const Uniform> uniforms, orr_gl2d_params& p) {
    struct U32 {
        std::string_view name;
        std::uint32_t* at;
    };
    struct F32 {
        std::string_view name;
        float* at;
    };
    const std::array<U32, 7> u32{{{"u_nx", &p.nx},
                                  {"u_ny", &p.ny},
                                  {"u_x_mode", &p.x_mode},
                                  {"u_bottom_kind", &p.bottom_kind},
                                  {"u_top_kind", &p.top_kind},
                                  {"u_link_count", &p.link_count},
                                  {"u_outlet_mode", &p.outlet_mode}}};
    const std::array<F32, 10> f32{{{"u_bottom_ux", &p.bottom_ux},
                                   {"u_top_ux", &p.top_ux},
                                   {"u_inlet_ux", &p.inlet[0]},
                                   {"u_inlet_uy", &p.inlet[1]},
                                   {"u_tau", &p.tau},
                                   {"u_smagorinsky_c2", &p.smagorinsky_c2},
                                   {"u_force_x", &p.force[0]},
                                   {"u_force_y", &p.force[1]},
                                   {"u_outlet_speed", &p.outlet_speed},
                                   {"", nullptr}}};
    for (const Uniform& u : uniforms) {
        for (const U32& k : u32) {
            if (k.name == u.name) {
                if (!std::holds_alternative<std::uint32_t>(u.value)) {
                    return "cuda backend: uniform " + std::string(u.name) + " must be an unsigned integer";
                }
                *k.at = std::get<std::uint32_t>(u.value);
            }
        }
        for (const F32& k : f32) {
            if (!k.name.empty() && k.name == u.name) {
                if (!std::holds_alternative<Float32Uniform>(u.value)) {
                    return "cuda backend: uniform " + std::string(u.name) + " must be a binary32 value";
                }
                *k.at = static_cast<float>(std::get<Float32Uniform>(u.value).value);
            }
        }
    }
    return std::nullopt;
}

} // namespace

CudaComputeBackend::CudaComputeBackend(int device) : device_(device) {
    slack_ = static_cast<std::size_t>(orr_gl3d_buffer_slack());
    cudaSetDevice(device_);
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess) {
        stream_ = s;
    }
}

CudaComputeBackend::~CudaComputeBackend() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(static_cast<cudaStream_t>(stream_));
    for (auto& [id, t] : tables_) {
        orr_gl3d_destroy(t.handle);
        orr_gl2d_destroy(t.handle2);
    }
    for (auto& [id, b] : buffers_) cudaFree(b.base);
    if (stream_) cudaStreamDestroy(static_cast<cudaStream_t>(stream_));
}

ComputeBackendInfo CudaComputeBackend::info() const {
    cudaDeviceProp prop{};
    std::string name = "CUDA device " + std::to_string(device_);
    if (cudaGetDeviceProperties(&prop, device_) == cudaSuccess) {
        name = prop.name;
    }
    return ComputeBackendInfo{"cuda", name, stream_ != nullptr};
}

void CudaComputeBackend::finish() {
    if (stream_ != nullptr) {
        cudaSetDevice(device_);
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream_));
    }
}

bool CudaComputeBackend::has_kernel(std::string_view name) const {
    return name == kStep || name == kMoments || name == kForce || name == kStep2 || name == kMoments2 ||
           name == kForce2;
}

DeviceMemory CudaComputeBackend::memory() const {
    DeviceMemory m;
    std::size_t free = 0, total = 0;
    cudaSetDevice(device_);
    if (cudaMemGetInfo(&free, &total) == cudaSuccess) {
        m.available_bytes = free;
    }
    return m;
}

core::Result<BufferId, std::string> CudaComputeBackend::create_buffer(std::size_t bytes) {
    if (bytes == 0) {
        return core::failure(std::string("cuda backend: empty buffer"));
    }
    if (stream_ == nullptr) {
        return core::failure(std::string("cuda backend: no CUDA stream (no usable device)"));
    }
    cudaSetDevice(device_);
    Buffer b;
    b.bytes = bytes;
    const std::size_t total = bytes + 2 * slack_;
    if (cudaError_t e = cudaMalloc(&b.base, total); e != cudaSuccess) {
        cudaGetLastError();
        return core::failure(cuda_text("buffer allocation", e));
    }
    // Cleared on the backend's stream, which every later upload, dispatch
    // and read-back of the buffer follows (a clear on the legacy stream would
    // not be ordered before them: the backend's stream does not synchronise
    // with it).
    auto s = static_cast<cudaStream_t>(stream_);
    if (cudaError_t e = cudaMemsetAsync(b.base, 0, total, s); e != cudaSuccess) {
        cudaFree(b.base);
        return core::failure(cuda_text("buffer clear", e));
    }
    b.data = static_cast<std::byte*>(b.base) + slack_;
    const std::uint32_t id = next_id_++;
    buffers_[id] = b;
    return BufferId{id};
}

void CudaComputeBackend::drop_tables(BufferId buffer) noexcept {
    auto it = tables_.find(buffer.value);
    if (it != tables_.end()) {
        orr_gl3d_destroy(it->second.handle);
        orr_gl2d_destroy(it->second.handle2);
        tables_.erase(it);
    }
}

void CudaComputeBackend::release_buffer(BufferId buffer) noexcept {
    auto it = buffers_.find(buffer.value);
    if (it == buffers_.end()) {
        return;
    }
    cudaSetDevice(device_);
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream_));
    drop_tables(buffer);
    cudaFree(it->second.base);
    buffers_.erase(it);
}

std::size_t CudaComputeBackend::buffer_size(BufferId buffer) const noexcept {
    auto it = buffers_.find(buffer.value);
    return it == buffers_.end() ? 0 : it->second.bytes;
}

Status CudaComputeBackend::upload(BufferId buffer, std::size_t offset, std::span<const std::byte> bytes) {
    auto it = buffers_.find(buffer.value);
    if (it == buffers_.end()) {
        return failure("cuda backend: upload to an unknown buffer");
    }
    if (offset > it->second.bytes || bytes.size() > it->second.bytes - offset) {
        return failure("cuda backend: upload outside the buffer");
    }
    // A new node-code buffer content invalidates the tables derived from it.
    drop_tables(buffer);
    cudaSetDevice(device_);
    auto s = static_cast<cudaStream_t>(stream_);
    if (cudaError_t e = cudaMemcpyAsync(it->second.data + offset, bytes.data(), bytes.size(),
                                        cudaMemcpyHostToDevice, s);
        e != cudaSuccess) {
        return failure(cuda_text("upload", e));
    }
    if (cudaError_t e = cudaStreamSynchronize(s); e != cudaSuccess) {
        return failure(cuda_text("upload", e));
    }
    return std::monostate{};
}

Status CudaComputeBackend::readback(BufferId buffer, std::size_t offset, std::span<std::byte> bytes) {
    auto it = buffers_.find(buffer.value);
    if (it == buffers_.end()) {
        return failure("cuda backend: readback of an unknown buffer");
    }
    if (offset > it->second.bytes || bytes.size() > it->second.bytes - offset) {
        return failure("cuda backend: readback outside the buffer");
    }
    cudaSetDevice(device_);
    auto s = static_cast<cudaStream_t>(stream_);
    if (cudaError_t e = cudaMemcpyAsync(bytes.data(), it->second.data + offset, bytes.size(),
                                        cudaMemcpyDeviceToHost, s);
        e != cudaSuccess) {
        return failure(cuda_text("readback", e));
    }
    if (cudaError_t e = cudaStreamSynchronize(s); e != cudaSuccess) {
        return failure(cuda_text("readback", e));
    }
    return std::monostate{};
}

Status CudaComputeBackend::tables_for(BufferId classes, const orr_gl3d_params& params, Tables*& out) {
    auto it = tables_.find(classes.value);
    if (it != tables_.end()) {
        const orr_gl3d_params& l = it->second.lattice;
        const bool same = it->second.handle != nullptr && l.nx == params.nx && l.ny == params.ny && l.nz == params.nz &&
                          l.x_mode == params.x_mode && l.outlet_mode == params.outlet_mode &&
                          std::equal(std::begin(l.wall_kind), std::end(l.wall_kind), std::begin(params.wall_kind));
        if (same) {
            out = &it->second;
            return std::monostate{};
        }
        drop_tables(classes);
    }
    const std::size_t cells = static_cast<std::size_t>(params.nx) * params.ny * params.nz;
    if (buffer_size(classes) < cells * sizeof(std::uint32_t)) {
        return failure("cuda backend: the node-code buffer is smaller than the lattice");
    }
    std::vector<std::uint32_t> codes(cells);
    if (Status read = readback(classes, 0, std::as_writable_bytes(std::span<std::uint32_t>(codes))); !read) {
        return read;
    }
    orr_gl3d* handle = nullptr;
    if (orr_gl3d_create(&params, codes.data(), device_, &handle) != ORR_OK) {
        return failure(std::string("cuda backend: ") + orr_last_error());
    }
    std::uint32_t top = 0;
    for (const std::uint32_t c : codes) top = std::max(top, c);
    const std::size_t wall_values = top >= 3 ? 19 * static_cast<std::size_t>(top - 2) : 0;
    Tables& entry = tables_[classes.value];
    entry = Tables{handle, params, wall_values};
    ++tables_built_;
    out = &entry;
    return std::monostate{};
}

Status CudaComputeBackend::tables2_for(BufferId solid, const orr_gl2d_params& params, Tables*& out) {
    auto it = tables_.find(solid.value);
    if (it != tables_.end()) {
        const orr_gl2d_params& l = it->second.lattice2;
        const bool same = it->second.handle2 != nullptr && l.nx == params.nx && l.ny == params.ny &&
                          l.x_mode == params.x_mode && l.outlet_mode == params.outlet_mode &&
                          l.bottom_kind == params.bottom_kind && l.top_kind == params.top_kind;
        if (same) {
            out = &it->second;
            return std::monostate{};
        }
        drop_tables(solid);
    }
    const std::size_t cells = static_cast<std::size_t>(params.nx) * params.ny;
    if (buffer_size(solid) < cells * sizeof(std::uint32_t)) {
        return failure("cuda backend: the solid-flag buffer is smaller than the lattice");
    }
    std::vector<std::uint32_t> flags(cells);
    if (Status read = readback(solid, 0, std::as_writable_bytes(std::span<std::uint32_t>(flags))); !read) {
        return read;
    }
    orr_gl2d* handle = nullptr;
    if (orr_gl2d_create(&params, flags.data(), device_, &handle) != ORR_OK) {
        return failure(std::string("cuda backend: ") + orr_last_error());
    }
    Tables& entry = tables_[solid.value];
    entry = Tables{};
    entry.handle2 = handle;
    entry.lattice2 = params;
    ++tables_built_;
    out = &entry;
    return std::monostate{};
}

// The D2Q9 driver's dispatches (GpuLbm2D::step, macroscopic, force:
// lbm2d_gpu.cpp:218-300).
Status CudaComputeBackend::dispatch2(const DispatchCommand& command) {
    orr_gl2d_params p{};
    if (auto bad = read_uniforms2(command.uniforms, p)) {
        return failure(*bad);
    }
    std::array<Buffer*, 8> bound{};
    std::array<BufferId, 8> ids{};
    for (const BufferBinding& b : command.buffers) {
        auto it = buffers_.find(b.buffer.value);
        if (it == buffers_.end()) {
            return failure("cuda backend: dispatch binds an unknown buffer");
        }
        if (b.binding < bound.size()) {
            bound[b.binding] = &it->second;
            ids[b.binding] = b.buffer;
        }
    }
    const std::size_t cells = static_cast<std::size_t>(p.nx) * p.ny;
    const auto need = [&](std::uint32_t binding, std::size_t bytes, const char* what) -> std::optional<std::string> {
        if (bound[binding] == nullptr) {
            return std::string("cuda backend: ") + what + " is not bound";
        }
        if (bound[binding]->bytes < bytes) {
            return std::string("cuda backend: the ") + what + " buffer is too small for the lattice";
        }
        return std::nullopt;
    };
    if (auto bad = need(kBindSource, 9 * cells * sizeof(float), "population source")) return failure(*bad);
    cudaSetDevice(device_);
    const auto* src = reinterpret_cast<const float*>(bound[kBindSource]->data);
    orr_status st = ORR_OK;
    orr_gl2d* t = nullptr;
    if (command.kernel == kForce2) {
        // The force kernel binds no solid flags and needs no tables (the
        // link list carries the geometry).
        if (auto bad = need(kBindLinks, 2 * static_cast<std::size_t>(p.link_count) * sizeof(std::uint32_t), "link")) {
            return failure(*bad);
        }
        if (auto bad = need(kBindLinkForce, 2 * static_cast<std::size_t>(p.link_count) * sizeof(float),
                            "link force")) {
            return failure(*bad);
        }
        st = orr_gl2d_link_force(t, &p, src, reinterpret_cast<const std::uint32_t*>(bound[kBindLinks]->data),
                                 reinterpret_cast<float*>(bound[kBindLinkForce]->data), stream_);
    } else {
        if (auto bad = need(kBindClass, cells * sizeof(std::uint32_t), "solid flag")) return failure(*bad);
        Tables* tables = nullptr;
        if (Status ok = tables2_for(ids[kBindClass], p, tables); !ok) {
            return ok;
        }
        t = tables->handle2;
        if (command.kernel == kStep2) {
            if (auto bad = need(kBindDestination, 9 * cells * sizeof(float), "population destination")) {
                return failure(*bad);
            }
            if (auto bad = need(kBindOutlet, 3 * static_cast<std::size_t>(p.ny) * sizeof(float), "outlet")) {
                return failure(*bad);
            }
            st = orr_gl2d_step(t, &p, src, reinterpret_cast<float*>(bound[kBindDestination]->data),
                               reinterpret_cast<float*>(bound[kBindOutlet]->data), stream_);
        } else {
            if (auto bad = need(kBindMoments, 3 * cells * sizeof(float), "moment")) return failure(*bad);
            st = orr_gl2d_moments(t, &p, src, reinterpret_cast<float*>(bound[kBindMoments]->data), stream_);
        }
    }
    if (st != ORR_OK) {
        return failure(std::string("cuda backend: ") + (t ? orr_gl2d_last_error(t) : orr_last_error()));
    }
    ++dispatches_;
    return std::monostate{};
}

Status CudaComputeBackend::dispatch(const DispatchCommand& command) {
    if (!has_kernel(command.kernel)) {
        return failure("cuda backend: unknown kernel " + std::string(command.kernel));
    }
    if (command.global.x == 0 || command.global.y == 0 || command.global.z == 0) {
        return failure("cuda backend: empty dispatch");
    }
    if (command.kernel == kStep2 || command.kernel == kMoments2 || command.kernel == kForce2) {
        return dispatch2(command);
    }
    orr_gl3d_params p{};
    if (auto bad = read_uniforms(command.uniforms, p)) {
        return failure(*bad);
    }
    std::array<Buffer*, 8> bound{};
    std::array<BufferId, 8> ids{};
    for (const BufferBinding& b : command.buffers) {
        auto it = buffers_.find(b.buffer.value);
        if (it == buffers_.end()) {
            return failure("cuda backend: dispatch binds an unknown buffer");
        }
        if (b.binding < bound.size()) {
            bound[b.binding] = &it->second;
            ids[b.binding] = b.buffer;
        }
    }
    const std::size_t cells = static_cast<std::size_t>(p.nx) * p.ny * p.nz;
    const auto need = [&](std::uint32_t binding, std::size_t bytes, const char* what) -> std::optional<std::string> {
        if (bound[binding] == nullptr) {
            return std::string("cuda backend: ") + what + " is not bound";
        }
        if (bound[binding]->bytes < bytes) {
            return std::string("cuda backend: the ") + what + " buffer is too small for the lattice";
        }
        return std::nullopt;
    };
    if (auto bad = need(kBindSource, 19 * cells * sizeof(float), "population source")) return failure(*bad);
    if (auto bad = need(kBindClass, cells * sizeof(std::uint32_t), "node code")) return failure(*bad);
    Tables* tables = nullptr;
    if (Status ok = tables_for(ids[kBindClass], p, tables); !ok) {
        return ok;
    }
    orr_gl3d* t = tables->handle;
    if (command.kernel != kMoments && tables->wall_values > 0) {
        if (auto bad = need(kBindWall, tables->wall_values * sizeof(float), "wall fraction")) return failure(*bad);
    }
    cudaSetDevice(device_);
    const auto* src = reinterpret_cast<const float*>(bound[kBindSource]->data);
    const float* wall = bound[kBindWall] ? reinterpret_cast<const float*>(bound[kBindWall]->data) : nullptr;
    orr_status st = ORR_OK;
    if (command.kernel == kStep) {
        if (auto bad = need(kBindDestination, 19 * cells * sizeof(float), "population destination")) {
            return failure(*bad);
        }
        if (auto bad = need(kBindOutlet, 5 * static_cast<std::size_t>(p.ny) * p.nz * sizeof(float), "outlet")) {
            return failure(*bad);
        }
        st = orr_gl3d_step(t, &p, src, reinterpret_cast<float*>(bound[kBindDestination]->data),
                           reinterpret_cast<float*>(bound[kBindOutlet]->data), wall, stream_);
    } else if (command.kernel == kMoments) {
        if (auto bad = need(kBindMoments, 4 * cells * sizeof(float), "moment")) return failure(*bad);
        st = orr_gl3d_moments(t, &p, src, reinterpret_cast<float*>(bound[kBindMoments]->data), stream_);
    } else {
        if (auto bad = need(kBindLinks, 2 * static_cast<std::size_t>(p.link_count) * sizeof(std::uint32_t), "link")) {
            return failure(*bad);
        }
        if (auto bad = need(kBindLinkForce, static_cast<std::size_t>(p.link_count) * sizeof(float), "link force")) {
            return failure(*bad);
        }
        st = orr_gl3d_link_force(t, &p, src, reinterpret_cast<const std::uint32_t*>(bound[kBindLinks]->data),
                                 reinterpret_cast<float*>(bound[kBindLinkForce]->data), wall, stream_);
    }
    if (st != ORR_OK) {
        return failure(std::string("cuda backend: ") + orr_gl3d_last_error(t));
    }
    ++dispatches_;
    return std::monostate{};
}

} // namespace orrery::aero::compute
