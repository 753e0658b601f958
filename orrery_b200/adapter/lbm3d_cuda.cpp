// Lbm3DSolver on the B200 library (see lbm3d_cuda.h).  Every member forwards
// to the C ABI of include/orrery_lbm.h; the solver keeps the reference's
// semantics: refusals before allocation with the reference's texts, a failed
// call returns core::failure with the library's text, populations unshifted
// in the reference layout, force and moment about the lattice origin, links()
// in scan order.
#include "lbm3d_cuda.h"

#include <array>
#include <utility>
#include <variant>
#include <vector>

namespace orrery::aero::lbm {
namespace {

orr_wall wall_of(const Wall& w) {
    orr_wall o{};
    o.kind = static_cast<std::int32_t>(w.kind);
    o.velocity_x = w.velocity_x;
    return o;
}

orr_lbm3d_config config_of(const Lbm3DConfig& c) {
    orr_lbm3d_config o{};
    o.nx = c.nx;
    o.ny = c.ny;
    o.nz = c.nz;
    o.tau = c.tau;
    o.x_boundary = static_cast<std::int32_t>(c.x_boundary);
    o.outlet = static_cast<std::int32_t>(c.outlet);
    o.y_low = wall_of(c.y_low);
    o.y_high = wall_of(c.y_high);
    o.z_low = wall_of(c.z_low);
    o.z_high = wall_of(c.z_high);
    o.inlet_ux = c.inlet_ux;
    o.inlet_uy = c.inlet_uy;
    o.inlet_uz = c.inlet_uz;
    o.body_force_x = c.body_force_x;
    o.body_force_y = c.body_force_y;
    o.body_force_z = c.body_force_z;
    o.smagorinsky_enabled = c.smagorinsky.enabled ? 1 : 0;
    o.smagorinsky_constant = c.smagorinsky.constant;
    o.sponge_strength = c.sponge.strength;
    o.sponge_inlet = c.sponge.inlet;
    o.sponge_outlet = c.sponge.outlet;
    o.sponge_sides = c.sponge.sides;
    o.solid_wall = static_cast<std::int32_t>(c.solid_wall);
    return o;
}

} // namespace

orr_lbm3d_config c_config(const Lbm3DConfig& config) {
    return config_of(config);
}

namespace {

class CudaLbm3D final : public Lbm3DSolver {
public:
    CudaLbm3D(orr_lbm3d* handle, const Lbm3DConfig& config, SolidMask3D mask)
        : h_(handle), config_(config), mask_(std::move(mask)) {
        std::uint64_t n = 0;
        if (orr_lbm3d_link_count(h_, &n) == ORR_OK && n > 0) {
            std::vector<std::uint32_t> cell(n), dir(n);
            std::vector<double> q(n);
            if (orr_lbm3d_links(h_, cell.data(), dir.data(), q.data()) == ORR_OK) {
                links_.reserve(n);
                for (std::uint64_t k = 0; k < n; ++k) {
                    links_.push_back(BoundaryLink3D{cell[k], dir[k], q[k]});
                }
            }
        }
    }
    ~CudaLbm3D() override { orr_lbm3d_destroy(h_); }

    const Lbm3DConfig& config() const noexcept override { return config_; }
    const SolidMask3D& mask() const noexcept override { return mask_; }
    std::uint64_t steps() const noexcept override {
        std::uint64_t s = 0;
        static_cast<void>(orr_lbm3d_steps(h_, &s));
        return s;
    }
    const std::vector<BoundaryLink3D>& links() const noexcept override { return links_; }

    Status initialize(const InitialState3D& initial) override {
        const std::size_t n = mask_.solid.size();
        std::vector<double> rho(n), ux(n), uy(n), uz(n);
        for (std::size_t z = 0; z < config_.nz; ++z) {
            for (std::size_t y = 0; y < config_.ny; ++y) {
                for (std::size_t x = 0; x < config_.nx; ++x) {
                    const d3q19::Moments m = initial(x, y, z);
                    const std::size_t c = mask_.index(x, y, z);
                    rho[c] = m.rho;
                    ux[c] = m.ux;
                    uy[c] = m.uy;
                    uz[c] = m.uz;
                }
            }
        }
        return status(orr_lbm3d_initialize(h_, rho.data(), ux.data(), uy.data(), uz.data()));
    }
    Status step(std::size_t count) override { return status(orr_lbm3d_step(h_, count)); }
    Status set_inlet_velocity(const std::array<double, 3>& velocity) override {
        return status(orr_lbm3d_set_inlet_velocity(h_, velocity.data()));
    }
    std::array<double, 3> inlet_velocity() const noexcept override {
        std::array<double, 3> v{};
        static_cast<void>(orr_lbm3d_inlet_velocity(h_, v.data()));
        return v;
    }

    core::Result<MacroFields3D, std::string> macroscopic() override {
        MacroFields3D out;
        out.nx = config_.nx;
        out.ny = config_.ny;
        out.nz = config_.nz;
        const std::size_t n = mask_.solid.size();
        out.density.resize(n);
        out.velocity_x.resize(n);
        out.velocity_y.resize(n);
        out.velocity_z.resize(n);
        out.solid = mask_.solid;
        if (orr_lbm3d_macroscopic(h_, out.density.data(), out.velocity_x.data(), out.velocity_y.data(),
                                  out.velocity_z.data()) != ORR_OK) {
            return core::failure(error());
        }
        return out;
    }
    core::Result<std::vector<double>, std::string> populations() override {
        std::vector<double> f(d3q19::q * mask_.solid.size());
        if (orr_lbm3d_populations(h_, f.data()) != ORR_OK) {
            return core::failure(error());
        }
        return f;
    }
    core::Result<Force3D, std::string> force() override {
        double fm[6] = {};
        if (orr_lbm3d_force(h_, fm) != ORR_OK) {
            return core::failure(error());
        }
        Force3D out;
        out.force = {fm[0], fm[1], fm[2]};
        out.moment = {fm[3], fm[4], fm[5]};
        return out;
    }
    core::Result<double, std::string> mass() override {
        double m = 0.0;
        if (orr_lbm3d_mass(h_, &m) != ORR_OK) {
            return core::failure(error());
        }
        return m;
    }

private:
    std::string error() const { return orr_lbm3d_last_error(h_); }
    Status status(orr_status s) const {
        if (s == ORR_OK) {
            return std::monostate{};
        }
        return core::failure(error());
    }

    orr_lbm3d* h_;
    Lbm3DConfig config_;
    SolidMask3D mask_;
    std::vector<BoundaryLink3D> links_;
};

} // namespace

core::Result<std::unique_ptr<Lbm3DSolver>, std::string>
make_cuda_solver(const Lbm3DConfig& config, SolidMask3D mask, std::int32_t storage, std::int32_t device) {
    const orr_lbm3d_config c = config_of(config);
    orr_solver_options options{};
    options.storage = storage;
    options.device = device;
    orr_lbm3d* h = nullptr;
    if (orr_lbm3d_create(&c, mask.solid.data(), mask.distance.empty() ? nullptr : mask.distance.data(), &options,
                         &h) != ORR_OK) {
        return core::failure(std::string(orr_last_error()));
    }
    return std::unique_ptr<Lbm3DSolver>(std::make_unique<CudaLbm3D>(h, config, std::move(mask)));
}

} // namespace orrery::aero::lbm
