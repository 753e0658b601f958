// Lbm2DSolver on the B200 library (see lbm2d_cuda.h).  Every member forwards
// to the D2Q9 C ABI of include/orrery_lbm.h with the reference's semantics:
// refusals before allocation with the reference's texts, a failed call
// returns core::failure with the library's text, populations unshifted in
// the reference layout, force and moment about the lattice origin.
#include "lbm2d_cuda.h"

#include <utility>
#include <variant>
#include <vector>

namespace orrery::aero::lbm {
namespace {

orr_wall wall2_of(const Wall& w) {
    orr_wall o{};
    o.kind = static_cast<std::int32_t>(w.kind);
    o.velocity_x = w.velocity_x;
    return o;
}

class CudaLbm2D final : public Lbm2DSolver {
public:
    CudaLbm2D(orr_lbm2d* handle, const Lbm2DConfig& config, SolidMask2D mask)
        : h_(handle), config_(config), mask_(std::move(mask)) {}
    ~CudaLbm2D() override { orr_lbm2d_destroy(h_); }

    const Lbm2DConfig& config() const noexcept override { return config_; }
    const SolidMask2D& mask() const noexcept override { return mask_; }
    std::uint64_t steps() const noexcept override {
        std::uint64_t s = 0;
        static_cast<void>(orr_lbm2d_steps(h_, &s));
        return s;
    }

    Status initialize(const InitialState& initial) override {
        const std::size_t n = mask_.solid.size();
        std::vector<double> rho(n), ux(n), uy(n);
        for (std::size_t y = 0; y < config_.ny; ++y) {
            for (std::size_t x = 0; x < config_.nx; ++x) {
                const d2q9::Moments m = initial(x, y);
                const std::size_t c = x + config_.nx * y;
                rho[c] = m.rho;
                ux[c] = m.ux;
                uy[c] = m.uy;
            }
        }
        return status(orr_lbm2d_initialize(h_, rho.data(), ux.data(), uy.data()));
    }
    Status step(std::size_t count) override { return status(orr_lbm2d_step(h_, count)); }

    core::Result<MacroFields2D, std::string> macroscopic() override {
        MacroFields2D out;
        out.nx = config_.nx;
        out.ny = config_.ny;
        const std::size_t n = mask_.solid.size();
        out.density.resize(n);
        out.velocity_x.resize(n);
        out.velocity_y.resize(n);
        out.solid = mask_.solid;
        if (orr_lbm2d_macroscopic(h_, out.density.data(), out.velocity_x.data(), out.velocity_y.data()) != ORR_OK) {
            return core::failure(error());
        }
        return out;
    }
    core::Result<std::vector<double>, std::string> populations() override {
        std::vector<double> f(d2q9::q * mask_.solid.size());
        if (orr_lbm2d_populations(h_, f.data()) != ORR_OK) {
            return core::failure(error());
        }
        return f;
    }
    core::Result<Force2D, std::string> force() override {
        double fm[3] = {};
        if (orr_lbm2d_force(h_, fm) != ORR_OK) {
            return core::failure(error());
        }
        Force2D out;
        out.x = fm[0];
        out.y = fm[1];
        out.moment = fm[2];
        return out;
    }
    core::Result<double, std::string> mass() override {
        double m = 0.0;
        if (orr_lbm2d_mass(h_, &m) != ORR_OK) {
            return core::failure(error());
        }
        return m;
    }

private:
    std::string error() const { return orr_lbm2d_last_error(h_); }
    Status status(orr_status s) const {
        if (s == ORR_OK) {
            return std::monostate{};
        }
        return core::failure(error());
    }

    orr_lbm2d* h_;
    Lbm2DConfig config_;
    SolidMask2D mask_;
};

} // namespace

orr_lbm2d_config c_config(const Lbm2DConfig& c) {
    orr_lbm2d_config o{};
    o.nx = c.nx;
    o.ny = c.ny;
    o.tau = c.tau;
    o.x_boundary = static_cast<std::int32_t>(c.x_boundary);
    o.outlet = static_cast<std::int32_t>(c.outlet);
    o.bottom = wall2_of(c.bottom);
    o.top = wall2_of(c.top);
    o.inlet_ux = c.inlet_ux;
    o.inlet_uy = c.inlet_uy;
    o.body_force_x = c.body_force_x;
    o.body_force_y = c.body_force_y;
    o.smagorinsky_enabled = c.smagorinsky.enabled ? 1 : 0;
    o.smagorinsky_constant = c.smagorinsky.constant;
    return o;
}

core::Result<std::unique_ptr<Lbm2DSolver>, std::string>
make_cuda_solver(const Lbm2DConfig& config, SolidMask2D mask, std::int32_t storage, std::int32_t device) {
    const orr_lbm2d_config c = c_config(config);
    orr_solver_options options{};
    options.storage = storage;
    options.device = device;
    orr_lbm2d* h = nullptr;
    if (orr_lbm2d_create(&c, mask.solid.data(), &options, &h) != ORR_OK) {
        return core::failure(std::string(orr_last_error()));
    }
    return std::unique_ptr<Lbm2DSolver>(std::make_unique<CudaLbm2D>(h, config, std::move(mask)));
}

} // namespace orrery::aero::lbm
