// Link-time stand-in for the reference's 3D panel solver.  TEST
// INFRASTRUCTURE ONLY, for oracle/_ref/libref_adapter.so.
//
// atmo::default_aero_solver_factory (src/atmo/aero_table.cpp) names
// aero::PanelSolver3D, whose implementation (src/aero/panel3d.cpp with
// linear_solve.cpp) needs Eigen, which this image does not have.  The drag
// tables built through the harness choose the lattice Boltzmann solver, so
// the panel solver is only linked, never run: its two out-of-line members
// refuse.
#include <stdexcept>

#include "orrery/aero/panel_method.h"

namespace orrery::aero {

void PanelSolver3D::setup(const AeroGeometry& /*geometry*/, const FlowConditions& /*conditions*/) {
    throw std::runtime_error("panel solver: not built in the oracle harness (it needs Eigen)");
}

bool PanelSolver3D::step() {
    throw std::runtime_error("panel solver: not built in the oracle harness (it needs Eigen)");
}

} // namespace orrery::aero
