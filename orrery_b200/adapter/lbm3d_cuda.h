// Lbm3DSolver on the B200 library: the file a maintainer adds under
// src/aero/lbm3d/ of the reference (next to lbm3d_cpu.cpp and lbm3d_gpu.cpp)
// so that LbmAeroSolver3D and every other caller of the solver seam
// (lbm3d.h:196-232) run on the CUDA solver.  Compiled against the reference's
// headers and linked with orrery_b200/_native/liborrery_lbm.so.
#pragma once

#include <cstdint>
#include <memory>
#include <string>

#include "orrery/aero/lbm3d/lbm3d.h"
#include "orrery_lbm.h"

namespace orrery::aero::lbm {

// The CUDA solver behind the Lbm3DSolver interface; beside make_cpu_solver
// and make_gpu_solver (lbm3d.h:236-247).  Refuses like make_gpu_solver, with
// the reference's texts, before allocating.  `storage` is an ORR_STORAGE_*
// form (binary32 by default, as the reference's GPU solver).
[[nodiscard]] core::Result<std::unique_ptr<Lbm3DSolver>, std::string>
make_cuda_solver(const Lbm3DConfig& config, SolidMask3D mask, std::int32_t storage = ORR_STORAGE_F32,
                 std::int32_t device = 0);

// The C ABI's configuration record of a reference configuration.
[[nodiscard]] orr_lbm3d_config c_config(const Lbm3DConfig& config);

} // namespace orrery::aero::lbm
