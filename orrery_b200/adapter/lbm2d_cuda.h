// Lbm2DSolver on the B200 library: the D2Q9 twin of lbm3d_cuda.h, the file a
// maintainer adds under src/aero/lbm/ of the reference (next to lbm2d_cpu.cpp
// and lbm2d_gpu.cpp) so that callers of the 2D solver seam (lbm2d.h:172-212)
// run on the CUDA solver.  Compiled against the reference's headers and
// linked with orrery_b200/_native/liborrery_lbm.so.
#pragma once

#include <cstdint>
#include <memory>
#include <string>

#include "orrery/aero/lbm/lbm2d.h"
#include "orrery_lbm.h"

namespace orrery::aero::lbm {

// The CUDA D2Q9 solver behind the Lbm2DSolver interface; beside
// make_cpu_solver and make_gpu_solver (lbm2d.h:204-212).  Refuses like
// make_gpu_solver, with the reference's texts, before allocating.  `storage`
// is an ORR_STORAGE_* form (binary32 by default, as the reference's GPU solver).
[[nodiscard]] core::Result<std::unique_ptr<Lbm2DSolver>, std::string>
make_cuda_solver(const Lbm2DConfig& config, SolidMask2D mask, std::int32_t storage = ORR_STORAGE_F32,
                 std::int32_t device = 0);

// The C ABI's configuration record of a reference configuration.
[[nodiscard]] orr_lbm2d_config c_config(const Lbm2DConfig& config);

} // namespace orrery::aero::lbm
