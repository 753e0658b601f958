// Named ranges around the library's host calls, for profilers and tracers
// (NVTX, header-only: without an attached tool each range costs a branch).
// The counterpart of the reference's tracing zones, ORRERY_ZONE("lbm_step")
// around every solver step (src/core/profile/include/orrery/core/profile.h;
// src/aero/lbm3d/lbm3d_gpu.cpp:334, lbm3d_cpu.cpp:139), with the same name
// for a solver step.  The ranges mark host-side calls; the device work they
// enqueue shows on the timeline of the stream they name in a tool that
// correlates the two.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace orr {

class Zone {
public:
    explicit Zone(const char* name) noexcept { nvtxRangePushA(name); }
    ~Zone() { nvtxRangePop(); }
    Zone(const Zone&) = delete;
    Zone& operator=(const Zone&) = delete;
};

} // namespace orr
