// D3Q19 and D2Q9 velocity sets, weights and symmetry tables, shared by host
// planning code and device kernels.  Direction order is the reference's
// (src/aero/lbm3d/include/orrery/aero/lbm3d/d3q19.h:15-36,
//  src/aero/lbm/include/orrery/aero/lbm/d2q9.h:12-23): the step, the
// boundary-link list and the population read-back all index by it.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define ORR_HD __host__ __device__ __forceinline__
#else
#define ORR_HD inline
#endif

namespace orr {

namespace d3 {
constexpr int Q = 19;
// 0 rest; 1 +x, 2 -x, 3 +y, 4 -y, 5 +z, 6 -z; then the face diagonals in
// opposite pairs.
ORR_HD constexpr int cx(int i) {
    constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[i];
}
ORR_HD constexpr int cy(int i) {
    constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[i];
}
ORR_HD constexpr int cz(int i) {
    constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[i];
}
ORR_HD constexpr int opposite(int i) {
    constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
    return t[i];
}
ORR_HD constexpr int mirror_y(int i) {
    constexpr int t[Q] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 18, 17, 16, 15};
    return t[i];
}
ORR_HD constexpr int mirror_z(int i) {
    constexpr int t[Q] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16};
    return t[i];
}
// Weights as the exact quotients the reference uses (1/3, 1/18, 1/36).
ORR_HD constexpr double w(int i) {
    return i == 0 ? 1.0 / 3.0 : (i <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
}
// Outlet history slot of the populations entering at x = nx - 1 (c_x = -1):
// directions 2, 8, 10, 12, 14 (src/aero/lbm3d/lbm3d_internal.h:30-46).
ORR_HD constexpr int outlet_slot(int i) {
    return i == 2 ? 0 : (i == 8 ? 1 : (i == 10 ? 2 : (i == 12 ? 3 : 4)));
}
constexpr int kOutletSlots = 5;
} // namespace d3

namespace d2 {
constexpr int Q = 9;
// 0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE.
ORR_HD constexpr int cx(int i) {
    constexpr int t[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    return t[i];
}
ORR_HD constexpr int cy(int i) {
    constexpr int t[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    return t[i];
}
ORR_HD constexpr int opposite(int i) {
    constexpr int t[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    return t[i];
}
ORR_HD constexpr int mirror_y(int i) {
    constexpr int t[Q] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
    return t[i];
}
ORR_HD constexpr double w(int i) {
    return i == 0 ? 4.0 / 9.0 : (i <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
}
// Outlet history slot of directions 3, 6, 7 (src/aero/lbm/lbm2d_internal.h:24-27).
ORR_HD constexpr int outlet_slot(int i) {
    return i == 3 ? 0 : (i == 6 ? 1 : 2);
}
constexpr int kOutletSlots = 3;
} // namespace d2

// Node classes of the step: solid (skipped), bulk fluid (interior, plain pull
// streaming), listed fluid (a solid source, or an x-edge node of an interior
// row: the general gather over the node list) and face fluid (a node of a
// row on the y or z faces with no solid source: the row-uniform side rules).
enum : uint8_t { kSolid = 0, kBulk = 1, kBoundary = 2, kFace = 3 };

} // namespace orr
