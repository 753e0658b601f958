// Instantiation of the D3Q19 and D2Q9 kernels for binary32 populations
// (binary32 arithmetic).  One unit per storage form, so they build in
// parallel.
#include "ops2d_impl.cuh"
#include "ops3d_impl.cuh"

namespace orr {

const Ops3D& ops3d_f32() {
    return Launch3D<float>::table();
}

const Ops2D& ops2d_f32() {
    return Launch2D<float>::table();
}

} // namespace orr
