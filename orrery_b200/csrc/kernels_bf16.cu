// Instantiation of the D3Q19 and D2Q9 kernels for bfloat16 populations
// (binary32 arithmetic).  One unit per storage form, so they build in
// parallel.
#include "ops2d_impl.cuh"
#include "ops3d_impl.cuh"

namespace orr {

const Ops3D& ops3d_bf16() {
    return Launch3D<__nv_bfloat16>::table();
}

const Ops2D& ops2d_bf16() {
    return Launch2D<__nv_bfloat16>::table();
}

} // namespace orr
