// Instantiation of the D3Q19 and D2Q9 kernels for the binary32-arithmetic
// storage forms: binary32, FP16S and bfloat16 populations.
#include "ops2d_impl.cuh"
#include "ops3d_impl.cuh"

namespace orr {

const Ops3D& ops3d_f32() {
    return Launch3D<float>::table();
}

const Ops3D& ops3d_f16() {
    return Launch3D<__half>::table();
}

const Ops3D& ops3d_bf16() {
    return Launch3D<__nv_bfloat16>::table();
}

const Ops2D& ops2d_f32() {
    return Launch2D<float>::table();
}

const Ops2D& ops2d_f16() {
    return Launch2D<__half>::table();
}

const Ops2D& ops2d_bf16() {
    return Launch2D<__nv_bfloat16>::table();
}

} // namespace orr
