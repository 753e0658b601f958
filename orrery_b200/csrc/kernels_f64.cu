// Instantiation of the D3Q19 and D2Q9 kernels for binary64 populations.
// This unit is compiled with FMA contraction off (-fmad=false) so that every
// expression of the step rounds exactly as the reference CPU solver's does.
#include "ops2d_impl.cuh"
#include "ops3d_impl.cuh"

namespace orr {

const Ops3D& ops3d_f64() {
    return Launch3D<double>::table();
}

const Ops2D& ops2d_f64() {
    return Launch2D<double>::table();
}

} // namespace orr
