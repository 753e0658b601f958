// Library-wide entry points of the C ABI and the shared error helpers.
#include "common.h"

#include <cstring>

namespace orr {

namespace {
thread_local std::string g_error;
} // namespace

orr_status fail(orr_status status, const std::string& text) {
    g_error = text;
    return status;
}

void clear_error() {
    g_error.clear();
}

const std::string& thread_error() {
    return g_error;
}

std::string describe(const CudaError& e) {
    return std::string(e.what) + ": " + cudaGetErrorString(e.code);
}

void require_device(int device) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Refusal{ORR_ERR_NO_DEVICE, "no CUDA device is available"};
    }
    if (device < 0 || device >= count) {
        throw Refusal{ORR_ERR_INVALID, "CUDA device ordinal out of range"};
    }
    // Two attributes rather than the whole property record, whose query
    // takes milliseconds.
    int major = 0, minor = 0;
    check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "cudaDeviceGetAttribute");
    check(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device), "cudaDeviceGetAttribute");
    if (major != 10) {
        throw Refusal{ORR_ERR_NO_DEVICE,
                      "the kernels are built for sm_100a; device " + std::to_string(device) +
                          " is sm_" + std::to_string(major) + std::to_string(minor)};
    }
    check(cudaSetDevice(device), "cudaSetDevice");
}

} // namespace orr

extern "C" {

const char* orr_last_error(void) {
    return orr::thread_error().c_str();
}

const char* orr_version(void) {
    return "orrery_b200 lbm 0.1 (sm_100a)";
}

orr_status orr_device_count(int32_t* count) {
    if (count == nullptr) {
        return orr::fail(ORR_ERR_INVALID, "null output pointer");
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return ORR_OK;
}

} // extern "C"
