// Shared helpers of the C ABI implementation: per-thread error text, CUDA
// status checks, and the exception barrier around every entry point.
#pragma once

#include <cuda_runtime.h>

#include <exception>
#include <string>

#include "orrery_lbm.h"

namespace orr {

// Sets the calling thread's last error and returns `status`.
orr_status fail(orr_status status, const std::string& text);
void clear_error();
const std::string& thread_error();

// A failed CUDA call: the call's text plus CUDA's error string.
struct CudaError {
    cudaError_t code;
    const char* what;
};

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw CudaError{e, what};
    }
}

// Thrown by planning or validation with the refusal status.
struct Refusal {
    orr_status status;
    std::string text;
};

std::string describe(const CudaError& e);

// Runs `body`, turning exceptions into a status and an error text (stored
// on the thread, and in `*handle_error` when given).
template <class F> orr_status guarded(std::string* handle_error, F&& body) {
    orr_status status = ORR_OK;
    std::string text;
    try {
        status = body();
    } catch (const Refusal& r) {
        status = r.status;
        text = r.text;
    } catch (const CudaError& e) {
        status = e.code == cudaErrorMemoryAllocation ? ORR_ERR_MEMORY : ORR_ERR_CUDA;
        if (e.code == cudaErrorNoDevice || e.code == cudaErrorInsufficientDriver) {
            status = ORR_ERR_NO_DEVICE;
        }
        text = describe(e);
    } catch (const std::bad_alloc&) {
        status = ORR_ERR_MEMORY;
        text = "host memory exhausted";
    } catch (const std::exception& e) {
        status = ORR_ERR_STATE;
        text = e.what();
    } catch (...) {
        status = ORR_ERR_STATE;
        text = "unknown failure";
    }
    if (status != ORR_OK) {
        if (text.empty()) {
            text = thread_error();
        }
        fail(status, text);
        if (handle_error != nullptr) {
            *handle_error = text;
        }
    }
    return status;
}

// Throws a NO_DEVICE refusal unless a compute capability 10.x device exists.
void require_device(int device);

} // namespace orr
