// errors.hpp — host-side failures carried as exceptions inside the library and converted to
// mr_status at the C ABI (the reference's exception types map one-to-one onto status codes).
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "minirender_b200.h"

namespace mr {

struct Error : std::runtime_error {
    mr_status status;
    Error(mr_status s, const std::string& message) : std::runtime_error(message), status(s) {}
};

[[noreturn]] inline void fail(mr_status status, const std::string& message) {
    throw Error(status, message);
}

inline void require(bool condition, const char* message) {
    if (!condition) {
        fail(MR_INVALID_ARGUMENT, message);
    }
}

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const mr_status s = e == cudaErrorMemoryAllocation ? MR_OUT_OF_MEMORY : MR_CUDA_ERROR;
        fail(s, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

#define MR_CUDA(call) ::mr::cuda_check((call), #call)

}  // namespace mr
