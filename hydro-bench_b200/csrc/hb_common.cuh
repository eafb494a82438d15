// hb_common.cuh -- status/error plumbing shared by the library's sources.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "hydrob200.h"

namespace hb {

// Records the status and a message for hb_last_error()/hb_last_error_string()
// (per host thread) and returns the status.
int set_error(int status, const char *fmt, ...);

// device error word bits
enum : uint32_t {
    ERRBIT_NONFINITE = 1u << HB_E_NONFINITE,
    ERRBIT_UNDEFINED = 1u << HB_E_UNDEFINED_REF,
    ERRBIT_TABLE_RANGE = 1u << HB_E_INVALID,
    ERRBIT_BARRIER = 1u << HB_E_BARRIER_TIMEOUT,
};

}  // namespace hb

#define HB_CUDA_RET(call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return hb::set_error(HB_E_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,                 \
                                 cudaGetErrorString(e_));                                              \
    } while (0)
