// weftk_common.cuh — host-side error plumbing shared by the libweftk translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/weftk.h"

namespace weftk {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// Check a CUDA runtime call; on failure record the message and return WEFTK_E_CUDA.
#define WEFTK_CUDA(call)                                    \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return weftk::cuda_fail(_e, #call); \
    } while (0)

#define WEFTK_REQUIRE(cond, msg)                                  \
    do {                                                          \
        if (!(cond)) return weftk::fail(WEFTK_E_ARG, (msg));      \
    } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace weftk
