// Shared helpers for libjamma_b200: error reporting, status codes, library handles.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/jamma_b200.h"

namespace jb {

// Last error text of the calling host thread (jb_last_error copies it out).
void set_error(const char* fmt, ...);

int32_t cuda_status(cudaError_t e, const char* what);
int32_t cublas_status(cublasStatus_t s, const char* what);
int32_t cusolver_status(cusolverStatus_t s, const char* what);

// Per-thread, per-device library handles (created on first use, never destroyed
// before process exit so that calls from many streams reuse them).
cublasHandle_t cublas_handle();
cusolverDnHandle_t cusolver_handle();

inline cudaStream_t as_stream(uintptr_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace jb

#define JB_CHECK_ARG(cond, ...)                 \
    do {                                        \
        if (!(cond)) {                          \
            ::jb::set_error(__VA_ARGS__);       \
            return JB_E_INVALID;                \
        }                                       \
    } while (0)

#define JB_CUDA(call)                                                 \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return ::jb::cuda_status(e_, #call);   \
    } while (0)

#define JB_LAUNCH_CHECK(name)                                         \
    do {                                                              \
        cudaError_t e_ = cudaGetLastError();                          \
        if (e_ != cudaSuccess) return ::jb::cuda_status(e_, name);    \
    } while (0)
