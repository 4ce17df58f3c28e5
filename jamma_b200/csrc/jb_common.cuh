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

// cuBLAS picks its kernels (and so its rounding) by the workspace it can use.  With the
// library's default pool that depends on how many streams are active, so a DGEMM run
// beside other jobs may round differently from the same DGEMM run alone.  Calls whose
// results must not depend on concurrent work bind a caller-owned workspace of this fixed
// size (one per concurrently used buffer set, so no two streams share it).
constexpr int64_t kCublasWorkspaceBytes = int64_t(32) << 20;

// Set the stream, then the workspace (cublasSetStream resets the workspace to the pool).
inline cublasStatus_t bind_cublas(cublasHandle_t h, cudaStream_t st, void* ws, int64_t bytes) {
    cublasStatus_t s = cublasSetStream(h, st);
    if (s != CUBLAS_STATUS_SUCCESS) return s;
    return cublasSetWorkspace(h, ws, (size_t)bytes);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// grid.y for kernels that stride one matrix column per y index: the hardware caps
// gridDim.y at 65535, so larger n loop over columns j = blockIdx.y, + gridDim.y, ...
inline unsigned grid_y(int64_t n) { return (unsigned)(n < 65535 ? (n > 0 ? n : 1) : 65535); }

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
