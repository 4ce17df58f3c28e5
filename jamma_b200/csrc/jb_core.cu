// libjamma_b200 core: error plumbing, PLINK decode, imputation, plain FP64 kinship,
// FP64 eigendecomposition (cuSOLVER) and plain FP64 rotation (cuBLAS).
#include <cusolverMg.h>
#include <dlfcn.h>

#include <mutex>
#include <string>
#include "jb_common.cuh"

#include <mutex>
#include <vector>

#define JB_VERSION_MAJOR 0
#define JB_VERSION_MINOR 1
#define JB_VERSION_PATCH 0

namespace jb {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int32_t cuda_status(cudaError_t e, const char* what) {
    set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
    return JB_E_CUDA;
}

int32_t cublas_status(cublasStatus_t s, const char* what) {
    set_error("cuBLAS status %d in %s", (int)s, what);
    return JB_E_LIBRARY;
}

int32_t cusolver_status(cusolverStatus_t s, const char* what) {
    set_error("cuSOLVER status %d in %s", (int)s, what);
    return JB_E_LIBRARY;
}

namespace {
constexpr int kMaxDevices = 64;
thread_local cublasHandle_t t_cublas[kMaxDevices] = {nullptr};
thread_local cusolverDnHandle_t t_cusolver[kMaxDevices] = {nullptr};
}  // namespace

cublasHandle_t cublas_handle() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    if (!t_cublas[dev]) {
        if (cublasCreate(&t_cublas[dev]) != CUBLAS_STATUS_SUCCESS) t_cublas[dev] = nullptr;
    }
    return t_cublas[dev];
}

cusolverDnHandle_t cusolver_handle() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    if (!t_cusolver[dev]) {
        if (cusolverDnCreate(&t_cusolver[dev]) != CUSOLVER_STATUS_SUCCESS)
            t_cusolver[dev] = nullptr;
    }
    return t_cusolver[dev];
}

// ---------------------------------------------------------------- kernels

// One CTA per SNP: decode the analysed samples, write int8 codes (3 = missing, zero
// padding up to ld), and reduce {n_obs, sum, n_het, n_hom2}.  Without a sample subset
// each thread decodes one packed byte (4 samples) and stores them as one 32-bit word.
__global__ void decode_bed_kernel(const uint8_t* __restrict__ packed, int64_t bps, int64_t m,
                                  const int32_t* __restrict__ sidx, int64_t n,
                                  int8_t* __restrict__ codes, int64_t ld,
                                  int32_t* __restrict__ counts) {
    const int64_t j = blockIdx.x;
    if (j >= m) return;
    const uint8_t* rec = packed + j * bps;
    int8_t* out = codes + j * ld;
    int obs = 0, sum = 0, het = 0, hom2 = 0;
    // count-A1: 00 -> 2, 01 -> missing (3), 10 -> 1, 11 -> 0
    auto code_of = [](int c) { return c == 0 ? 2 : (c == 1 ? 3 : (c == 2 ? 1 : 0)); };
    if (!sidx && (ld & 15) == 0 && (bps & 3) == 0 &&
        (reinterpret_cast<uintptr_t>(packed) & 3) == 0 && (reinterpret_cast<uintptr_t>(codes) & 15) == 0) {
        // 16 samples per thread: one 32-bit record word (sample e at bits 2e, 2e+1 = l, h)
        // to 16 code bytes.  count-A1 code = (~h, l ^ h) per field; the per-SNP counts come
        // from popcounts of the code bit-planes.  bps % 4 == 0 keeps every word in the record.
        for (int64_t q = threadIdx.x; q < ld / 16; q += blockDim.x) {
            const int64_t s0 = 16 * q;
            uint4 o = make_uint4(0u, 0u, 0u, 0u);
            if (s0 < n) {
                const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(rec) + q);
                const int64_t nv = n - s0 < 16 ? n - s0 : 16;
                const uint32_t vm = (nv >= 16 ? 0xffffffffu : ((1u << (2 * nv)) - 1u)) & 0x55555555u;
                const uint32_t h = (w >> 1) & 0x55555555u, l = w & 0x55555555u;
                const uint32_t c0 = (l ^ h) & vm, c1 = ~h & vm;
                const uint32_t vo = vm & ~(l & ~h);  // observed (not code 3)
                obs += __popc(vo);
                sum += 2 * __popc(c1 & vo) + __popc(c0 & vo);
                het += __popc(~c1 & c0 & vo);
                hom2 += __popc(c1 & ~c0 & vo);
                const uint32_t code = c0 | (c1 << 1);
                auto spread4 = [](uint32_t x) {  // four 2-bit fields -> four bytes
                    x &= 0xffu;
                    x = (x | (x << 12)) & 0x000f000fu;
                    return (x | (x << 6)) & 0x03030303u;
                };
                o = make_uint4(spread4(code), spread4(code >> 8), spread4(code >> 16), spread4(code >> 24));
            }
            *reinterpret_cast<uint4*>(out + s0) = o;
        }
    } else if (!sidx && (ld & 3) == 0) {
        for (int64_t q = threadIdx.x; q < ld / 4; q += blockDim.x) {
            const int64_t s0 = 4 * q;
            uint32_t word = 0;
            if (s0 < n) {
                const int byte = rec[q];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (s0 + e < n) {
                        const int v = code_of((byte >> (2 * e)) & 3);
                        word |= (uint32_t)v << (8 * e);
                        if (v != 3) {
                            obs += 1;
                            sum += v;
                            het += (v == 1);
                            hom2 += (v == 2);
                        }
                    }
                }
            }
            *reinterpret_cast<uint32_t*>(out + s0) = word;
        }
    } else {
        for (int64_t s = threadIdx.x; s < ld; s += blockDim.x) {
            int8_t v = 0;
            if (s < n) {
                const int64_t fi = sidx ? (int64_t)sidx[s] : s;
                v = (int8_t)code_of((rec[fi >> 2] >> (2 * (fi & 3))) & 3);
                if (v != 3) {
                    obs += 1;
                    sum += v;
                    het += (v == 1);
                    hom2 += (v == 2);
                }
            }
            out[s] = v;
        }
    }
    __shared__ int red[4][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        obs += __shfl_xor_sync(0xffffffffu, obs, o);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        het += __shfl_xor_sync(0xffffffffu, het, o);
        hom2 += __shfl_xor_sync(0xffffffffu, hom2, o);
    }
    if (lane == 0) {
        red[0][w] = obs;
        red[1][w] = sum;
        red[2][w] = het;
        red[3][w] = hom2;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        int acc = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) acc += red[threadIdx.x][k];
        counts[j * 4 + threadIdx.x] = acc;
    }
}

// Inverse of the decode: int8 codes (0/1/2, 3 = missing) -> count-A1 2-bit records,
// samples past n padded with "0 copies" (11).
__global__ void pack_codes_kernel(const int8_t* __restrict__ codes, int64_t ldc, int64_t n,
                                  int64_t m, uint8_t* __restrict__ packed, int64_t bps) {
    const int64_t j = blockIdx.x;
    if (j >= m) return;
    for (int64_t q = threadIdx.x; q < bps; q += blockDim.x) {
        uint32_t byte = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int64_t s = 4 * q + e;
            uint32_t bits = 3u;
            if (s < n) {
                const int8_t v = codes[j * ldc + s];
                bits = v == 2 ? 0u : (v == 3 ? 1u : (v == 1 ? 2u : 3u));
            }
            byte |= bits << (2 * e);
        }
        packed[j * bps + q] = (uint8_t)byte;
    }
}

__global__ void impute_f64_kernel(const int8_t* __restrict__ codes, int64_t ldc, int64_t n,
                                  int64_t m, const double* __restrict__ mean,
                                  double* __restrict__ G, int64_t ldg) {
    const int64_t j = blockIdx.y;
    const double mu = mean[j];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int8_t c = codes[j * ldc + i];
        G[j * ldg + i] = (c == 3) ? mu : (double)c;
    }
}

// Centred (sd == NULL) or standardized FP64 batch: x - mean[j] for observed codes, 0 for
// missing ones (imputed to the mean), divided by sd[j] when given (0 where sd[j] == 0).
__global__ void center_f64_kernel(const int8_t* __restrict__ codes, int64_t ldc, int64_t n,
                                  int64_t m, const double* __restrict__ mean,
                                  const double* __restrict__ sd, double* __restrict__ X) {
    const int64_t j = blockIdx.y;
    const double mu = mean[j];
    const double s = sd ? sd[j] : 1.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int8_t c = codes[j * ldc + i];
        const double v = (c == 3) ? 0.0 : ((double)c - mu);
        X[j * n + i] = sd ? (s > 0.0 ? v / s : 0.0) : v;
    }
}

__global__ void symmetrize_scale_kernel(double* K, int64_t n, int64_t ldk, double scale) {
    for (int64_t col = blockIdx.y; col < n; col += gridDim.y) {
        for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
             row += (int64_t)gridDim.x * blockDim.x) {
            if (row >= col) {
                const double v = K[col * ldk + row] * scale;
                K[col * ldk + row] = v;
                if (row != col) K[row * ldk + col] = v;
            }
        }
    }
}

__global__ void threshold_kernel(double* w, int64_t n, double thr) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (fabs(w[i]) < thr) w[i] = 0.0;
    }
}

static dim3 col_grid(int64_t n, int64_t m) {
    const int64_t bx = ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64;
    return dim3((unsigned)(bx > 0 ? bx : 1), (unsigned)m, 1);
}

}  // namespace jb

using namespace jb;

extern "C" {

int32_t jb_version(void) {
    return JB_VERSION_MAJOR * 10000 + JB_VERSION_MINOR * 100 + JB_VERSION_PATCH;
}

int32_t jb_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return JB_E_INVALID;
    strncpy(buf, g_err, len - 1);
    buf[len - 1] = 0;
    return JB_OK;
}

int32_t jb_device_arch(void) {
    int dev = 0;
    JB_CUDA(cudaGetDevice(&dev));
    int major = 0, minor = 0;
    JB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    JB_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
    return major * 10 + minor;
}

int32_t jb_decode_bed(const uint8_t* packed, int64_t bytes_per_snp, int64_t m,
                      const int32_t* sample_idx, int64_t n, int8_t* codes, int64_t ld_codes,
                      int32_t* counts, uintptr_t stream) {
    JB_CHECK_ARG(m >= 0 && n >= 0, "jb_decode_bed: negative size");
    JB_CHECK_ARG(ld_codes >= n, "jb_decode_bed: ld_codes (%lld) < n (%lld)",
                 (long long)ld_codes, (long long)n);
    JB_CHECK_ARG(sample_idx || n <= 4 * bytes_per_snp,
                 "jb_decode_bed: n exceeds the record length");
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(packed && codes && counts, "jb_decode_bed: null pointer");
    JB_CHECK_ARG(m < (1ll << 31), "jb_decode_bed: too many SNPs in one call");
    decode_bed_kernel<<<(unsigned)m, 256, 0, as_stream(stream)>>>(packed, bytes_per_snp, m,
                                                                 sample_idx, n, codes,
                                                                 ld_codes, counts);
    JB_LAUNCH_CHECK("decode_bed_kernel");
    return JB_OK;
}

int32_t jb_pack_codes(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                      uint8_t* packed, int64_t bytes_per_snp, uintptr_t stream) {
    JB_CHECK_ARG(n >= 0 && m >= 0 && ld_codes >= n && 4 * bytes_per_snp >= n,
                 "jb_pack_codes: bad shape");
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(m < (1ll << 31), "jb_pack_codes: too many SNPs");
    pack_codes_kernel<<<(unsigned)m, 128, 0, as_stream(stream)>>>(codes, ld_codes, n, m, packed,
                                                                 bytes_per_snp);
    JB_LAUNCH_CHECK("pack_codes_kernel");
    return JB_OK;
}

int32_t jb_impute_f64(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                      const double* mean, double* G, int64_t ldg, uintptr_t stream) {
    JB_CHECK_ARG(n >= 0 && m >= 0 && ldg >= n && ld_codes >= n, "jb_impute_f64: bad shape");
    if (n == 0 || m == 0) return JB_OK;
    JB_CHECK_ARG(m < 65536, "jb_impute_f64: m must be < 65536 per call");
    impute_f64_kernel<<<col_grid(n, m), 256, 0, as_stream(stream)>>>(codes, ld_codes, n, m,
                                                                     mean, G, ldg);
    JB_LAUNCH_CHECK("impute_f64_kernel");
    return JB_OK;
}

int64_t jb_kinship_f64_workspace_size(int64_t n, int64_t m) { return n * m * 8; }

static int32_t kinship_accumulate(const char* name, const int8_t* codes, int64_t ld_codes, int64_t n,
                                  int64_t m, const double* mean, const double* sd, double* K,
                                  int64_t ldk, void* workspace, int64_t workspace_bytes,
                                  uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && m >= 0 && ldk >= n && ld_codes >= n, "%s: bad shape", name);
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(m < 65536, "%s: m must be < 65536 per call", name);
    JB_CHECK_ARG(workspace_bytes >= jb_kinship_f64_workspace_size(n, m),
                 "%s: workspace too small", name);
    double* X = static_cast<double*>(workspace);
    center_f64_kernel<<<col_grid(n, m), 256, 0, as_stream(stream)>>>(codes, ld_codes, n, m, mean,
                                                                    sd, X);
    JB_LAUNCH_CHECK("center_f64_kernel");
    cublasHandle_t h = cublas_handle();
    if (!h) {
        set_error("cuBLAS handle creation failed");
        return JB_E_LIBRARY;
    }
    // no workspace: the kernel choice must not depend on other streams' work
    cublasStatus_t s = bind_cublas(h, as_stream(stream), nullptr, 0);
    if (s != CUBLAS_STATUS_SUCCESS) return cublas_status(s, "cublasSetStream/Workspace");
    const double one = 1.0;
    s = cublasDsyrk(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, (int)n, (int)m, &one, X, (int)n, &one,
                    K, (int)ldk);
    if (s != CUBLAS_STATUS_SUCCESS) return cublas_status(s, "cublasDsyrk");
    return JB_OK;
}

int32_t jb_kinship_accumulate_f64(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                                  const double* mean, double* K, int64_t ldk, void* workspace,
                                  int64_t workspace_bytes, uintptr_t stream) {
    return kinship_accumulate("jb_kinship_accumulate_f64", codes, ld_codes, n, m, mean, nullptr, K,
                              ldk, workspace, workspace_bytes, stream);
}

int32_t jb_kinship_accumulate_std_f64(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                                      const double* mean, const double* sd, double* K, int64_t ldk,
                                      void* workspace, int64_t workspace_bytes, uintptr_t stream) {
    JB_CHECK_ARG(sd != nullptr, "jb_kinship_accumulate_std_f64: sd is required");
    return kinship_accumulate("jb_kinship_accumulate_std_f64", codes, ld_codes, n, m, mean, sd, K,
                              ldk, workspace, workspace_bytes, stream);
}

int32_t jb_kinship_finalize(double* K, int64_t n, int64_t ldk, double scale, uintptr_t stream) {
    JB_CHECK_ARG(n >= 0 && ldk >= n, "jb_kinship_finalize: bad shape");
    if (n == 0) return JB_OK;
    const int64_t bx = ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64;
    dim3 grid((unsigned)bx, grid_y(n), 1);
    symmetrize_scale_kernel<<<grid, 256, 0, as_stream(stream)>>>(K, n, ldk, scale);
    JB_LAUNCH_CHECK("symmetrize_scale_kernel");
    return JB_OK;
}

// The single-GPU divide-and-conquer solver (cusolverDnXsyevd) rejects matrices whose
// workspace, about 4 n^2 doubles, passes 2^31 elements (n above ~23 000).  Larger n go to
// the cusolverMg solver on a one-device grid, whose workspace size is 64-bit: with one
// device its 1-D column block-cyclic layout is the plain column-major matrix (ld = n).
namespace {
constexpr int64_t kMgColBlock = 256;

// cusolverMg is loaded at its first use, from the directory of the libcusolver the process
// already runs (in a PyTorch process that is PyTorch's own copy), so it pairs with the
// cuBLAS that is loaded; linking it at build time could pair it with another cuBLAS.
struct MgApi {
    decltype(&cusolverMgCreate) create;
    decltype(&cusolverMgDestroy) destroy;
    decltype(&cusolverMgDeviceSelect) device_select;
    decltype(&cusolverMgCreateDeviceGrid) create_grid;
    decltype(&cusolverMgDestroyGrid) destroy_grid;
    decltype(&cusolverMgCreateMatrixDesc) create_desc;
    decltype(&cusolverMgDestroyMatrixDesc) destroy_desc;
    decltype(&cusolverMgSyevd_bufferSize) syevd_buffer_size;
    decltype(&cusolverMgSyevd) syevd;
};

const MgApi* mg_api() {
    static MgApi api;
    static bool ok = false;
    static std::once_flag once;
    std::call_once(once, [] {
        void* lib = nullptr;
        Dl_info info;
        if (dladdr(reinterpret_cast<void*>(&cusolverDnCreate), &info) && info.dli_fname) {
            std::string path(info.dli_fname);
            const size_t slash = path.rfind('/');
            if (slash != std::string::npos) {
                path = path.substr(0, slash + 1) + "libcusolverMg.so.11";
                lib = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
            }
        }
        if (!lib) lib = dlopen("libcusolverMg.so.11", RTLD_NOW | RTLD_LOCAL);
        if (!lib) return;
        auto sym = [&](const char* name) { return dlsym(lib, name); };
        api.create = reinterpret_cast<decltype(api.create)>(sym("cusolverMgCreate"));
        api.destroy = reinterpret_cast<decltype(api.destroy)>(sym("cusolverMgDestroy"));
        api.device_select = reinterpret_cast<decltype(api.device_select)>(sym("cusolverMgDeviceSelect"));
        api.create_grid = reinterpret_cast<decltype(api.create_grid)>(sym("cusolverMgCreateDeviceGrid"));
        api.destroy_grid = reinterpret_cast<decltype(api.destroy_grid)>(sym("cusolverMgDestroyGrid"));
        api.create_desc = reinterpret_cast<decltype(api.create_desc)>(sym("cusolverMgCreateMatrixDesc"));
        api.destroy_desc = reinterpret_cast<decltype(api.destroy_desc)>(sym("cusolverMgDestroyMatrixDesc"));
        api.syevd_buffer_size =
            reinterpret_cast<decltype(api.syevd_buffer_size)>(sym("cusolverMgSyevd_bufferSize"));
        api.syevd = reinterpret_cast<decltype(api.syevd)>(sym("cusolverMgSyevd"));
        ok = api.create && api.destroy && api.device_select && api.create_grid && api.destroy_grid &&
             api.create_desc && api.destroy_desc && api.syevd_buffer_size && api.syevd;
    });
    return ok ? &api : nullptr;
}

// cusolverMg keeps handle-independent state; two of its solves (or workspace queries) from
// different threads at once failed with CUSOLVER_STATUS_INTERNAL_ERROR, so every use is
// serialised on this lock.
std::mutex g_mg_mutex;

struct MgSolver {
    const MgApi* api = mg_api();
    cusolverMgHandle_t h = nullptr;
    cudaLibMgGrid_t grid = nullptr;
    cudaLibMgMatrixDesc_t desc = nullptr;
    ~MgSolver() {
        if (desc) api->destroy_desc(desc);
        if (grid) api->destroy_grid(grid);
        if (h) api->destroy(h);
    }
    cusolverStatus_t init(int64_t n) {
        if (!api) return CUSOLVER_STATUS_NOT_INITIALIZED;  // libcusolverMg not found
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return CUSOLVER_STATUS_INTERNAL_ERROR;
        cusolverStatus_t s = api->create(&h);
        if (s != CUSOLVER_STATUS_SUCCESS) return s;
        int ids[1] = {dev};
        s = api->device_select(h, 1, ids);
        if (s != CUSOLVER_STATUS_SUCCESS) return s;
        int32_t gids[1] = {dev};
        s = api->create_grid(&grid, 1, 1, gids, CUDALIBMG_GRID_MAPPING_COL_MAJOR);
        if (s != CUSOLVER_STATUS_SUCCESS) return s;
        return api->create_desc(&desc, n, n, n, kMgColBlock, CUDA_R_64F, grid);
    }
    // workspace in doubles; A may be null for the query, W is a host array of n doubles
    cusolverStatus_t query(int64_t n, double* A, double* w_host, int64_t* lwork) {
        void* arr[1] = {A};
        return api->syevd_buffer_size(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)n,
                                      arr, 1, 1, desc, w_host, CUDA_R_64F, CUDA_R_64F, lwork);
    }
};

// true when cusolverDnXsyevd takes n; dev_bytes: its device workspace
bool dn_syevd_fits(int64_t n, size_t* dev_bytes) {
    cusolverDnHandle_t h = cusolver_handle();
    cusolverDnParams_t params;
    if (!h || cusolverDnCreateParams(&params) != CUSOLVER_STATUS_SUCCESS) return false;
    size_t host_bytes = 0;
    const cusolverStatus_t s = cusolverDnXsyevd_bufferSize(
        h, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, nullptr, n,
        CUDA_R_64F, nullptr, CUDA_R_64F, dev_bytes, &host_bytes);
    cusolverDnDestroyParams(params);
    return s == CUSOLVER_STATUS_SUCCESS;
}
}  // namespace

int64_t jb_eigh_workspace_size(int64_t n) {
    if (n <= 0) return -1;
    size_t dev_bytes = 0;
    if (dn_syevd_fits(n, &dev_bytes))
        return (int64_t)(((dev_bytes + 255) / 256) * 256) + 256;  // + device info word
    if (n > 2147483647ll) return -1;
    std::lock_guard<std::mutex> lock(g_mg_mutex);
    MgSolver mg;
    std::vector<double> w_host((size_t)n);
    int64_t lwork = 0;
    cusolverStatus_t s = mg.init(n);
    if (s == CUSOLVER_STATUS_SUCCESS) s = mg.query(n, nullptr, w_host.data(), &lwork);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        set_error("eigendecomposition workspace query failed for n = %lld (cusolverMg status %d%s)",
                  (long long)n, (int)s, mg_api() ? "" : "; libcusolverMg.so.11 not found");
        return -1;
    }
    return ((lwork * 8 + 255) / 256) * 256;
}

// Large-n path of jb_eigh_f64 (lda == n): blocking cusolverMgSyevd on this device.
static int32_t eigh_f64_mg(double* A, int64_t n, double* w, double threshold, void* workspace,
                           int64_t workspace_bytes, cudaStream_t st) {
    std::lock_guard<std::mutex> lock(g_mg_mutex);
    MgSolver mg;
    double* w_host = nullptr;  // pinned: valid for the solver as a host or a device address
    JB_CUDA(cudaMallocHost(&w_host, (size_t)n * sizeof(double)));
    int64_t lwork = 0;
    cusolverStatus_t s = mg.init(n);
    if (s == CUSOLVER_STATUS_SUCCESS) s = mg.query(n, A, w_host, &lwork);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        cudaFreeHost(w_host);
        return cusolver_status(s, "cusolverMgSyevd_bufferSize");
    }
    if (workspace_bytes < lwork * 8) {
        cudaFreeHost(w_host);
        set_error("jb_eigh_f64: workspace %lld < required %lld", (long long)workspace_bytes,
                  (long long)(lwork * 8));
        return JB_E_INVALID;
    }
    cudaError_t e = cudaStreamSynchronize(st);  // the solver runs on its own streams
    int info = 0;
    if (e == cudaSuccess) {
        void* arr_a[1] = {A};
        void* arr_w[1] = {workspace};
        s = mg.api->syevd(mg.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)n, arr_a, 1,
                          1, mg.desc, w_host, CUDA_R_64F, CUDA_R_64F, arr_w, lwork, &info);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess && s == CUSOLVER_STATUS_SUCCESS && info == 0)
        e = cudaMemcpyAsync(w, w_host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && s == CUSOLVER_STATUS_SUCCESS && info == 0) e = cudaStreamSynchronize(st);
    cudaFreeHost(w_host);
    if (e != cudaSuccess) return cuda_status(e, "cusolverMg eigendecomposition");
    if (s != CUSOLVER_STATUS_SUCCESS) return cusolver_status(s, "cusolverMgSyevd");
    if (info != 0) {
        set_error("cusolverMgSyevd: info = %d (no convergence or bad argument)", info);
        return JB_E_NUMERIC;
    }
    threshold_kernel<<<64, 256, 0, st>>>(w, n, threshold);
    JB_LAUNCH_CHECK("threshold_kernel");
    return JB_OK;
}

int32_t jb_eigh_f64(double* A, int64_t n, int64_t lda, double* w, double threshold,
                    void* workspace, int64_t workspace_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && lda >= n && A && w, "jb_eigh_f64: bad arguments");
    {
        size_t dn_bytes = 0;
        if (!dn_syevd_fits(n, &dn_bytes)) {
            JB_CHECK_ARG(lda == n && n <= 2147483647ll, "jb_eigh_f64: n = %lld needs lda == n",
                         (long long)n);
            return eigh_f64_mg(A, n, w, threshold, workspace, workspace_bytes, as_stream(stream));
        }
    }
    cusolverDnHandle_t h = cusolver_handle();
    if (!h) {
        set_error("cuSOLVER handle creation failed");
        return JB_E_LIBRARY;
    }
    cusolverStatus_t s = cusolverDnSetStream(h, as_stream(stream));
    if (s != CUSOLVER_STATUS_SUCCESS) return cusolver_status(s, "cusolverDnSetStream");
    cusolverDnParams_t params;
    s = cusolverDnCreateParams(&params);
    if (s != CUSOLVER_STATUS_SUCCESS) return cusolver_status(s, "cusolverDnCreateParams");
    size_t dev_bytes = 0, host_bytes = 0;
    s = cusolverDnXsyevd_bufferSize(h, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                    CUDA_R_64F, A, lda, CUDA_R_64F, w, CUDA_R_64F, &dev_bytes,
                                    &host_bytes);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        cusolverDnDestroyParams(params);
        return cusolver_status(s, "cusolverDnXsyevd_bufferSize");
    }
    const size_t info_off = ((dev_bytes + 255) / 256) * 256;
    if (workspace_bytes < (int64_t)info_off + 256) {
        cusolverDnDestroyParams(params);
        set_error("jb_eigh_f64: workspace %lld < required %lld", (long long)workspace_bytes,
                  (long long)info_off + 256);
        return JB_E_INVALID;
    }
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    int* d_info = reinterpret_cast<int*>(ws + info_off);  // after the solver's bytes
    std::vector<uint8_t> host_ws(host_bytes > 0 ? host_bytes : 1);
    s = cusolverDnXsyevd(h, params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                         CUDA_R_64F, A, lda, CUDA_R_64F, w, CUDA_R_64F, ws, dev_bytes,
                         host_ws.data(), host_bytes, d_info);
    cusolverDnDestroyParams(params);
    if (s != CUSOLVER_STATUS_SUCCESS) return cusolver_status(s, "cusolverDnXsyevd");
    threshold_kernel<<<64, 256, 0, as_stream(stream)>>>(w, n, threshold);
    JB_LAUNCH_CHECK("threshold_kernel");
    int info = 0;
    JB_CUDA(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    JB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (info != 0) {
        set_error("cusolverDnXsyevd: info = %d (no convergence or bad argument)", info);
        return JB_E_NUMERIC;
    }
    return JB_OK;
}

int32_t jb_rotate_f64(const double* U, int64_t n, int64_t ldu, const double* B, int64_t m,
                      int64_t ldb, double* C, int64_t ldc, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && m >= 0 && ldu >= n && ldb >= n && ldc >= n, "jb_rotate_f64: bad shape");
    if (m == 0) return JB_OK;
    cublasHandle_t h = cublas_handle();
    if (!h) {
        set_error("cuBLAS handle creation failed");
        return JB_E_LIBRARY;
    }
    // no workspace: the kernel choice (and rounding) of U^T B must not depend on other
    // streams' work -- U^T W and U^T y feed every SNP's search
    cublasStatus_t s = bind_cublas(h, as_stream(stream), nullptr, 0);
    if (s != CUBLAS_STATUS_SUCCESS) return cublas_status(s, "cublasSetStream/Workspace");
    const double one = 1.0, zero = 0.0;
    s = cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)n, (int)m, (int)n, &one, U, (int)ldu, B,
                    (int)ldb, &zero, C, (int)ldc);
    if (s != CUBLAS_STATUS_SUCCESS) return cublas_status(s, "cublasDgemm");
    return JB_OK;
}

}  // extern "C"
