// Mixed-precision eigenvector rotation x~ = U^T g on INT8 tensor cores.
//
// Each eigenvector u_i (column i of U) is scaled by s_i = max_k |U_ki| / 127 and split
// into four signed 8-bit digit planes in base 254, U_ki = s_i * sum_{t<4} q_t(k,i) 254^-t
// (+ error below s_i * 0.5 * 254^-3, i.e. ~2.4e-10 of max |U_ki|): with round-to-nearest
// digits every remainder lies in [-0.5, 0.5], so the next digit (remainder * 254) stays
// within [-127, 127].  Genotype calls are exact int8 values, so every digit product
// C_t = q_t^T z accumulates exactly in int32 on tcgen05 (kind::i8; |C_t| <= 254 n), and the
// epilogue recombines  x~_i = s_i * sum_t 254^-t C_t  in FP64.
//
// Missing calls are mean-imputed without centring (src/jamma/lmm/runner_streaming.py:
// 427-434): g_j = z_j + mu_j m_j with m_j the missing mask, so  x~ = U^T z + mu_j U^T m.
// The B operand therefore pairs, per block of 128 SNPs, their 128 call rows with their
// 128 mask rows; the epilogue forms  C^z + mu_j C^m  before recombining.  Chunks without
// missing calls use the calls directly (256 SNPs per tile).
//
// A-operand layout (digits along M): tile row r of eigenvector block b holds digit
// t = r / 32 of eigenvector 32 b + r % 32, so one 128 x 256 accumulator carries all four
// digits of 32 eigenvectors; TMEM lane quarter q = digit q, and the four epilogue warps
// exchange their FP64 digit contributions through shared memory.
#include "jb_common.cuh"
#include "jb_gemm_i8.cuh"
#include "jb_rotate_i8.cuh"

#include <atomic>

namespace jb {
namespace tc {

int32_t make_map_i8(CUtensorMap* map, const void* base, int64_t rows, int64_t k, int64_t ld,
                    int box_rows);
int num_sms();

constexpr double kDigitBase = 254.0;
// 254^-t, t = 0..3, for the FP64 recombination of the digit products
__device__ __constant__ double kDigitWeight[4] = {1.0, 1.0 / 254.0, 1.0 / (254.0 * 254.0),
                                                  1.0 / (254.0 * 254.0 * 254.0)};
constexpr int kRotBN = 256;
constexpr int kRotStages = 4;
constexpr int kRotPairStages = 6;
constexpr int kRotEpiSmem = 4 * 32 * 32 * 8;  // [digit][column][eigvec] doubles

// ---------------------------------------------------------------- digit split
__global__ void ozaki_scale_kernel(const double* __restrict__ U, int64_t n, int64_t ldu,
                                   double* __restrict__ scale) {
    const int64_t i = blockIdx.x;
    const double* col = U + i * ldu;
    double mx = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) mx = fmax(mx, fabs(col[k]));
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        scale[i] = m;  // max |U_ki|; 0 for an all-zero column
    }
}

__global__ void ozaki_split_kernel(const double* __restrict__ U, int64_t n, int64_t ldu,
                                   const double* __restrict__ smax, int8_t* __restrict__ A,
                                   int64_t lda) {
    const int64_t i = blockIdx.x;  // eigenvector
    const double s = smax[i];
    const double inv = s > 0.0 ? 127.0 / s : 0.0;
    const int64_t base = (i / 32) * 128 + (i % 32);
    for (int64_t k = threadIdx.x; k < lda; k += blockDim.x) {
        int8_t q[4] = {0, 0, 0, 0};
        if (k < n) {
            double a = U[i * ldu + k] * inv;  // |a| <= 127
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const double r = rint(a);
                q[t] = (int8_t)r;             // |r| <= 127
                a = (a - r) * kDigitBase;     // a - r exact, |a - r| <= 0.5 -> |a| <= 127
            }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) A[(base + 32 * t) * lda + k] = q[t];
    }
}

// ---------------------------------------------------------------- B operand
// Paired layout: block b of 128 SNPs occupies B rows [256 b, 256 b + 128) with the calls
// (missing -> 0) and [256 b + 128, 256 b + 256) with the missing masks.
__global__ void rot_pack_pairs_kernel(const int8_t* __restrict__ codes, int64_t ldc, int64_t n,
                                      int64_t m, int8_t* __restrict__ B, int64_t ldb) {
    const int64_t j = blockIdx.x;
    const int64_t rz = (j / 128) * 256 + (j % 128);
    const int64_t rm = rz + 128;
    const bool vec = ((ldc & 3) == 0) && ((ldb & 3) == 0);
    for (int64_t k = 4 * (int64_t)threadIdx.x; k < ldb; k += 4 * (int64_t)blockDim.x) {
        uint32_t c4 = 0;
        if (j < m) {
            if (vec && k + 4 <= n) {
                c4 = *reinterpret_cast<const uint32_t*>(codes + j * ldc + k);
            } else {
                for (int q = 0; q < 4; ++q)
                    if (k + q < n) c4 |= (uint32_t)(uint8_t)codes[j * ldc + k + q] << (8 * q);
            }
        }
        // per byte: code 3 (missing) -> call 0, mask 1; else call = code, mask 0
        const uint32_t lo = c4 & 0x01010101u, hi = (c4 >> 1) & 0x01010101u;
        const uint32_t mk = lo & hi;
        const uint32_t z = c4 & ~(mk * 3u);
        if (vec) {
            *reinterpret_cast<uint32_t*>(B + rz * ldb + k) = z;
            *reinterpret_cast<uint32_t*>(B + rm * ldb + k) = mk;
        } else {
            for (int q = 0; q < 4 && k + q < ldb; ++q) {
                B[rz * ldb + k + q] = (int8_t)((z >> (8 * q)) & 0xff);
                B[rm * ldb + k + q] = (int8_t)((mk >> (8 * q)) & 0xff);
            }
        }
    }
}

// ---------------------------------------------------------------- epilogue
template <bool PAIRED>
struct RotEpi {
    static constexpr int kSmem = kRotEpiSmem;
    double* X;             // x~ (n x m, column-major, ld ldx)
    int64_t ldx;
    const double* smax;    // per-eigenvector max |U_ki|
    const double* mu;      // per-SNP imputation mean (PAIRED only)
    int n;
    int m;
    __device__ __forceinline__ void run(int mb, int nb, uint32_t taddr, int q, int lane,
                                        uint8_t* smem) const {
        double* S = reinterpret_cast<double*>(smem);  // [4][32][32]
        const int i = mb * 32 + lane;                 // eigenvector of this lane (any digit)
        constexpr int kCols = PAIRED ? 128 : 256;
        const int j_base = nb * kCols;
        const double w = kDigitWeight[q];              // 254^-q
        double sc = 0.0;
        if (i < n) sc = smax[i] * (1.0 / 127.0);
#pragma unroll 1
        for (int c0 = 0; c0 < kCols; c0 += 32) {
            uint32_t vz[32];
            tmem_ld32(taddr + (uint32_t)c0, vz);
            double val[32];
#pragma unroll
            for (int t = 0; t < 32; ++t) val[t] = (double)(int32_t)vz[t] * w;
            if (PAIRED) {
                uint32_t vm[32];
                tmem_ld32(taddr + 128u + (uint32_t)c0, vm);
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    const int j = j_base + c0 + t;
                    const double u = j < m ? __ldg(mu + j) : 0.0;
                    val[t] = fma(u, (double)(int32_t)vm[t] * w, val[t]);
                }
            }
#pragma unroll
            for (int t = 0; t < 32; ++t) S[(q * 32 + t) * 32 + lane] = val[t];
            asm volatile("bar.sync 1, 128;" ::: "memory");
#pragma unroll
            for (int cc = 0; cc < 8; ++cc) {
                const int t = q * 8 + cc;
                const int j = j_base + c0 + t;
                // smallest digit first: ((d3 + d2) + d1) + d0
                const double x = ((S[(3 * 32 + t) * 32 + lane] + S[(2 * 32 + t) * 32 + lane]) +
                                  S[(1 * 32 + t) * 32 + lane]) +
                                 S[(0 * 32 + t) * 32 + lane];
                if (i < n && j < m) X[(int64_t)j * ldx + i] = x * sc;
            }
            asm volatile("bar.sync 1, 128;" ::: "memory");
        }
    }
};

// Tiles over (eigenvector blocks of 32, SNP blocks) in groups of GM x GN (GN SNP blocks
// per group column, groups visited column by column), one thread per tile: tile (mb, nb)
// sits at its closed-form position in that order.  The group shape sets which A (digit)
// and B (calls) slices the persistent CTAs share in L2 at a time.
__global__ void rot_tiles_kernel(int MB, int NB, int GM, int GN, Tile* out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)MB * NB) return;
    const int mb = (int)(t / NB), nb = (int)(t % NB);
    const int gc = nb / GN, gr = mb / GM;
    const int w = NB - gc * GN < GN ? NB - gc * GN : GN;  // width of this group column
    const int64_t k = (int64_t)MB * GN * gc + (int64_t)gr * GM * w + (int64_t)(mb - gr * GM) * w +
                      (nb - gc * GN);
    out[k] = Tile{mb, nb};
}

}  // namespace tc
}  // namespace jb

using namespace jb;
using namespace jb::tc;

namespace jb {
namespace tc {
using RotSmem = GemmSmem<kRotBN, kRotStages, kRotEpiSmem>;

// Tile-group shape of the rotation schedule (jb_rotate_set_schedule; the autotuner's knob)
// and the GEMM variant (jb_rotate_set_kernel: 0 = one CTA per tile, 1 = CTA pairs).
std::atomic<int> g_group_m{9}, g_group_n{16};
std::atomic<int> g_rot_kernel{0};
using PairRotSmem = PairSmem<kRotPairStages, kRotEpiSmem>;

template <bool P>
int32_t launch_rot_pair(const CUtensorMap& ta, const CUtensorMap& tb, const Tile* tiles,
                        int n_tiles, int num_kb, const RotEpi<P>& epi, int* status,
                        cudaStream_t st) {
    auto kern = i8_gemm_pair_kernel<kRotPairStages, RotEpi<P>>;
    JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 PairRotSmem::TOTAL));
    // persistent: as many pairs as can be resident at once (clusters need two SMs of one
    // GPC); queried once per device and kernel, so launches inside graph capture skip it
    static std::atomic<int> cached[2][64];
    int dev = 0;
    JB_CUDA(cudaGetDevice(&dev));
    int resident = dev < 64 ? cached[P ? 1 : 0][dev].load(std::memory_order_relaxed) : 0;
    if (resident <= 0) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(2 * (num_sms() / 2)));
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = PairRotSmem::TOTAL;
        cfg.stream = st;
        JB_CUDA(cudaOccupancyMaxActiveClusters(&resident, kern, &cfg));
        JB_CHECK_ARG(resident >= 1, "rotation: no CTA pair fits on the device");
        if (dev < 64) cached[P ? 1 : 0][dev].store(resident, std::memory_order_relaxed);
    }
    const int pairs = n_tiles < resident ? n_tiles : resident;
    kern<<<2 * pairs, kThreads, PairRotSmem::TOTAL, st>>>(ta, tb, tiles, n_tiles, num_kb, epi,
                                                         status);
    JB_LAUNCH_CHECK("i8_gemm_pair_kernel<rotate>");
    return JB_OK;
}

int32_t launch_group_tiles(int MB, int NB, int GM, int GN, Tile* out, cudaStream_t st) {
    const int64_t n_tiles = (int64_t)MB * NB;
    rot_tiles_kernel<<<(unsigned)ceil_div(n_tiles, 256), 256, 0, st>>>(MB, NB, GM, GN, out);
    JB_LAUNCH_CHECK("rot_tiles_kernel");
    return JB_OK;
}

OzakiLayout ozaki_layout(int64_t n_out, int64_t n_k) {
    OzakiLayout L;
    L.lda = (n_k + 127) / 128 * 128;
    L.rows = ceil_div(n_out, 32) * 128;
    L.a_off = 0;
    L.s_off = ((L.rows * L.lda + 255) / 256) * 256;
    L.total = L.s_off + ((n_out * 8 + 255) / 256) * 256;
    return L;
}

RotChunkLayout rot_chunk_layout(int64_t n, int64_t m) {
    RotChunkLayout L;
    L.ldb = (n + 127) / 128 * 128;
    const int64_t MB = ceil_div(n, 32), NB = ceil_div(m, 128);
    L.status = 0;
    L.tiles = 256;
    L.b_off = L.tiles + ((MB * NB * (int64_t)sizeof(Tile) + 255) / 256) * 256;
    L.total = L.b_off + NB * 256 * L.ldb;
    return L;
}

int32_t ozaki_split(const double* V, int64_t n_k, int64_t n_out, int64_t ldv, uint8_t* ws,
                    cudaStream_t st) {
    const OzakiLayout L = ozaki_layout(n_out, n_k);
    double* smax = reinterpret_cast<double*>(ws + L.s_off);
    int8_t* A = reinterpret_cast<int8_t*>(ws + L.a_off);
    // rows of column blocks past n_out and K padding stay zero
    JB_CUDA(cudaMemsetAsync(A, 0, (size_t)(L.rows * L.lda), st));
    ozaki_scale_kernel<<<(unsigned)n_out, 256, 0, st>>>(V, n_k, ldv, smax);
    JB_LAUNCH_CHECK("ozaki_scale_kernel");
    ozaki_split_kernel<<<(unsigned)n_out, 256, 0, st>>>(V, n_k, ldv, smax, A, L.lda);
    JB_LAUNCH_CHECK("ozaki_split_kernel");
    return JB_OK;
}

int32_t rotate_i8_gemm(const uint8_t* ozaki_ws, int64_t n_out, int64_t n_k, const int8_t* B,
                       int64_t b_rows, int64_t ldb, bool paired, int64_t m, const double* mean,
                       double* X, int64_t ldx, Tile* tiles, int* status, cudaStream_t st) {
    const OzakiLayout OL = ozaki_layout(n_out, n_k);
    const int8_t* A = reinterpret_cast<const int8_t*>(ozaki_ws + OL.a_off);
    const double* smax = reinterpret_cast<const double*>(ozaki_ws + OL.s_off);
    const int MB = (int)ceil_div(n_out, 32);
    const int NB = (int)ceil_div(m, paired ? 128 : 256);
    const int num_kb = (int)ceil_div(n_k, kBK);
    CUtensorMap ta, tb;
    int32_t rc = make_map_i8(&ta, A, OL.rows, n_k, OL.lda, kBM);
    if (rc) return rc;
    if (g_rot_kernel.load(std::memory_order_relaxed) == 1) {
        // CTA pairs: tile = 2 eigenvector blocks (one per CTA) x 256 B rows (128 per CTA)
        rc = make_map_i8(&tb, B, b_rows, n_k, ldb, 128);
        if (rc) return rc;
        const int MB2 = (MB + 1) / 2;
        const int n_pairs_tiles = MB2 * NB;
        rot_tiles_kernel<<<(unsigned)ceil_div((int64_t)n_pairs_tiles, 256), 256, 0, st>>>(
            MB2, NB, g_group_m.load(std::memory_order_relaxed),
            g_group_n.load(std::memory_order_relaxed), tiles);
        JB_LAUNCH_CHECK("rot_tiles_kernel");
        if (paired)
            return launch_rot_pair<true>(ta, tb, tiles, n_pairs_tiles, num_kb,
                                         RotEpi<true>{X, ldx, smax, mean, (int)n_out, (int)m},
                                         status, st);
        return launch_rot_pair<false>(ta, tb, tiles, n_pairs_tiles, num_kb,
                                      RotEpi<false>{X, ldx, smax, nullptr, (int)n_out, (int)m},
                                      status, st);
    }
    const int n_tiles = MB * NB;
    rc = make_map_i8(&tb, B, b_rows, n_k, ldb, kRotBN);
    if (rc) return rc;
    rot_tiles_kernel<<<(unsigned)ceil_div((int64_t)n_tiles, 256), 256, 0, st>>>(
        MB, NB, g_group_m.load(std::memory_order_relaxed), g_group_n.load(std::memory_order_relaxed),
        tiles);
    JB_LAUNCH_CHECK("rot_tiles_kernel");
    const int grid = n_tiles < num_sms() ? n_tiles : num_sms();
    if (paired) {
        auto kern = i8_gemm_kernel<kRotBN, kRotStages, RotEpi<true>>;
        JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     RotSmem::TOTAL));
        RotEpi<true> epi{X, ldx, smax, mean, (int)n_out, (int)m};
        kern<<<grid, kThreads, RotSmem::TOTAL, st>>>(ta, tb, tiles, n_tiles, num_kb, epi, status);
    } else {
        auto kern = i8_gemm_kernel<kRotBN, kRotStages, RotEpi<false>>;
        JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     RotSmem::TOTAL));
        RotEpi<false> epi{X, ldx, smax, nullptr, (int)n_out, (int)m};
        kern<<<grid, kThreads, RotSmem::TOTAL, st>>>(ta, tb, tiles, n_tiles, num_kb, epi, status);
    }
    JB_LAUNCH_CHECK("i8_gemm_kernel<rotate>");
    return JB_OK;
}

cudaError_t rotate_pipeline_test_mode(int skip_loads, unsigned long long wait_limit_ns) {
    return pipeline_test_mode(skip_loads, wait_limit_ns);
}

}  // namespace tc
}  // namespace jb

extern "C" {

int64_t jb_ozaki_workspace_size(int64_t n) {
    if (n <= 0) return -1;
    return ozaki_layout(n, n).total;
}

int32_t jb_ozaki_prepare(const double* U, int64_t n, int64_t ldu, void* ozaki_ws,
                         int64_t ozaki_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && ldu >= n && U, "jb_ozaki_prepare: bad arguments");
    JB_CHECK_ARG(n < (1ll << 31), "jb_ozaki_prepare: n too large");
    const OzakiLayout L = ozaki_layout(n, n);
    JB_CHECK_ARG(ozaki_ws && ozaki_bytes >= L.total, "jb_ozaki_prepare: workspace too small");
    return ozaki_split(U, n, n, ldu, static_cast<uint8_t*>(ozaki_ws), as_stream(stream));
}

int64_t jb_rotate_i8_workspace_size(int64_t n, int64_t m) {
    if (n <= 0 || m <= 0) return -1;
    return rot_chunk_layout(n, m).total;
}

int32_t jb_rotate_i8(const void* ozaki_ws, int64_t n, const int8_t* codes, int64_t ld_codes,
                     int64_t m, const double* mean, int32_t has_missing, double* X, int64_t ldx,
                     void* workspace, int64_t workspace_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && m >= 0 && ld_codes >= n && ldx >= n, "jb_rotate_i8: bad shape");
    JB_CHECK_ARG(n < (1ll << 23), "jb_rotate_i8: n too large for exact int32 digit sums");
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(ozaki_ws && codes && X, "jb_rotate_i8: null pointer");
    JB_CHECK_ARG(!has_missing || mean, "jb_rotate_i8: mean needed when calls are missing");
    const RotChunkLayout L = rot_chunk_layout(n, m);
    JB_CHECK_ARG(workspace && workspace_bytes >= L.total, "jb_rotate_i8: workspace too small");
    cudaStream_t st = as_stream(stream);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    int* status = reinterpret_cast<int*>(ws + L.status);
    Tile* tiles = reinterpret_cast<Tile*>(ws + L.tiles);
    const uint8_t* ows = static_cast<const uint8_t*>(ozaki_ws);
    const int NB = (int)ceil_div(m, has_missing ? 128 : 256);
    JB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    if (has_missing) {
        int8_t* B = reinterpret_cast<int8_t*>(ws + L.b_off);
        rot_pack_pairs_kernel<<<(unsigned)(NB * 128), 256, 0, st>>>(codes, ld_codes, n, m, B, L.ldb);
        JB_LAUNCH_CHECK("rot_pack_pairs_kernel");
        return rotate_i8_gemm(ows, n, n, B, (int64_t)NB * 256, L.ldb, true, m, mean, X, ldx, tiles,
                              status, st);
    }
    // no missing calls: the decoded codes are the calls themselves
    return rotate_i8_gemm(ows, n, n, codes, m, ld_codes, false, m, nullptr, X, ldx, tiles, status,
                          st);
}

int32_t jb_rotate_set_schedule(int32_t group_m, int32_t group_n) {
    JB_CHECK_ARG(group_m >= 1 && group_m <= 1024 && group_n >= 1 && group_n <= 1024,
                 "jb_rotate_set_schedule: group sizes must be in 1..1024");
    g_group_m.store(group_m, std::memory_order_relaxed);
    g_group_n.store(group_n, std::memory_order_relaxed);
    return JB_OK;
}

int32_t jb_rotate_set_kernel(int32_t variant) {
    JB_CHECK_ARG(variant == 0 || variant == 1, "jb_rotate_set_kernel: variant must be 0 or 1");
    g_rot_kernel.store(variant, std::memory_order_relaxed);
    return JB_OK;
}

int32_t jb_rotate_get_kernel(void) { return g_rot_kernel.load(std::memory_order_relaxed); }

int32_t jb_rotate_get_schedule(int32_t* group_m, int32_t* group_n) {
    JB_CHECK_ARG(group_m && group_n, "jb_rotate_get_schedule: null pointer");
    *group_m = g_group_m.load(std::memory_order_relaxed);
    *group_n = g_group_n.load(std::memory_order_relaxed);
    return JB_OK;
}

int32_t jb_rotate_status(const void* workspace, int32_t* out, uintptr_t stream) {
    JB_CHECK_ARG(workspace && out, "jb_rotate_status: null pointer");
    JB_CUDA(cudaMemcpyAsync(out, workspace, sizeof(int32_t), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    JB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return JB_OK;
}

}  // extern "C"
