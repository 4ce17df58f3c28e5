// INT8 tensor-core kinship Gram (mixed-precision form of GEMMA -gk 1) and its FP64
// centring / missing-genotype corrections.
//
// Genotype calls 0/1/2 are exact in int8 and Z Z^T accumulates exactly in int32, so the
// Gram is bit-exact whatever the tiling.  With mu_j the float64 mean of SNP j over
// observed samples and M the missing-call mask (Z = 0 where missing), the centred,
// mean-imputed matrix of jamma's impute_and_center (src/jamma/kinship/missing.py:22-61)
// is Xc = Z - 1 mu^T + M diag(mu), hence
//
//   p K = Z Z^T - a 1^T - 1 a^T + (sum mu^2) 1 1^T - b 1^T - 1 b^T + R + R^T + T
//   a = Z mu,  b = M mu^2,  R = Z diag(mu) M^T,  T = M diag(mu^2) M^T
//
// T is symmetric, so R + R^T + T = Q + Q^T with Q = R + T/2: one n x n buffer holds both
// sparse terms.  The dense Z Z^T runs on tcgen05 (kind::i8); the vectors and Q are FP64
// on the CUDA cores.
#include "jb_common.cuh"
#include "jb_gemm_i8.cuh"
#include "jb_rotate_i8.cuh"

#include <mutex>
#include <vector>

namespace jb {
namespace tc {

// ---------------------------------------------------------------- tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// K-major int8 matrix `rows x k` with row stride ld bytes; box = 128 (K) x box_rows.
int32_t make_map_i8(CUtensorMap* map, const void* base, int64_t rows, int64_t k, int64_t ld,
                    int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is unavailable from the driver");
        return JB_E_CUDA;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld & 15)) {
        set_error("TMA operand needs a 16-byte aligned base and row stride (ld=%lld)",
                  (long long)ld);
        return JB_E_INVALID;
    }
    cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return JB_E_CUDA;
    }
    return JB_OK;
}

int num_sms() {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

// ---------------------------------------------------------------- Gram epilogue
struct GramEpi {
    static constexpr int kSmem = 0;
    int32_t* C;
    int64_t ldc;
    int n;
    __device__ __forceinline__ void run(int mb, int nb, uint32_t taddr, int q, int lane,
                                        uint8_t*) const {
        const int i = mb * kBM + 32 * q + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < 256; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(taddr + (uint32_t)c0, v);
            const int j0 = nb * 256 + c0;
            if (i < n) {
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    if (j0 + t < n) C[(int64_t)(j0 + t) * ldc + i] = (int32_t)v[t];
                }
            }
        }
    }
};

// Upper-triangle tiles (128-row x 256-column blocks touching col >= row), visited in
// groups of GM x GN tiles so that concurrently running CTAs share A and B row blocks.
__host__ __device__ inline int gram_tiles(int MB, int NB, Tile* out) {
    const int GM = 16, GN = 8;
    int k = 0;
    for (int gm = 0; gm < MB; gm += GM)
        for (int gn = 0; gn < NB; gn += GN)
            for (int nb = gn; nb < NB && nb < gn + GN; ++nb)
                for (int mb = gm; mb < MB && mb < gm + GM; ++mb)
                    if (kBM * mb <= 256 * nb + 255) {
                        if (out) out[k] = Tile{mb, nb};
                        ++k;
                    }
    return k;
}

__global__ void gram_tiles_kernel(int MB, int NB, Tile* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) gram_tiles(MB, NB, out);
}

// ---------------------------------------------------------------- layout kernels
// SNP-major codes (m x ldc, 3 = missing) -> sample-major int8 calls Zs[i, col0 + j]
// (missing -> 0), through 32x32 shared-memory tiles.
// Optionally also the raw codes Cs[i, j] (3 kept) of this chunk, sample-major.
__global__ void codes_to_sample_major_kernel(const int8_t* __restrict__ codes, int64_t ldc,
                                             int64_t n, int64_t m, int8_t* __restrict__ Zs,
                                             int64_t ldz, int64_t col0, int8_t* __restrict__ Cs,
                                             int64_t ldcs) {
    __shared__ int8_t t[32][33];
    const int64_t j0 = (int64_t)blockIdx.x * 32, i0 = (int64_t)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int64_t j = j0 + r, i = i0 + tx;
        t[r][tx] = (j < m && i < n) ? codes[j * ldc + i] : (int8_t)0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + r, j = j0 + tx;
        if (i < n && j < m) {
            const int8_t v = t[tx][r];
            if (Zs) Zs[i * ldz + col0 + j] = (v == 3) ? (int8_t)0 : v;
            if (Cs) Cs[i * ldcs + j] = v;
        }
    }
}

// The same transpose for Zs alone when codes and Zs allow 4-byte accesses: 64 SNPs x 64
// samples per CTA, every thread loading 4 samples of one SNP and storing 4 SNPs of one
// sample as one uint32 each.
__global__ void __launch_bounds__(256) codes_to_sample_major_vec_kernel(
    const int8_t* __restrict__ codes, int64_t ldc, int64_t n, int64_t m, int8_t* __restrict__ Zs,
    int64_t ldz, int64_t col0) {
    __shared__ uint32_t t[64][17];  // t[j][i / 4]: samples i..i+3 of SNP j
    const int64_t j0 = (int64_t)blockIdx.x * 64, i0 = (int64_t)blockIdx.y * 64;
    for (int r = threadIdx.x; r < 64 * 16; r += 256) {
        const int jj = r >> 4, ii = (r & 15) * 4;
        const int64_t j = j0 + jj, i = i0 + ii;
        uint32_t v = 0u;
        if (j < m) {
            const int8_t* p = codes + j * ldc + i;
            if (i + 4 <= n)
                v = __ldg(reinterpret_cast<const uint32_t*>(p));
            else
                for (int e = 0; e < 4; ++e)
                    if (i + e < n) v |= (uint32_t)(uint8_t)p[e] << (8 * e);
        }
        t[jj][ii >> 2] = v;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < 64 * 16; r += 256) {
        const int ii = r >> 4, jq = (r & 15) * 4;  // sample ii, SNPs jq..jq+3
        const int64_t i = i0 + ii, j = j0 + jq;
        if (i >= n || j >= m) continue;
        uint32_t w = 0u;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            uint32_t b = (t[jq + e][ii >> 2] >> (8 * (ii & 3))) & 0xffu;
            w |= (b == 3u ? 0u : b) << (8 * e);  // missing -> 0
        }
        int8_t* q = Zs + i * ldz + col0 + j;
        if (j + 4 <= m)
            *reinterpret_cast<uint32_t*>(q) = w;
        else
            for (int e = 0; j + e < m; ++e) q[e] = (int8_t)(w >> (8 * e));
    }
}

// a_i = sum_j Z_ij mu_j and b_i = sum_{j missing at i} mu_j^2 from SNP-major codes, in
// two deterministic stages: block (256 samples) x (256 SNPs) partial sums, then an
// ordered sum over the SNP blocks (no atomics, so results are bit-reproducible).
__global__ void kin_vectors_partial_kernel(const int8_t* __restrict__ codes, int64_t ldc,
                                           int64_t n, int64_t m, int vec,
                                           const double* __restrict__ mu,
                                           double* __restrict__ pa, double* __restrict__ pb) {
    const int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;  // 4 samples
    const int64_t jb = blockIdx.y;
    if (i0 >= n) return;
    double sa[4] = {0.0, 0.0, 0.0, 0.0}, sb[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t j0 = jb * 256, j1 = j0 + 256 < m ? j0 + 256 : m;
    const bool full = vec && i0 + 4 <= n;
    for (int64_t j = j0; j < j1; ++j) {
        const int8_t* p = codes + j * ldc + i0;
        uint32_t v = 0u;
        if (full)
            v = __ldg(reinterpret_cast<const uint32_t*>(p));
        else
            for (int e = 0; e < 4; ++e)
                if (i0 + e < n) v |= (uint32_t)(uint8_t)p[e] << (8 * e);
        const double u = __ldg(mu + j);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t c = (v >> (8 * e)) & 0xffu;
            if (c == 3u)
                sb[e] = fma(u, u, sb[e]);
            else
                sa[e] = fma((double)c, u, sa[e]);
        }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (i0 + e < n) {
            pa[jb * n + i0 + e] = sa[e];
            pb[jb * n + i0 + e] = sb[e];
        }
    }
}

__global__ void kin_vectors_reduce_kernel(int64_t n, int64_t nblk, const double* __restrict__ pa,
                                          const double* __restrict__ pb, double* __restrict__ a,
                                          double* __restrict__ b) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sa = 0.0, sb = 0.0;
    for (int64_t k = 0; k < nblk; ++k) {
        sa += pa[k * n + i];
        sb += pb[k * n + i];
    }
    a[i] += sa;
    b[i] += sb;
}

// Missing-call terms for one SNP chunk (at most kSpMaxChunk SNPs):
//   Q[i, k] += R_ik + T_ik / 2,   R_ik = sum_{j in miss(k)} mu_j z_ij,
//                                 T_ik = sum_{j in miss(k) and miss(i)} mu_j^2
// (z_ij the 0/1/2 call, 0 where missing).  R is n x nnz(M) multiply-adds: with 1 % of calls
// missing that is 1 % of a dense Z diag(mu) M^T, so it runs on the FP64 pipe from
// registers rather than densely on the tensor cores.
//
// kin_sp_words_kernel (one warp per SNP): the chunk's calls as "dosage words", 16 samples
// per uint32, 2 bits each: the call 0/1/2, or 3 where it is missing.
//
// kin_sp_kernel: one CTA per (sample k, block b of 4096 samples i).  The CTA turns k's
// missing-SNP bitmask into an increasing list in shared memory, then walks it once with
// every thread owning 16 consecutive samples i: per SNP j one dosage word, and per sample
// one FMA of mu_j with the word's 2-bit value c as the double 4 + c.  A missing call
// (c = 3) adds 3 mu_j more than R wants; it also marks the (i, k, j) triple of T.  Two
// bit operations per word find the missing calls, and for each of them a rare branch adds
// mu_j^2/2 - 3 mu_j into the sample's slot in shared memory (thread-private, summed in SNP
// order).  So R + T/2 comes out of one walk with no per-SNP lists and no atomics.
constexpr int kSpThreads = 256;
constexpr int kSpSpt = 16;                      // samples per thread = one dosage word
constexpr int kSpBlock = kSpThreads * kSpSpt;  // samples per CTA
constexpr int kSpWords = kSpBlock / 16;        // dosage words per CTA
constexpr int kSpMaxChunk = 16384;             // SNPs per call (list in shared memory)

struct SpSmem {
    double corr[kSpSpt][kSpThreads];  // per-thread missing-call terms, [sample][thread]
    uint16_t jl[kSpMaxChunk];         // k's missing SNPs, increasing
    int warp_sum[kSpThreads / 32];
};

// 16 samples s0..s0+15 of one SNP row of int8 codes (0/1/2 calls, 3 missing; samples at
// or beyond n read as call 0): z = the calls, 2 bits each (missing -> 0); miss = bit 2q
// set where sample s0 + q is missing.
__device__ __forceinline__ void sp_load16(const int8_t* __restrict__ row, int64_t s0, int64_t n,
                                          bool vec, uint32_t& z, uint32_t& miss) {
    uint32_t x[4] = {0u, 0u, 0u, 0u};
    if (vec && s0 + 16 <= n) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(row + s0));
        x[0] = v.x;
        x[1] = v.y;
        x[2] = v.z;
        x[3] = v.w;
    } else {
        for (int q = 0; q < 16; ++q)
            if (s0 + q < n) x[q >> 2] |= (uint32_t)(uint8_t)row[s0 + q] << (8 * (q & 3));
    }
    z = 0u;
    miss = 0u;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const uint32_t m3 = __vcmpeq4(x[e], 0x03030303u);  // 0xff in each missing byte
        const uint32_t c = x[e] & ~m3 & 0x03030303u;
        const uint32_t pz = (c & 0x3u) | ((c >> 6) & 0xCu) | ((c >> 12) & 0x30u) | ((c >> 18) & 0xC0u);
        const uint32_t pm = (m3 & 0x1u) | ((m3 >> 6) & 0x4u) | ((m3 >> 12) & 0x10u) | ((m3 >> 18) & 0x40u);
        z |= pz << (8 * e);
        miss |= pm << (8 * e);
    }
}

__global__ void __launch_bounds__(256) kin_sp_words_kernel(const int8_t* __restrict__ codes,
                                                           int64_t ldc, int64_t n, int64_t m,
                                                           int64_t wpr, int vec,
                                                           uint32_t* __restrict__ zb) {
    const int64_t j = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= m) return;  // warp-uniform
    const int8_t* row = codes + j * ldc;
    for (int64_t wi = lane; wi < wpr; wi += 32) {
        uint32_t z, miss;
        sp_load16(row, wi * 16, n, vec != 0, z, miss);
        zb[j * wpr + wi] = z | miss | (miss << 1);  // missing -> 3
    }
}

// Each sample's missing SNPs of the chunk as bitmasks (mask[k * words + w], bit b = SNP
// 32 w + b missing at sample k) from the SNP-major codes: a warp takes a tile of 32 SNPs x
// 32 samples, each lane the 32 calls of one SNP, and 32 ballots transpose the bit tile.
__global__ void __launch_bounds__(256) kin_mask_kernel(const int8_t* __restrict__ codes,
                                                       int64_t ldc, int64_t n, int64_t m, int vec,
                                                       uint32_t* __restrict__ mask, int64_t words) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t jt = blockIdx.x;
    const int64_t s0 = ((int64_t)blockIdx.y * 8 + warp) * 32;
    if (s0 >= n) return;  // warp-uniform
    const int64_t j = jt * 32 + lane;
    uint32_t mm = 0u;  // bit q: sample s0 + q missing at SNP j
    if (j < m) {
        const int8_t* row = codes + j * ldc + s0;
        if (vec && s0 + 32 <= n) {
            const uint4 a = __ldg(reinterpret_cast<const uint4*>(row));
            const uint4 c = __ldg(reinterpret_cast<const uint4*>(row + 16));
            const uint32_t x[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const uint32_t m3 = __vcmpeq4(x[e], 0x03030303u);
                mm |= ((m3 & 1u) | ((m3 >> 7) & 2u) | ((m3 >> 14) & 4u) | ((m3 >> 21) & 8u)) << (4 * e);
            }
        } else {
            for (int q = 0; q < 32; ++q)
                if (s0 + q < n && row[q] == 3) mm |= 1u << q;
        }
    }
    uint32_t out = 0u;
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const uint32_t bal = __ballot_sync(0xffffffffu, (mm >> q) & 1u);
        if (lane == q) out = bal;
    }
    if (s0 + lane < n) mask[(s0 + lane) * words + jt] = out;
}

// One SNP for a thread's 16 samples.  A word value c (0..3) becomes the double 4 + c built
// in one 64-bit integer multiply-add: the two bits, masked at bit position pos (20..30) of
// w or of w shifted by 10 or 20, times 2^(50 - pos) land at bits 50-51 -- the top two
// mantissa bits -- of the bit pattern of 4.0 (exponent 2, so they weigh 1 and 2), and the
// result is already the register pair the FMA with mu_j reads.  The offset 4 sum_j mu_j is
// removed afterwards (4 mu is exact, so a sample with only zero calls ends with exactly
// 4 x the plain sum).
__device__ __forceinline__ double sp_call_double(uint32_t masked, uint32_t mult) {
    unsigned long long d;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(masked), "r"(mult), "l"(0x4010000000000000ull));
    return __longlong_as_double((long long)d);
}

__device__ __forceinline__ void sp_word(uint32_t w, double u, double (&r)[kSpSpt]) {
    const uint32_t g[3] = {w << 20, w << 10, w};  // samples 0-4, 5-9, 10-15 at bits 20-31
#pragma unroll
    for (int q = 0; q < kSpSpt; ++q) {
        const int gi = q < 5 ? 0 : (q < 10 ? 1 : 2);
        const int pos = 2 * q + (gi == 0 ? 20 : (gi == 1 ? 10 : 0));
        r[q] = fma(u, sp_call_double(g[gi] & (3u << pos), 1u << (50 - pos)), r[q]);
    }
}

template <bool kR>
__global__ void __launch_bounds__(kSpThreads, 3) kin_sp_kernel(
    const uint32_t* __restrict__ zb, int64_t wpr, const uint32_t* __restrict__ mask,
    int64_t words, const double* __restrict__ mu, int64_t n, double* __restrict__ Q,
    int64_t ldq) {
    extern __shared__ __align__(16) unsigned char sp_smem_raw[];
    SpSmem& S = *reinterpret_cast<SpSmem*>(sp_smem_raw);
    const int64_t k = blockIdx.x;
    const int b = blockIdx.y;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // k's missing SNPs in increasing order: thread t owns mask words 2t, 2t+1
    const uint32_t* __restrict__ mk = mask + k * words;
    uint32_t m0 = 2 * tid < words ? __ldg(mk + 2 * tid) : 0u;
    uint32_t m1 = 2 * tid + 1 < words ? __ldg(mk + 2 * tid + 1) : 0u;
    const int c = __popc(m0) + __popc(m1);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) S.warp_sum[warp] = incl;
#pragma unroll
    for (int q = 0; q < kSpSpt; ++q) S.corr[q][tid] = 0.0;  // this thread's own slots
    __syncthreads();
    int pos = incl - c, cnt = 0;
#pragma unroll
    for (int w = 0; w < kSpThreads / 32; ++w) {
        pos += w < warp ? S.warp_sum[w] : 0;
        cnt += S.warp_sum[w];
    }
    while (m0) {
        S.jl[pos++] = (uint16_t)(64 * tid + __ffs(m0) - 1);
        m0 &= m0 - 1u;
    }
    while (m1) {
        S.jl[pos++] = (uint16_t)(64 * tid + 32 + __ffs(m1) - 1);
        m1 &= m1 - 1u;
    }
    __syncthreads();
    double r[kSpSpt];
#pragma unroll
    for (int q = 0; q < kSpSpt; ++q) r[q] = 0.0;
    double s = 0.0;
    const int64_t wi = (int64_t)b * kSpWords + tid;
    const bool act = wi < wpr;
    const uint32_t* __restrict__ zc = zb + (act ? wi : 0);
    uint32_t wn[4];
    double un[4];
    auto fetch = [&](int p0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int p = p0 + e;
            if (p < cnt) {
                const int64_t j = S.jl[p];
                un[e] = __ldg(mu + j);
                wn[e] = act ? __ldg(zc + j * wpr) : 0u;
            } else {
                un[e] = 0.0;
                wn[e] = 0u;
            }
        }
    };
    fetch(0);
#pragma unroll 1
    for (int p0 = 0; p0 < cnt; p0 += 4) {
        uint32_t w[4];
        double u[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            w[e] = wn[e];
            u[e] = un[e];
        }
        fetch(p0 + 4);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (kR) {
                s += u[e];
                sp_word(w[e], u[e], r);
            }
            uint32_t mm = w[e] & (w[e] >> 1) & 0x55555555u;  // bit 2q: sample q missing
            if (mm) {
                const double h = kR ? fma(0.5 * u[e], u[e], -3.0 * u[e]) : 0.5 * u[e] * u[e];
                do {
                    const int q = (__ffs(mm) - 1) >> 1;
                    S.corr[q][tid] += h;
                    mm &= mm - 1u;
                } while (mm);
            }
        }
    }
    const double s4 = 4.0 * s;
    const int64_t i0 = (int64_t)b * kSpBlock + (int64_t)tid * kSpSpt;
#pragma unroll
    for (int q = 0; q < kSpSpt; ++q) {
        const int64_t i = i0 + q;
        double v = S.corr[q][tid];
        if (kR) v += r[q] - s4;
        if (i < n && v != 0.0) Q[k * ldq + i] += v;  // Q[i, k] (column-major, column k)
    }
}

// ---------------------------------------------------------------- tensor-core correction
// The same sparse terms on INT8 tensor cores, for chunks with many missing calls.
//   R = Z diag(mu) M^T   (Z: calls, missing -> 0; M: missing masks; n x m each)
// With mu_j = (2/127) sum_{t<4} 254^-t d_t(mu_j) (four base-254 digits of mu_j * 127/2,
// error <= 4.8e-10 per mu_j), R = (2/127) sum_t 254^-t Z B_t^T, B_t = M diag(d_t), whose
// int32 products are exact.  The digit planes are interleaved along N -- row 4k + t of B
// is B_t's row k -- so one GEMM per chunk (M = n samples i, N = 4n, K = m SNPs) leaves
// every (i, k) with its four planes in one tile, and the epilogue adds
// (2/127) (((C3 w3 + C2 w2) + C1 w1) + C0) to Q[i, k].  The missing x missing term
// T/2 = M diag(mu^2/2) M^T comes from the dosage-word walk (kin_sp_kernel<false>).
constexpr double kMuScale = 2.0 / 127.0;
__device__ __constant__ double kPlaneW[4] = {1.0, 1.0 / 254.0, 1.0 / (254.0 * 254.0),
                                             1.0 / (254.0 * 254.0 * 254.0)};

__device__ __forceinline__ void mu_digits(double mu, int8_t (&d)[4]) {
    double a = mu * (127.0 / 2.0);  // [0, 127]
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const double r = rint(a);
        d[t] = (int8_t)r;
        a = (a - r) * 254.0;  // remainder within +-0.5 -> next digit within +-127
    }
}

// B (4n x ldb, K-major): B[(4k + t) * ldb + j] = d_t(mu_j) if sample k is missing at SNP j
// (bit j of k's missing-SNP mask).
__global__ void kin_rmask_kernel(const uint32_t* __restrict__ mask, int64_t words, int64_t n,
                                 int64_t m, const double* __restrict__ mu, int8_t* __restrict__ B,
                                 int64_t ldb) {
    for (int64_t k = blockIdx.y; k < n; k += gridDim.y) {
        for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ldb;
             j += (int64_t)gridDim.x * blockDim.x) {
            int8_t d[4] = {0, 0, 0, 0};
            if (j < m && ((__ldg(mask + k * words + (j >> 5)) >> (j & 31)) & 1u)) mu_digits(mu[j], d);
#pragma unroll
            for (int t = 0; t < 4; ++t) B[(4 * k + t) * ldb + j] = d[t];
        }
    }
}

struct KinREpi {
    static constexpr int kSmem = 0;
    double* Q;
    int64_t ldq;
    int n;
    __device__ __forceinline__ void run(int mb, int nb, uint32_t taddr, int q, int lane,
                                        uint8_t*) const {
        const int i = mb * kBM + 32 * q + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < 256; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(taddr + (uint32_t)c0, v);
            if (i < n) {
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    const int k = (nb * 256 + c0) / 4 + kk;
                    if (k < n) {
                        const double x =
                            (((double)(int32_t)v[4 * kk + 3] * kPlaneW[3] +
                              (double)(int32_t)v[4 * kk + 2] * kPlaneW[2]) +
                             (double)(int32_t)v[4 * kk + 1] * kPlaneW[1]) +
                            (double)(int32_t)v[4 * kk];
                        Q[(int64_t)k * ldq + i] += x * kMuScale;
                    }
                }
            }
        }
    }
};

// K = (C - a_i - a_j + s - b_i - b_j + Q_ij + Q_ji) / p, symmetric, column-major.
__global__ void kin_finalize_i8_kernel(const int32_t* __restrict__ C, int64_t ldc, int64_t n,
                                       const double* __restrict__ a, const double* __restrict__ b,
                                       double s, const double* __restrict__ RT, int64_t ldr,
                                       double inv_p, double* __restrict__ K, int64_t ldk) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= j && i < n;
             i += (int64_t)gridDim.x * blockDim.x) {
            // the int32 Gram holds the upper triangle (row i <= column j) at C[j*ldc + i]
            double v = (double)C[j * ldc + i] - a[i] - a[j] + s - b[i] - b[j];
            if (RT) v += RT[j * ldr + i] + RT[i * ldr + j];
            v *= inv_p;
            K[j * ldk + i] = v;
            K[i * ldk + j] = v;
        }
    }
}

// Leave-one-chromosome-out: every term of p K is a sum over SNPs, so the kinship without
// chromosome c is the full-genome combination minus chromosome c's, over p - p_c SNPs.
// The int32 Grams subtract exactly.
__global__ void kin_finalize_loco_kernel(const int32_t* __restrict__ Cf, const int32_t* __restrict__ Cc,
                                         int64_t ldc, int64_t n, const double* __restrict__ af,
                                         const double* __restrict__ ac, const double* __restrict__ bf,
                                         const double* __restrict__ bc, double s,
                                         const double* __restrict__ Qf,
                                         const double* __restrict__ Qc, int64_t ldq, double inv_p,
                                         double* __restrict__ K, int64_t ldk) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= j && i < n;
             i += (int64_t)gridDim.x * blockDim.x) {
            const int32_t g = Cf[j * ldc + i] - Cc[j * ldc + i];
            const double ai = af[i] - ac[i], aj = af[j] - ac[j];
            const double bi = bf[i] - bc[i], bj = bf[j] - bc[j];
            double v = (double)g - ai - aj + s - bi - bj;
            if (Qf) v += (Qf[j * ldq + i] + Qf[i * ldq + j]) - (Qc[j * ldq + i] + Qc[i * ldq + j]);
            v *= inv_p;
            K[j * ldk + i] = v;
            K[i * ldk + j] = v;
        }
    }
}

// Plain FP64 form: K = (S_full - S_c) * scale from lower triangles, written symmetric.
__global__ void kin_sub_scale_kernel(const double* __restrict__ Sf, const double* __restrict__ Sc,
                                     int64_t n, int64_t lds, double scale, double* __restrict__ K,
                                     int64_t ldk) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += (int64_t)gridDim.x * blockDim.x) {
            if (i >= j) {
                const double v = (Sf[j * lds + i] - Sc[j * lds + i]) * scale;
                K[j * ldk + i] = v;
                K[i * ldk + j] = v;
            }
        }
    }
}

}  // namespace tc
}  // namespace jb

using namespace jb;
using namespace jb::tc;

namespace {
constexpr int kGramBN = 256;
constexpr int kGramStages = 4;
using GramSmem = GemmSmem<kGramBN, kGramStages, 0>;

struct GramWs {
    int64_t status, tiles, total;
};
GramWs gram_ws(int64_t n) {
    const int64_t MB = ceil_div(n, kBM), NB = ceil_div(n, kGramBN);
    GramWs w;
    w.status = 0;
    w.tiles = 256;
    w.total = w.tiles + ((MB * NB * (int64_t)sizeof(Tile) + 255) / 256) * 256;
    return w;
}
// Scratch for jb_gram_i8_noalloc: one file-scope device array, 1 MiB, present on every
// GPU that loads this library until the process exits.  Host code cannot use the symbol
// itself as a device address; its address on each device is looked up once with
// cudaGetSymbolAddress while that device is current.
constexpr int64_t kNoAllocScratchBytes = 1 << 20;
static __device__ __align__(256) unsigned char g_gram_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

int32_t noalloc_scratch(void** out) {
    int dev = 0;
    JB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("jb_gram_i8_noalloc: device ordinal %d out of range", dev);
        return JB_E_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_gram_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(gram scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return JB_OK;
}
}  // namespace

extern "C" {

int64_t jb_gram_i8_workspace_size(int64_t n) {
    if (n <= 0) return -1;
    return gram_ws(n).total;
}

int32_t jb_gram_i8(const int8_t* Z, int64_t n, int64_t p, int64_t ldz, int32_t* C, int64_t ldc,
                   void* workspace, int64_t workspace_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && p > 0 && ldz >= p && ldc >= n, "jb_gram_i8: bad shape");
    JB_CHECK_ARG(n < (1ll << 31) && p < (1ll << 31), "jb_gram_i8: size too large");
    JB_CHECK_ARG(4ll * p < (1ll << 31), "jb_gram_i8: p too large for exact int32 accumulation");
    const GramWs L = gram_ws(n);
    JB_CHECK_ARG(workspace && workspace_bytes >= L.total, "jb_gram_i8: workspace too small");
    cudaStream_t st = as_stream(stream);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    int* status = reinterpret_cast<int*>(ws + L.status);
    Tile* tiles = reinterpret_cast<Tile*>(ws + L.tiles);
    const int MB = (int)ceil_div(n, kBM), NB = (int)ceil_div(n, kGramBN);
    const int n_tiles = gram_tiles(MB, NB, nullptr);
    CUtensorMap ta, tb;
    int32_t rc = make_map_i8(&ta, Z, n, p, ldz, kBM);
    if (rc) return rc;
    rc = make_map_i8(&tb, Z, n, p, ldz, kGramBN);
    if (rc) return rc;
    JB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    gram_tiles_kernel<<<1, 32, 0, st>>>(MB, NB, tiles);
    JB_LAUNCH_CHECK("gram_tiles_kernel");
    auto kern = i8_gemm_kernel<kGramBN, kGramStages, GramEpi>;
    JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 GramSmem::TOTAL));
    GramEpi epi{C, ldc, (int)n};
    const int grid = n_tiles < num_sms() ? n_tiles : num_sms();
    const int num_kb = (int)ceil_div(p, kBK);
    kern<<<grid, kThreads, GramSmem::TOTAL, st>>>(ta, tb, tiles, n_tiles, num_kb, epi, status);
    JB_LAUNCH_CHECK("i8_gemm_kernel<gram>");
    return JB_OK;
}

int32_t jb_kinship_i8_finalize_loco(const int32_t* C_full, const int32_t* C_chr, int64_t ldc,
                                    int64_t n, const double* a_full, const double* a_chr,
                                    const double* b_full, const double* b_chr, double sum_mu2_loco,
                                    const double* Q_full, const double* Q_chr, int64_t ldq,
                                    int64_t p_loco, double* K, int64_t ldk, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && ldc >= n && ldk >= n && p_loco > 0, "jb_kinship_i8_finalize_loco: bad shape");
    JB_CHECK_ARG((Q_full == nullptr) == (Q_chr == nullptr) && (!Q_full || ldq >= n),
                 "jb_kinship_i8_finalize_loco: Q_full and Q_chr go together");
    dim3 grid((unsigned)(ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64), grid_y(n), 1);
    kin_finalize_loco_kernel<<<grid, 256, 0, as_stream(stream)>>>(
        C_full, C_chr, ldc, n, a_full, a_chr, b_full, b_chr, sum_mu2_loco, Q_full, Q_chr, ldq,
        1.0 / (double)p_loco, K, ldk);
    JB_LAUNCH_CHECK("kin_finalize_loco_kernel");
    return JB_OK;
}

int32_t jb_kinship_loco_f64(const double* S_full, const double* S_chr, int64_t n, int64_t lds,
                            int64_t p_loco, double* K, int64_t ldk, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && lds >= n && ldk >= n && p_loco > 0, "jb_kinship_loco_f64: bad shape");
    dim3 grid((unsigned)(ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64), grid_y(n), 1);
    kin_sub_scale_kernel<<<grid, 256, 0, as_stream(stream)>>>(S_full, S_chr, n, lds,
                                                             1.0 / (double)p_loco, K, ldk);
    JB_LAUNCH_CHECK("kin_sub_scale_kernel");
    return JB_OK;
}

int32_t jb_gram_i8_noalloc(const int8_t* Zs, int64_t n, int64_t p, int64_t ldz, int32_t* C,
                           int64_t ldc, uintptr_t stream) {
    JB_CHECK_ARG(n > 0, "jb_gram_i8_noalloc: bad shape");
    const int64_t need = gram_ws(n).total;
    JB_CHECK_ARG(need <= kNoAllocScratchBytes,
                 "jb_gram_i8_noalloc: n = %lld needs %lld bytes of scratch, more than the "
                 "library's static %lld bytes (n <= 65408); use jb_gram_i8 with a workspace",
                 (long long)n, (long long)need, (long long)kNoAllocScratchBytes);
    void* scratch = nullptr;
    const int32_t rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return jb_gram_i8(Zs, n, p, ldz, C, ldc, scratch, kNoAllocScratchBytes, stream);
}

int32_t jb_gram_i8_noalloc_status(int32_t* out, uintptr_t stream) {
    JB_CHECK_ARG(out, "jb_gram_i8_noalloc_status: null pointer");
    void* scratch = nullptr;
    const int32_t rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return jb_gram_status(scratch, out, stream);
}

int32_t jb_test_pipeline_timeout(int32_t skip_loads, int64_t wait_limit_ns) {
    JB_CHECK_ARG(wait_limit_ns > 0, "jb_test_pipeline_timeout: wait limit must be positive");
    JB_CUDA(cudaDeviceSynchronize());  // no kernel of the old mode still running
    const unsigned long long lim = (unsigned long long)wait_limit_ns;
    JB_CUDA(pipeline_test_mode(skip_loads ? 1 : 0, lim));
    JB_CUDA(rotate_pipeline_test_mode(skip_loads ? 1 : 0, lim));
    return JB_OK;
}

int32_t jb_gram_status(const void* workspace, int32_t* out, uintptr_t stream) {
    JB_CHECK_ARG(workspace && out, "jb_gram_status: null pointer");
    JB_CUDA(cudaMemcpyAsync(out, workspace, sizeof(int32_t), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    JB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return JB_OK;
}

int32_t jb_codes_to_sample_major(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                                 int8_t* Zs, int64_t ldz, int64_t col0, int8_t* Cs, int64_t ldcs,
                                 uintptr_t stream) {
    JB_CHECK_ARG(n >= 0 && m >= 0 && ld_codes >= n && col0 >= 0,
                 "jb_codes_to_sample_major: bad shape");
    JB_CHECK_ARG(!Zs || ldz >= col0 + m, "jb_codes_to_sample_major: ldz too small");
    JB_CHECK_ARG(!Cs || ldcs >= m, "jb_codes_to_sample_major: ldcs too small");
    if (n == 0 || m == 0) return JB_OK;
    JB_CHECK_ARG(ceil_div(n, 32) < 65536, "jb_codes_to_sample_major: n too large");
    const bool vec = Zs && !Cs && (reinterpret_cast<uintptr_t>(codes) & 3) == 0 && ld_codes % 4 == 0 &&
                     (reinterpret_cast<uintptr_t>(Zs) & 3) == 0 && ldz % 4 == 0 && col0 % 4 == 0;
    if (vec) {
        JB_CHECK_ARG(ceil_div(n, 64) < 65536, "jb_codes_to_sample_major: n too large");
        dim3 grid((unsigned)ceil_div(m, 64), (unsigned)ceil_div(n, 64), 1);
        codes_to_sample_major_vec_kernel<<<grid, 256, 0, as_stream(stream)>>>(codes, ld_codes, n, m, Zs,
                                                                              ldz, col0);
        JB_LAUNCH_CHECK("codes_to_sample_major_vec_kernel");
        return JB_OK;
    }
    dim3 grid((unsigned)ceil_div(m, 32), (unsigned)ceil_div(n, 32), 1);
    codes_to_sample_major_kernel<<<grid, dim3(32, 8), 0, as_stream(stream)>>>(codes, ld_codes, n,
                                                                              m, Zs, ldz, col0, Cs, ldcs);
    JB_LAUNCH_CHECK("codes_to_sample_major_kernel");
    return JB_OK;
}

// Workspace of the correction entry points (tc: with the tensor-core R operand).
struct KinCorrWs {
    int64_t status, pa, mask, zb, tiles, B, ldb, total, wpr, words;
    int nb;
};
static KinCorrWs kin_corr_ws(int64_t n, int64_t m, bool tc) {
    KinCorrWs w;
    const int64_t mm = m > 0 ? m : 1;
    const int64_t nblk = ceil_div(mm, 256);
    auto a256 = [](int64_t x) { return (x + 255) / 256 * 256; };
    w.words = ceil_div(mm, 32);
    w.wpr = ceil_div(n, 16);
    w.nb = (int)ceil_div(n, kSpBlock);
    int64_t off = 0;
    w.status = off;
    off += 256;
    w.pa = off;
    off += a256(2 * nblk * n * 8);
    w.mask = off;
    off += a256(n * w.words * 4);
    w.zb = off;
    off += a256(mm * w.wpr * 4);
    w.ldb = (mm + 127) / 128 * 128;
    w.tiles = off;
    off += tc ? a256(ceil_div(n, kBM) * ceil_div(4 * n, 256) * (int64_t)sizeof(Tile)) : 0;
    w.B = off;
    off += tc ? a256(4 * n * w.ldb) : 0;
    w.total = off;
    return w;
}

// a, b: ordered two-stage sums over the chunk's SNPs.
static int32_t kin_vectors(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                           const double* mu, double* a, double* b, double* pa, cudaStream_t st) {
    const int64_t nblk = ceil_div(m, 256);
    double* pb = pa + nblk * n;
    const int vec = ((reinterpret_cast<uintptr_t>(codes) & 3) == 0 && ld_codes % 4 == 0) ? 1 : 0;
    kin_vectors_partial_kernel<<<dim3((unsigned)ceil_div(n, 1024), (unsigned)nblk), 256, 0, st>>>(
        codes, ld_codes, n, m, vec, mu, pa, pb);
    JB_LAUNCH_CHECK("kin_vectors_partial_kernel");
    kin_vectors_reduce_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(n, nblk, pa, pb, a, b);
    JB_LAUNCH_CHECK("kin_vectors_reduce_kernel");
    return JB_OK;
}

// Per-sample missing-SNP bitmasks of the chunk into the workspace.
static int32_t kin_masks(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                         const KinCorrWs& L, uint8_t* ws, cudaStream_t st) {
    uint32_t* mask = reinterpret_cast<uint32_t*>(ws + L.mask);
    const int vec = ((reinterpret_cast<uintptr_t>(codes) & 15) == 0 && ld_codes % 16 == 0) ? 1 : 0;
    JB_CHECK_ARG(ceil_div(n, 256) < 65536, "kinship corrections: n too large");
    kin_mask_kernel<<<dim3((unsigned)L.words, (unsigned)ceil_div(n, 256)), 256, 0, st>>>(
        codes, ld_codes, n, m, vec, mask, L.words);
    JB_LAUNCH_CHECK("kin_mask_kernel");
    return JB_OK;
}

// Q += T/2 (with_r: + R) for one chunk from the masks (kin_masks) and the dosage words.
static int32_t kin_missing_terms(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                                 const double* mu, double* RT, int64_t ldr, const KinCorrWs& L,
                                 uint8_t* ws, bool with_r, cudaStream_t st) {
    const uint32_t* mask = reinterpret_cast<const uint32_t*>(ws + L.mask);
    uint32_t* zb = reinterpret_cast<uint32_t*>(ws + L.zb);
    const int vec = ((reinterpret_cast<uintptr_t>(codes) & 15) == 0 && ld_codes % 16 == 0) ? 1 : 0;
    kin_sp_words_kernel<<<(unsigned)ceil_div(m, 8), 256, 0, st>>>(codes, ld_codes, n, m, L.wpr, vec, zb);
    JB_LAUNCH_CHECK("kin_sp_words_kernel");
    auto kern = with_r ? kin_sp_kernel<true> : kin_sp_kernel<false>;
    JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SpSmem)));
    kern<<<dim3((unsigned)n, (unsigned)L.nb), kSpThreads, sizeof(SpSmem), st>>>(
        zb, L.wpr, mask, L.words, mu, n, RT, ldr);
    JB_LAUNCH_CHECK("kin_sp_kernel");
    return JB_OK;
}

int64_t jb_kinship_i8_corrections_workspace_size(int64_t n, int64_t m) {
    if (n <= 0 || m < 0) return -1;
    return kin_corr_ws(n, m, false).total;
}

int32_t jb_kinship_i8_corrections(const int8_t* codes, int64_t ld_codes, int32_t has_missing,
                                  int64_t n, int64_t m, const double* mu, double* a, double* b,
                                  double* RT, int64_t ldr, void* workspace,
                                  int64_t workspace_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && m >= 0 && ld_codes >= n, "jb_kinship_i8_corrections: bad shape");
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(m <= kSpMaxChunk, "jb_kinship_i8_corrections: at most %d SNPs per call", kSpMaxChunk);
    JB_CHECK_ARG(codes && mu && a && b, "jb_kinship_i8_corrections: null pointer");
    JB_CHECK_ARG(n * ceil_div(n, kSpBlock) < (1ll << 31) && n < (1ll << 31),
                 "jb_kinship_i8_corrections: n too large");
    const KinCorrWs L = kin_corr_ws(n, m, false);
    JB_CHECK_ARG(workspace && workspace_bytes >= L.total,
                 "jb_kinship_i8_corrections: workspace too small");
    cudaStream_t st = as_stream(stream);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    JB_CUDA(cudaMemsetAsync(ws + L.status, 0, sizeof(int), st));
    int32_t rc = kin_vectors(codes, ld_codes, n, m, mu, a, b, reinterpret_cast<double*>(ws + L.pa), st);
    if (rc || !has_missing) return rc;
    JB_CHECK_ARG(RT && ldr >= n, "jb_kinship_i8_corrections: Q buffer needed");
    rc = kin_masks(codes, ld_codes, n, m, L, ws, st);
    if (rc) return rc;
    return kin_missing_terms(codes, ld_codes, n, m, mu, RT, ldr, L, ws, true, st);
}

int64_t jb_kinship_i8_tc_workspace_size(int64_t n, int64_t m) {
    if (n <= 0 || m < 0) return -1;
    return kin_corr_ws(n, m, true).total;
}

int32_t jb_kinship_i8_corrections_tc(const int8_t* codes, int64_t ld_codes, const int8_t* Zs,
                                     int64_t ldz, int64_t col0, int64_t n, int64_t m,
                                     const double* mu, double* a, double* b, double* RT,
                                     int64_t ldr, void* workspace, int64_t workspace_bytes,
                                     uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && m >= 0 && ld_codes >= n && ldr >= n,
                 "jb_kinship_i8_corrections_tc: bad shape");
    if (m == 0) return JB_OK;
    JB_CHECK_ARG(codes && Zs && mu && a && b && RT, "jb_kinship_i8_corrections_tc: null pointer");
    JB_CHECK_ARG(m <= kSpMaxChunk && 4 * n < (1ll << 31), "jb_kinship_i8_corrections_tc: chunk too large");
    JB_CHECK_ARG(col0 % 16 == 0 && ldz % 16 == 0 && ldz >= col0 + m,
                 "jb_kinship_i8_corrections_tc: Zs column block must start on 16 bytes");
    const KinCorrWs L = kin_corr_ws(n, m, true);
    JB_CHECK_ARG(workspace && workspace_bytes >= L.total, "jb_kinship_i8_corrections_tc: workspace too small");
    cudaStream_t st = as_stream(stream);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    int* status = reinterpret_cast<int*>(ws + L.status);
    JB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    int32_t rc = kin_vectors(codes, ld_codes, n, m, mu, a, b, reinterpret_cast<double*>(ws + L.pa), st);
    if (rc) return rc;
    // R on the tensor cores
    rc = kin_masks(codes, ld_codes, n, m, L, ws, st);
    if (rc) return rc;
    int8_t* B = reinterpret_cast<int8_t*>(ws + L.B);
    kin_rmask_kernel<<<dim3((unsigned)ceil_div(L.ldb, 256), grid_y(n)), 256, 0, st>>>(
        reinterpret_cast<const uint32_t*>(ws + L.mask), L.words, n, m, mu, B, L.ldb);
    JB_LAUNCH_CHECK("kin_rmask_kernel");
    const int MB = (int)ceil_div(n, kBM), NB = (int)ceil_div(4 * n, 256);
    Tile* tiles = reinterpret_cast<Tile*>(ws + L.tiles);
    rc = launch_group_tiles(MB, NB, 8, 16, tiles, st);
    if (rc) return rc;
    CUtensorMap ta, tb;
    rc = make_map_i8(&ta, Zs + col0, n, m, ldz, kBM);
    if (rc) return rc;
    rc = make_map_i8(&tb, B, 4 * n, m, L.ldb, 256);
    if (rc) return rc;
    auto kern = i8_gemm_kernel<kGramBN, kGramStages, KinREpi>;
    JB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, GramSmem::TOTAL));
    const int n_tiles = MB * NB;
    KinREpi epi{RT, ldr, (int)n};
    kern<<<n_tiles < num_sms() ? n_tiles : num_sms(), kThreads, GramSmem::TOTAL, st>>>(
        ta, tb, tiles, n_tiles, (int)ceil_div(m, kBK), epi, status);
    JB_LAUNCH_CHECK("i8_gemm_kernel<kinship R>");
    // T/2 from the per-SNP missing lists
    return kin_missing_terms(codes, ld_codes, n, m, mu, RT, ldr, L, ws, false, st);
}

int32_t jb_kinship_i8_finalize(const int32_t* C, int64_t ldc, int64_t n, const double* a,
                               const double* b, double sum_mu2, const double* RT, int64_t ldr,
                               int64_t p_kept, double* K, int64_t ldk, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && ldc >= n && ldk >= n && p_kept > 0, "jb_kinship_i8_finalize: bad shape");
    dim3 grid((unsigned)(ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64), grid_y(n), 1);
    kin_finalize_i8_kernel<<<grid, 256, 0, as_stream(stream)>>>(C, ldc, n, a, b, sum_mu2, RT, ldr,
                                                               1.0 / (double)p_kept, K, ldk);
    JB_LAUNCH_CHECK("kin_finalize_i8_kernel");
    return JB_OK;
}

}  // extern "C"
