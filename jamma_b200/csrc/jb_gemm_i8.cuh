// Persistent warp-specialised INT8 tensor-core GEMM core for sm_100a.
//
//   D (tile BM x BN, int32 in TMEM) = A_tile (BM x K) * B_tile (BN x K)^T
//
// A and B are K-major int8 matrices described by TMA tensor maps (128-byte K boxes,
// 128B swizzle).  One CTA per SM walks a tile list; its 6 warps split the work:
//   warp 0      TMA producer: fills a STAGES-deep ring of (A, B) K-slices;
//   warp 1      allocates TMEM (2 accumulators x BN columns) and, from one thread,
//               issues tcgen05.mma (M=128, N=BN, K=32) into the current accumulator,
//               committing each consumed stage back to the producer and each finished
//               tile to the epilogue;
//   warps 2-5   epilogue: wait for a finished accumulator, read it with tcgen05.ld
//               (warp w owns TMEM lanes 32*(w%4)..+31 = tile rows), hand the values to
//               the Epi functor, then release the accumulator.
// Integer accumulation is exact, so results do not depend on K order or tiling.
#pragma once

#include "jb_tc.cuh"

namespace jb {
namespace tc {

constexpr int kBM = 128;
constexpr int kBK = 128;  // bytes of K per stage (one 128B swizzle row)
constexpr int kThreads = 192;

// Test hooks of the bounded pipeline waits, one copy per translation unit that launches
// these kernels: the deadline of every wait and a switch that makes the producer issue no
// tile load (so the MMA thread's first wait runs out, with no copy or MMA ever in flight).
// Each kernel reads them once at start.  Set only through pipeline_test_mode (the
// jb_test_pipeline_timeout entry point); the defaults are a 2 s deadline and loads on.
static __device__ unsigned long long g_pipe_wait_limit_ns = kWaitLimitNs;
static __device__ int g_pipe_skip_loads = 0;

static inline cudaError_t pipeline_test_mode(int skip_loads, unsigned long long wait_limit_ns) {
    cudaError_t e = cudaMemcpyToSymbol(g_pipe_skip_loads, &skip_loads, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(g_pipe_wait_limit_ns, &wait_limit_ns, sizeof(wait_limit_ns));
}

template <int BN, int STAGES, int EPI_SMEM>
struct GemmSmem {
    static constexpr int A_BYTES = kBM * kBK;
    static constexpr int B_BYTES = BN * kBK;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
    static constexpr int EPI_OFF = BAR_OFF + 256;
    static constexpr int TOTAL = EPI_OFF + EPI_SMEM + 1024;  // + alignment slack
};

struct Tile {
    int32_t mb, nb;
};

template <int BN, int STAGES, class Epi>
__global__ void __launch_bounds__(kThreads, 1)
    i8_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const Tile* __restrict__ tiles, int n_tiles, int num_kb, Epi epi, int* err) {
    using S = GemmSmem<BN, STAGES, Epi::kSmem>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFF);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    uint8_t* epi_smem = smem + S::EPI_OFF;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const unsigned long long wait_ns = g_pipe_wait_limit_ns;
    const bool skip_loads = g_pipe_skip_loads != 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 128);
        }
        *abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) tmem_alloc(tmem_slot, 2 * BN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // ---------------- TMA producer
            int stage = 0;
            uint32_t phase = 0;
            for (int t = blockIdx.x; t < n_tiles && !*abort; t += gridDim.x) {
                const Tile tl = tiles[t];
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, abort, err, 1, wait_ns)) break;
                    uint8_t* sa = smem + stage * S::STAGE_BYTES;
                    if (!skip_loads) {
                        mbar_expect_tx(&full[stage], S::STAGE_BYTES);
                        tma_load_2d(sa, &tmA, &full[stage], kb * kBK, tl.mb * kBM);
                        tma_load_2d(sa + S::A_BYTES, &tmB, &full[stage], kb * kBK, tl.nb * BN);
                    }
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // ---------------- MMA issuer
            constexpr uint32_t idesc = idesc_i8(kBM, BN);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            for (int t = blockIdx.x; t < n_tiles && !*abort; t += gridDim.x) {
                if (!mbar_wait(&tempty[acc], acc_phase ^ 1, abort, err, 2, wait_ns)) break;
                tc_fence_after();
                const uint32_t d = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&full[stage], phase, abort, err, 3, wait_ns)) break;
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + stage * S::STAGE_BYTES);
                    const uint32_t sb = sa + S::A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < kBK / 32; ++kk) {
                        umma_i8(d, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), idesc,
                                (kb | kk) != 0);
                    }
                    umma_commit(&empty[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                umma_commit(&tfull[acc]);
                acc ^= 1;
                if (acc == 0) acc_phase ^= 1;
            }
        }
    } else {  // ---------------- epilogue warps 2..5
        // One thread waits for the accumulator and broadcasts the outcome, so the four
        // warps always take the same branch (their named barriers stay matched).
        volatile int* go = reinterpret_cast<volatile int*>(tmem_slot + 2);
        const int q = warp & 3;  // TMEM lane quarter this warp may access
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
            if (threadIdx.x == 64) *go = mbar_wait(&tfull[acc], acc_phase, abort, err, 4, wait_ns) ? 1 : 0;
            asm volatile("bar.sync 1, 128;" ::: "memory");
            const int proceed = *go;
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (!proceed) break;
            tc_fence_after();
            const Tile tl = tiles[t];
            epi.run(tl.mb, tl.nb, tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * BN), q,
                    lane, epi_smem);
            tc_fence_before();
            mbar_arrive(&tempty[acc]);
            acc ^= 1;
            if (acc == 0) acc_phase ^= 1;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem_base, 2 * BN);
}

// ---------------------------------------------------------------- CTA-pair variant
// Same roles, on a cluster of two CTAs (cta_group::2): tile = 256 A rows x 256 B rows.
// CTA r of the pair loads A rows [256 mb + 128 r, +128) and B rows [256 nb + 128 r, +128)
// into its own ring (both TMA completions counted on the even CTA's full barrier); the
// even CTA's MMA thread issues M = 256, N = 256 MMAs whose accumulator rows 128 r.. land
// in CTA r's TMEM; commits arrive on both CTAs' barriers; each CTA's epilogue handles its
// 128 rows (A block 2 mb + r) and releases the accumulator on the even CTA's barrier.
// Per SM each K step streams 128 A + 128 B rows for 128 x 256 MACs (2/3 of the
// single-CTA operand traffic).
template <int STAGES, int EPI_SMEM>
struct PairSmem {
    static constexpr int A_BYTES = kBM * kBK;
    static constexpr int B_BYTES = 128 * kBK;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
    static constexpr int EPI_OFF = BAR_OFF + 256;
    static constexpr int TOTAL = EPI_OFF + EPI_SMEM + 1024;
};

template <int STAGES, class Epi>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    i8_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, const Tile* __restrict__ tiles,
                        int n_tiles, int num_kb, Epi epi, int* err) {
    constexpr int BN = 256;  // accumulator columns
    using S = PairSmem<STAGES, Epi::kSmem>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S::BAR_OFF);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    uint8_t* epi_smem = smem + S::EPI_OFF;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int pair = blockIdx.x >> 1, n_pairs = gridDim.x >> 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);   // the even CTA's arrive.expect_tx (both CTAs' bytes)
            mbar_init(&empty[s], 1);  // the pair's MMA commit
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 8);  // lane 0 of the 4 epilogue warps of both CTAs
        }
        *abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) tmem_alloc_pair(tmem_slot, 2 * BN);
    tc_fence_before();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // ---------------- TMA producer (both CTAs)
            int stage = 0;
            uint32_t phase = 0;
            for (int t = pair; t < n_tiles && !*abort; t += n_pairs) {
                const Tile tl = tiles[t];
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, abort, err, 1)) break;
                    uint8_t* sa = smem + stage * S::STAGE_BYTES;
                    if (rank == 0) mbar_expect_tx(&full[stage], 2 * S::STAGE_BYTES);
                    const uint32_t fb = mapa_u32(&full[stage], 0);
                    tma_load_2d_pair(sa, &tmA, fb, kb * kBK, (2 * tl.mb + (int)rank) * kBM);
                    tma_load_2d_pair(sa + S::A_BYTES, &tmB, fb, kb * kBK, tl.nb * BN + (int)rank * 128);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {  // ---------------- MMA issuer (even CTA)
            constexpr uint32_t idesc = idesc_i8(2 * kBM, BN);
            int stage = 0;
            uint32_t phase = 0;
            int acc = 0;
            uint32_t acc_phase = 0;
            for (int t = pair; t < n_tiles && !*abort; t += n_pairs) {
                if (!mbar_wait(&tempty[acc], acc_phase ^ 1, abort, err, 2)) break;
                tc_fence_after();
                const uint32_t d = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&full[stage], phase, abort, err, 3)) break;
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + stage * S::STAGE_BYTES);
                    const uint32_t sb = sa + S::A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < kBK / 32; ++kk) {
                        umma_i8_pair(d, sdesc_k128(sa + kk * 32), sdesc_k128(sb + kk * 32), idesc,
                                     (kb | kk) != 0);
                    }
                    umma_commit_pair(&empty[stage]);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                umma_commit_pair(&tfull[acc]);
                acc ^= 1;
                if (acc == 0) acc_phase ^= 1;
            }
        }
    } else {  // ---------------- epilogue warps 2..5 (both CTAs)
        volatile int* go = reinterpret_cast<volatile int*>(tmem_slot + 2);
        const int q = warp & 3;
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int t = pair; t < n_tiles; t += n_pairs) {
            if (threadIdx.x == 64) *go = mbar_wait(&tfull[acc], acc_phase, abort, err, 4) ? 1 : 0;
            asm volatile("bar.sync 1, 128;" ::: "memory");
            const int proceed = *go;
            asm volatile("bar.sync 1, 128;" ::: "memory");
            if (!proceed) break;
            tc_fence_after();
            const Tile tl = tiles[t];
            epi.run(2 * tl.mb + (int)rank, tl.nb,
                    tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(acc * BN), q, lane,
                    epi_smem);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(&tempty[acc], 0);
            acc ^= 1;
            if (acc == 0) acc_phase ^= 1;
        }
    }
    __syncwarp();
    tc_fence_before();
    cluster_sync();  // no CTA leaves while its peer may still signal its barriers
    tc_fence_after();
    if (warp == 1) tmem_dealloc_pair(tmem_base, 2 * BN);
}

}  // namespace tc
}  // namespace jb
