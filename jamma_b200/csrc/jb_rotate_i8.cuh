// Internal interface of the INT8 rotation core (jb_rotate_i8.cu), shared with the
// mixed-form series sums in jb_lmm.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace jb {
namespace tc {

struct Tile;

// Digit planes of n_out columns of length n_k: int8 A (rows x lda, digits along M in
// blocks of 32 columns x 4 digits) followed by the per-column max |v|.
struct OzakiLayout {
    int64_t lda, rows, a_off, s_off, total;
};
OzakiLayout ozaki_layout(int64_t n_out, int64_t n_k);

// Per-chunk scratch of jb_rotate_i8: status word, tile list, packed [calls | masks] B.
struct RotChunkLayout {
    int64_t status, tiles, b_off, ldb, total;
};
RotChunkLayout rot_chunk_layout(int64_t n, int64_t m);

// Full MB x NB tile grid in groups of GM x GN tiles (closed-form order, one thread per tile).
int32_t launch_group_tiles(int MB, int NB, int GM, int GN, Tile* out, cudaStream_t st);

// Split the n_out columns of V (column-major, length n_k, stride ldv) into ws.
int32_t ozaki_split(const double* V, int64_t n_k, int64_t n_out, int64_t ldv, uint8_t* ws,
                    cudaStream_t st);

// X[j * ldx + i] = sum_k V[k, i] g[k, j] for i < n_out, j < m, from the digit planes in
// ozaki_ws and a B operand of int8 calls (b_rows x n_k, stride ldb): the paired layout
// of rot_pack_pairs_kernel (calls and missing masks, g = z + mean_j * mask) or plain calls.
int32_t rotate_i8_gemm(const uint8_t* ozaki_ws, int64_t n_out, int64_t n_k, const int8_t* B,
                       int64_t b_rows, int64_t ldb, bool paired, int64_t m, const double* mean,
                       double* X, int64_t ldx, Tile* tiles, int* status, cudaStream_t st);

// Test hooks of the rotation kernels' bounded waits (this translation unit's copy of the
// GEMM core's hooks; see jb_test_pipeline_timeout).
cudaError_t rotate_pipeline_test_mode(int skip_loads, unsigned long long wait_limit_ns);

}  // namespace tc
}  // namespace jb
