/*
 * jamma_b200.h -- C ABI of libjamma_b200.so, the sm_100a implementation of jamma's
 * GEMMA-style LMM association hot path.
 *
 * Conventions
 *   - Every entry point returns int32 status: 0 = OK, < 0 = error (JB_E_*).  The
 *     text of the last error on the calling thread is available from jb_last_error.
 *   - All array arguments are DEVICE pointers owned by the caller (torch tensors in
 *     the Python host code), with explicit sizes and leading dimensions.  Matrices are
 *     column-major ("ld" = distance between columns, in elements) unless stated.
 *   - `stream` is a cudaStream_t passed as uintptr_t (0 = legacy default stream).
 *     Work is enqueued asynchronously on it; nothing synchronises unless stated.
 *   - Library-internal scratch comes from a caller-provided workspace where a function
 *     needs one; the matching *_workspace_size query gives the byte count.
 *
 * Each function cites the jamma call site it replaces (paths inside the jamma
 * project, version 2.0.1).
 */
#ifndef JAMMA_B200_H
#define JAMMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JB_OK 0
#define JB_E_INVALID (-1)   /* bad argument / shape */
#define JB_E_CUDA (-2)      /* CUDA runtime error */
#define JB_E_LIBRARY (-3)   /* cuBLAS / cuSOLVER error */
#define JB_E_UNSUPPORTED (-4)
#define JB_E_NUMERIC (-5)   /* eigensolver did not converge */

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int32_t jb_version(void);

/* Copy the last error message of this thread into buf (always NUL-terminated). */
int32_t jb_last_error(char* buf, size_t len);

/* Compute capability of the current device as major*10+minor (100 for B200). */
int32_t jb_device_arch(void);

/* ------------------------------------------------------------------ genotypes */

/*
 * Decode PLINK .bed records (SNP-major, ceil(n_file/4) bytes per SNP, count-A1 codes
 * 00->2, 01->missing, 10->1, 11->0) for m SNPs into int8 codes, keeping only the
 * analysed samples sample_idx[0..n) (NULL = identity, n == n_file).
 *   codes  : m x ld_codes int8, SNP-major (one row of ld_codes bytes per SNP; sample
 *            s at [j*ld_codes + s]); value 0/1/2, or 3 for a missing call.  Entries
 *            s in [n, ld_codes) are written as 0 (zero padding for tensor-core tiles).
 *   counts : m x 4 int32 per SNP: {n_obs, sum of counts, n_het(=#1), n_hom2(=#2)}.
 * Replaces bed-reader's windowed read (src/jamma/io/plink.py:299) and the pass-1
 * statistics loop (src/jamma/lmm/runner_streaming.py:246-256).
 */
int32_t jb_decode_bed(const uint8_t* packed, int64_t bytes_per_snp, int64_t m,
                      const int32_t* sample_idx, int64_t n, int8_t* codes,
                      int64_t ld_codes, int32_t* counts, uintptr_t stream);

/* Re-pack decoded codes (m x ld_codes) into count-A1 .bed records (m x bytes_per_snp). */
int32_t jb_pack_codes(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                      uint8_t* packed, int64_t bytes_per_snp, uintptr_t stream);

/*
 * Mean-impute (no centering) decoded codes into FP64 genotype columns:
 * G[i + j*ldg] = code (0/1/2) or mean[j] where the code is 3 (missing).
 * Replaces the imputation at src/jamma/lmm/runner_streaming.py:427-434.
 */
int32_t jb_impute_f64(const int8_t* codes, int64_t ld_codes, int64_t n, int64_t m,
                      const double* mean, double* G, int64_t ldg, uintptr_t stream);

/* ------------------------------------------------------------------ kinship */

/*
 * Plain FP64 centered-kinship accumulation: K (n x n, ldk) += Xc * Xc^T over m SNP
 * columns, where Xc = code - mean[j] for observed codes and 0 for missing ones
 * (impute_and_center, src/jamma/kinship/missing.py:22-61, then the batch Gram of
 * _accumulate_kinship, src/jamma/kinship/compute.py:46-57).  Only the lower triangle
 * of K is updated (cuBLAS DSYRK); workspace holds the FP64 centered batch.
 */
int64_t jb_kinship_f64_workspace_size(int64_t n, int64_t m);
int32_t jb_kinship_accumulate_f64(const int8_t* codes, int64_t ld_codes, int64_t n,
                                  int64_t m, const double* mean, double* K, int64_t ldk,
                                  void* workspace, int64_t workspace_bytes,
                                  uintptr_t stream);

/*
 * Standardized kinship (-gk 2) accumulation: as jb_kinship_accumulate_f64 with every
 * centred column divided by sd[j] (0 where sd[j] == 0) -- impute_center_and_standardize
 * (src/jamma/kinship/missing.py:64-119) feeding compute_standardized_kinship
 * (src/jamma/kinship/compute.py:229-360).  sd[j] = sqrt(mean over all n samples of the
 * mean-imputed x^2 - mean^2), computed by the caller from the pass-1 counts.
 */
int32_t jb_kinship_accumulate_std_f64(const int8_t* codes, int64_t ld_codes, int64_t n,
                                      int64_t m, const double* mean, const double* sd, double* K,
                                      int64_t ldk, void* workspace, int64_t workspace_bytes,
                                      uintptr_t stream);

/* Symmetrise from the lower triangle and scale: K = K * scale (ldk). */
int32_t jb_kinship_finalize(double* K, int64_t n, int64_t ldk, double scale,
                            uintptr_t stream);

/*
 * Mixed-precision centered kinship.  Replaces the FP64 batch Gram of
 * _accumulate_kinship (src/jamma/kinship/compute.py:46-57) with an exact INT8 tensor-core
 * Gram plus FP64 corrections that reproduce impute_and_center
 * (src/jamma/kinship/missing.py:22-61):
 *   p K = Z Z^T - a 1^T - 1 a^T + (sum mu^2) 1 1^T - b 1^T - 1 b^T + R + R^T + T
 * with Z the int8 calls (0 where missing), mu the per-SNP float64 means, M the missing
 * mask, a = Z mu, b = M mu^2, R = Z diag(mu) M^T, T = M diag(mu^2) M^T.
 *
 * jb_codes_to_sample_major: transpose SNP-major codes (m x ld_codes) into the
 *   sample-major Gram operand Zs[i*ldz + col0 + j] (missing -> 0; ldz multiple of 16)
 *   and, if Cs != NULL, the raw sample-major codes Cs[i*ldcs + j] of this chunk.
 * jb_gram_i8: C[j*ldc + i] = sum_k Zs[i,k] Zs[j,k] for i <= j (int32, exact; tcgen05
 *   kind::i8).  Zs: n x p, row stride ldz bytes.  workspace: jb_gram_i8_workspace_size;
 *   its first int32 is a status word (non-zero if a pipeline wait timed out), read with
 *   jb_gram_status (synchronises the stream).
 * jb_kinship_i8_corrections: accumulate a, b (n doubles each) and, when has_missing
 *   is non-zero (the chunk has missing calls), Q = R + T/2 into RT (column-major n x n, ld ldr;
 *   T is symmetric, so R + R^T + T = Q + Q^T).  At most 16384 SNPs per call.  R runs as
 *   FP64 multiply-adds over each sample's missing SNPs (n per missing call); the same walk
 *   finds the samples missing at those SNPs and adds T/2.  workspace:
 *   jb_kinship_i8_corrections_workspace_size(n, m) bytes.  Every sum runs in a fixed
 *   order: results are bit-reproducible.
 * jb_kinship_i8_finalize: K (n x n, ldk) = symmetric combination above / p_kept.
 */
/*
 * jb_kinship_i8_corrections_tc: the same a, b and Q = R + T/2 updates as
 * jb_kinship_i8_corrections (no reference counterpart: an evaluation of
 * impute_and_center's missing-call terms, src/jamma/kinship/missing.py:22-61), with the
 * dense part R = Z diag(mu) M^T on the INT8 tensor cores: mu_j as four base-254 digits
 * (|error| <= 4.8e-10 per mu_j, mu_j in [0, 2]) interleaved along N of one GEMM per chunk
 * whose A operand is the chunk's columns col0..col0+m of the sample-major Gram operand Zs
 * (col0 and ldz multiples of 16); T/2 = M diag(mu^2/2) M^T from the same dosage-word walk
 * as jb_kinship_i8_corrections without its FMAs.  Faster than the FP64 walk of
 * jb_kinship_i8_corrections only when several per cent of the calls are missing (the
 * dense GEMM costs the same at any density).  workspace: jb_kinship_i8_tc_workspace_size(n,
 * m) bytes, first int32 a status word read with jb_gram_status (non-zero after a pipeline
 * timeout).
 */
int64_t jb_kinship_i8_tc_workspace_size(int64_t n, int64_t m);
int32_t jb_kinship_i8_corrections_tc(const int8_t* codes, int64_t ld_codes, const int8_t* Zs,
                                     int64_t ldz, int64_t col0, int64_t n, int64_t m,
                                     const double* mu, double* a, double* b, double* RT,
                                     int64_t ldr, void* workspace, int64_t workspace_bytes,
                                     uintptr_t stream);

int64_t jb_gram_i8_workspace_size(int64_t n);
int32_t jb_gram_i8(const int8_t* Zs, int64_t n, int64_t p, int64_t ldz, int32_t* C,
                   int64_t ldc, void* workspace, int64_t workspace_bytes, uintptr_t stream);
int32_t jb_gram_status(const void* workspace, int32_t* out, uintptr_t stream);

/*
 * jb_gram_i8_noalloc: the same exact INT8 Gram as jb_gram_i8, for callers that cannot
 * allocate device memory -- e.g. a host application whose memory pool already owns the
 * GPU's free HBM, or code that must not trigger the implicit device synchronisation of
 * cudaMalloc.  It takes no workspace: its scratch (pipeline status word and tile
 * schedule) lives in a 1 MiB static device array inside this library, which every GPU
 * that loads the library keeps until the process exits; n <= 65408 fits, larger n is
 * rejected with JB_E_INVALID and a message.  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress), so make it before any stream capture.
 * The looked-up address is kept for the life of the process, so the device's primary
 * context must not be reset (cudaDeviceReset) after that first call.
 * Every call reuses the one array (the status word is cleared on each call), so calls
 * that overlap on the GPU -- on different streams, or from different host threads --
 * race: serialise them.  No counterpart in the jamma reference.
 *
 * jb_gram_i8_noalloc_status: after jb_gram_i8_noalloc calls on `stream`, copy the
 * pipeline status word of the static scratch to *out (host memory) and synchronise the
 * stream: 0 = OK, non-zero = a bounded tensor-core pipeline wait ran out and C is
 * incomplete.  Allocates nothing.  No counterpart in the jamma reference.
 */
int32_t jb_gram_i8_noalloc(const int8_t* Zs, int64_t n, int64_t p, int64_t ldz, int32_t* C,
                           int64_t ldc, uintptr_t stream);
int32_t jb_gram_i8_noalloc_status(int32_t* out, uintptr_t stream);

/*
 * Test hook of the tensor-core pipelines (no reference counterpart).  Every wait of the
 * INT8 GEMM kernels (jb_gram_i8, jb_gram_i8_noalloc, jb_kinship_i8_corrections_tc,
 * jb_rotate_i8 and jb_lmm_chunk_series_i8 with the one-CTA kernel) is bounded: when its
 * deadline passes, the kernel records 100 + (the waiting role) in its status word, winds
 * down and frees its tensor memory, so the context stays usable.  This call sets the
 * deadline (wait_limit_ns; the default is 2 s) for later launches and, with skip_loads
 * non-zero, makes the producer issue no tile load, so that the first MMA wait runs out
 * with no copy or MMA in flight -- a fault-free way to test that path.  Synchronises the
 * device.  Restore with (0, 2000000000).  Not for production use.
 */
int32_t jb_test_pipeline_timeout(int32_t skip_loads, int64_t wait_limit_ns);
int32_t jb_codes_to_sample_major(const int8_t* codes, int64_t ld_codes, int64_t n,
                                 int64_t m, int8_t* Zs, int64_t ldz, int64_t col0,
                                 int8_t* Cs, int64_t ldcs, uintptr_t stream);
int64_t jb_kinship_i8_corrections_workspace_size(int64_t n, int64_t m);
int32_t jb_kinship_i8_corrections(const int8_t* codes, int64_t ld_codes, int32_t has_missing,
                                  int64_t n, int64_t m, const double* mu, double* a, double* b,
                                  double* RT, int64_t ldr, void* workspace,
                                  int64_t workspace_bytes, uintptr_t stream);
int32_t jb_kinship_i8_finalize(const int32_t* C, int64_t ldc, int64_t n, const double* a,
                               const double* b, double sum_mu2, const double* RT,
                               int64_t ldr, int64_t p_kept, double* K, int64_t ldk,
                               uintptr_t stream);

/*
 * Leave-one-chromosome-out kinship (compute_loco_kinship_streaming,
 * src/jamma/kinship/compute.py:693-916): K_loco = (S_full - S_chr) / p_loco.
 * jb_kinship_i8_finalize_loco: from the full-genome and one chromosome's int32 Grams
 *   (exact integer difference), correction vectors a, b, Q (Q pair may be NULL when no
 *   call is missing) and sum_mu2_loco = sum over the kept non-chromosome SNPs of mu^2.
 * jb_kinship_loco_f64: plain FP64 form from the lower triangles of two centred Grams.
 */
int32_t jb_kinship_i8_finalize_loco(const int32_t* C_full, const int32_t* C_chr, int64_t ldc,
                                    int64_t n, const double* a_full, const double* a_chr,
                                    const double* b_full, const double* b_chr,
                                    double sum_mu2_loco, const double* Q_full,
                                    const double* Q_chr, int64_t ldq, int64_t p_loco,
                                    double* K, int64_t ldk, uintptr_t stream);
int32_t jb_kinship_loco_f64(const double* S_full, const double* S_chr, int64_t n, int64_t lds,
                            int64_t p_loco, double* K, int64_t ldk, uintptr_t stream);

/* ------------------------------------------------------------------ eigen */

/*
 * FP64 symmetric eigendecomposition (cuSOLVER Xsyevd, lower triangle): on return A
 * holds the eigenvectors as columns and w the eigenvalues in ascending order, with
 * |w| < threshold set to 0.  Replaces np.linalg.eigh + thresholding
 * (src/jamma/lmm/eigen.py:94,118).  workspace: jb_eigh_workspace_size bytes.
 * Synchronises the stream (cuSOLVER reports convergence on the host).  Above the
 * single-GPU solver's size limit (n ~ 23 000) it runs cusolverMgSyevd on a one-device
 * grid, which synchronises the whole device; those calls (and their workspace queries)
 * are serialised process-wide, since two at once failed inside the library.
 */
int64_t jb_eigh_workspace_size(int64_t n);
int32_t jb_eigh_f64(double* A, int64_t n, int64_t lda, double* w, double threshold,
                    void* workspace, int64_t workspace_bytes, uintptr_t stream);

/* ------------------------------------------------------------------ rotation */

/*
 * Plain FP64 rotation C (n x m, ldc) = U^T * B with U n x n (ldu) and B n x m (ldb)
 * (cuBLAS DGEMM).  Replaces the host products UT @ G / UT @ W / UT @ y
 * (src/jamma/lmm/runner_streaming.py:349-352,409).
 */
int32_t jb_rotate_f64(const double* U, int64_t n, int64_t ldu, const double* B,
                      int64_t m, int64_t ldb, double* C, int64_t ldc, uintptr_t stream);

/*
 * Tile schedule of the INT8 rotation kernels (no reference counterpart: a launch
 * parameter).  Output tiles (32 eigenvectors x 128 or 256 SNPs) are visited in groups of
 * group_m eigenvector blocks x group_n SNP blocks, which sets which operand slices the
 * persistent CTAs share in L2.  Process-wide; default 9 x 16; set by the autotuner
 * (jamma_b200.autotune).  Applies to launches issued after the call.
 */
int32_t jb_rotate_set_schedule(int32_t group_m, int32_t group_n);
int32_t jb_rotate_get_schedule(int32_t* group_m, int32_t* group_n);

/*
 * GEMM variant of the INT8 rotation kernels (no reference counterpart).  0: one CTA per
 * 128-row x 256-column output tile (tcgen05 cta_group::1).  1: clusters of two CTAs on
 * neighbouring SMs share one 256 x 256 tile (cta_group::2, M = 256): each SM streams half
 * of the B operand, so operand traffic from L2 per MAC falls by a third.  Results are
 * identical (exact integer products).  Process-wide; applies to later launches.
 */
int32_t jb_rotate_set_kernel(int32_t variant);
int32_t jb_rotate_get_kernel(void);

/*
 * Mixed-precision rotation on INT8 tensor cores (replaces the host UT @ G of
 * src/jamma/lmm/runner_streaming.py:409).  jb_ozaki_prepare splits the eigenvectors U
 * (n x n, column-major, ldu) once per cohort into four int8 digit planes (base 254) with a
 * per-eigenvector scale (ozaki workspace: jb_ozaki_workspace_size).  jb_rotate_i8 then
 * forms X = U^T G for m SNPs given as decoded codes (SNP-major, ld_codes a multiple of
 * 16; 3 = missing, mean-imputed with mean[j] without centring): every digit product
 * accumulates exactly in int32 on tcgen05 and the epilogue recombines in FP64
 * (|error| <= ~2.4e-10 max|U_col| * sum|g|: four base-254 digits).  has_missing = 0 promises the chunk holds
 * no missing call.  workspace: jb_rotate_i8_workspace_size(n, m); its first int32 is a
 * pipeline status word (0 = OK), read with jb_rotate_status (synchronises).
 */
int64_t jb_ozaki_workspace_size(int64_t n);
int32_t jb_ozaki_prepare(const double* U, int64_t n, int64_t ldu, void* ozaki_ws,
                         int64_t ozaki_bytes, uintptr_t stream);
int64_t jb_rotate_i8_workspace_size(int64_t n, int64_t m);
int32_t jb_rotate_i8(const void* ozaki_ws, int64_t n, const int8_t* codes, int64_t ld_codes,
                     int64_t m, const double* mean, int32_t has_missing, double* X,
                     int64_t ldx, void* workspace, int64_t workspace_bytes,
                     uintptr_t stream);
int32_t jb_rotate_status(const void* workspace, int32_t* out, uintptr_t stream);

/* ------------------------------------------------------------------ association */

/* Output arrays of jb_lmm_chunk; each is phi x m (phenotype-major, ld = m) or NULL. */
typedef struct jb_lmm_out {
    double* lambda_remle; /* l_remle          (modes 1,4) */
    double* logl_h1;      /* REML logl at it  (modes 1,4) */
    double* beta;         /* Wald beta (1,4) or score beta (3) */
    double* se;
    double* p_wald;       /* (1,4) */
    double* lambda_mle;   /* l_mle            (2,4) */
    double* logl_mle;     /* MLE logl at it   (2,4) */
    double* p_lrt;        /* (2,4) */
    double* p_score;      /* (3,4) */
} jb_lmm_out;

/*
 * Per-SNP association for one rotated chunk, FP64, all phenotypes of a cohort.
 *   evals : n eigenvalues (thresholded)
 *   UtW   : n x n_cvt rotated covariates (ld = ldw)
 *   Uty   : n x phi rotated phenotypes (ld = ldy)
 *   UtG   : n x m rotated genotypes (ld = ldg)
 *   lam0, logl0 : per-phenotype null-model MLE lambda and log-likelihood (modes 2,3,4;
 *                 may be NULL for mode 1)
 * Runs, per (SNP, phenotype): the Score statistics at the null H^-1, the MLE grid +
 * golden-section search and LRT p-value, the REML grid + golden search and the Wald
 * statistics -- whichever lmm_mode (1 Wald, 2 LRT, 3 Score, 4 all) asks for.
 * Replaces batch_compute_uab / batch_compute_iab / golden_section_optimize_lambda[_mle]
 * / batch_calc_wald_stats / batch_calc_score_stats / calc_lrt_pvalue_jax
 * (src/jamma/lmm/likelihood_jax.py:231-883) as driven by
 * src/jamma/lmm/runner_streaming.py:469-554.
 * workspace: jb_lmm_workspace_size bytes, filled by jb_lmm_prepare.
 * chunk_workspace: jb_lmm_chunk_workspace_size(n, n_cvt, phi, n_grid, m) bytes of scratch:
 * the weighted genotype sums of all m SNPs are formed there before the per-SNP kernel runs
 * -- the squared sums sum_i h_i x_i^2 by one fused kernel that reads each rotated genotype
 * once and squares it on chip (FP64, fixed summation order), the linear sums by a cuBLAS
 * DGEMM (precision 0 and 1) or by jb_lmm_chunk_series_i8 (precision 2).  The chunk's
 * precision must match the one its workspace was prepared with (0 with 0; 1 or 2 with 1).
 * precision: 0 = every likelihood evaluation is a direct FP64 reduction over n (plain
 * form; grid, ones and null rows by DGEMM);
 * 1 = mixed form: the c+2 genotype-dependent sums are a degree-95 Chebyshev series in
 * log lambda over [1e-5, 1e5] whose coefficients come from the chunk DGEMMs; log|H^-1|
 * and the genotype-free sums come from per-bracket degree-24 expansions of exact FP64
 * node values (both built by jb_lmm_prepare with precision 1); grid points and golden
 * probes and the final evaluation at each optimum read these series (no pass over the
 * genotypes).  Needs 1e-5 <= l_min < l_max <= 1e5 and
 * 1 + 1e5 * min(eval) > 0.5 (no pole of 1/(lambda eval + 1) near the domain);
 * 2 = as 1, with the linear series sums already placed in chunk_workspace by
 * jb_lmm_chunk_series_i8 for the same chunk (only the squared sums use a DGEMM).
 */
int64_t jb_lmm_workspace_size(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid);

/*
 * Fill the association workspace for one cohort + phenotype set: the numpy-style
 * log-lambda grid (likelihood_jax.py:540-543), the tabulated H = 1/(lambda*eval+1)
 * rows for every grid lambda and every phenotype's null lambda0, log|H^-1| per grid
 * point and the SNP-independent weighted sums.  Must precede jb_lmm_chunk calls that
 * use the same inputs; n_cvt in 1..4.
 */
int32_t jb_lmm_prepare(int32_t lmm_mode, int32_t precision, int64_t n, int32_t n_cvt,
                       int32_t phi, const double* evals, const double* UtW, int64_t ldw,
                       const double* Uty, int64_t ldy, const double* lam0, double l_min,
                       double l_max, int32_t n_grid, void* workspace,
                       int64_t workspace_bytes, uintptr_t stream);

int64_t jb_lmm_chunk_workspace_size(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid,
                                    int64_t m);
int32_t jb_lmm_chunk(int32_t lmm_mode, int32_t precision, int64_t n, int32_t n_cvt,
                     int32_t phi, int64_t m,
                     const double* evals, const double* UtW, int64_t ldw,
                     const double* Uty, int64_t ldy, const double* UtG, int64_t ldg,
                     const double* lam0, const double* logl0, double l_min, double l_max,
                     int32_t n_grid, int32_t n_iter, jb_lmm_out out, void* workspace,
                     int64_t workspace_bytes, void* chunk_workspace, int64_t chunk_bytes,
                     uintptr_t stream);

/*
 * Mixed form, genotype-side linear sums (no reference counterpart: an evaluation order
 * of the sums in likelihood_jax.py:148-186).  The weighted sums sum_i h_i(lambda) x_i v_i
 * of the rotated genotype x = U^T g are linear in g, so with the series tables A_lin of a
 * workspace prepared by jb_lmm_prepare(precision 1) the basis V = U A_lin^T is formed once
 * (one DGEMM) and split into INT8 digit planes like the eigenvectors
 * (jb_ozaki_prepare); every chunk then obtains the linear sums from the int8 calls on the
 * tcgen05 rotation core.  U: column-major eigenvectors (ldu >= n).
 * series_ws: jb_lmm_series_workspace_size(n, n_cvt, phi) bytes, kept per cohort and
 * phenotype set (it depends on W and y).
 */
int64_t jb_lmm_series_workspace_size(int64_t n, int32_t n_cvt, int32_t phi);
/* Rows per linear sum in the series tables: the ones row + the series coefficients; the
 * genotype-side path needs (c + phi) * rows <= n rounded up to 32. */
int32_t jb_lmm_series_rows(void);
int32_t jb_lmm_series_prepare(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid,
                              const void* workspace, int64_t workspace_bytes, const double* U,
                              int64_t ldu, void* series_ws, int64_t series_bytes,
                              uintptr_t stream);

/*
 * Per chunk, after jb_rotate_i8 ran on the same codes with rot_ws on the same stream
 * (its packed [calls | masks] operand and tile list are reused; errors go to the same
 * status word, read by jb_rotate_status): write the chunk's linear series sums into
 * chunk_workspace, then call jb_lmm_chunk with precision 2.  codes / mean / has_missing
 * as for jb_rotate_i8.
 */
int32_t jb_lmm_chunk_series_i8(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid, int64_t m,
                               const void* series_ws, int64_t series_bytes, const int8_t* codes,
                               int64_t ld_codes, const double* mean, int32_t has_missing,
                               void* rot_ws, int64_t rot_bytes, void* chunk_workspace,
                               int64_t chunk_bytes, uintptr_t stream);

/*
 * Null-model MLE (lambda0, logl_H0) per phenotype on the device: the scalar 50-point
 * grid and 20-step golden search of _golden_section_minimize
 * (src/jamma/lmm/likelihood.py:395-474) over mle_log_likelihood_null (349-392), as
 * compute_null_model_mle (571-607) runs it.  lam0, logl0: phi doubles (device).
 */
int32_t jb_null_mle(int64_t n, int32_t n_cvt, int32_t phi, const double* evals,
                    const double* UtW, int64_t ldw, const double* Uty, int64_t ldy,
                    double l_min, double l_max, int32_t n_grid, int32_t n_iter,
                    double* lam0, double* logl0, uintptr_t stream);

#ifdef __cplusplus
}
#endif
#endif /* JAMMA_B200_H */
