// libjamma_b200: per-SNP LMM association (FP64) on B200.
//
// One warp owns one (SNP, phenotype) pair and runs its whole pipeline without
// materialising Uab: the weighted dot products of [W_1..W_c, x, y] are formed on the
// fly from the rotated vectors while streaming them once per likelihood evaluation.
//
//   phase 1  one pass with two fixed weightings: H = 1 (Iab, for REML's logdet term)
//            and H = H0 (the null-model MLE lambda, for the score test);
//   phase 2  the shared lambda grid; every grid point's H row is tabulated once per
//            cohort (SNP independent), the x-free dot products are pre-reduced, so a
//            grid evaluation only needs the c+2 x-dependent sums; REML and MLE grid
//            log-likelihoods come from the same sums;
//   phase 3  JAX-style golden-section refinement for MLE and REML, per-SNP lambda;
//   epilogue Wald (from the final REML evaluation), LRT and score statistics.
//
// Mixed form (precision >= 1): no likelihood evaluation streams x.  The x-dependent sums
// come from the SNP's global Chebyshev series in log lambda (chunk GEMM rows), log|H^-1|
// and the x-free sums from per-bracket expansions; the final evaluation at each optimum
// is one more such probe.
//
// The sequence of evaluations, bracket rules and NaN behaviour follow
// src/jamma/lmm/likelihood_jax.py (148-339 likelihoods, 419-598 search, 601-798
// statistics) exactly; only the summation order of the length-n reductions differs.
#include "jb_common.cuh"
#include "jb_rotate_i8.cuh"

#include <cmath>

namespace jb {
namespace lmm {

constexpr double kPhi = 0.6180339887498949;
constexpr double kPyyMin = 1e-8;
constexpr int kMaxCvt = 4;

template <int C>
struct Lay {
    static constexpr int R = C + 2;  // vector columns: W_0..W_{C-1}, X = C, Y = C+1
    static constexpr int NI = R * (R + 1) / 2;
    static constexpr int NX = C + 2;  // pairs containing X: (W_a,X) a<C, (X,X), (X,Y)
    static constexpr int NS = NI - NX;
    // GEMMA GetabIndex on 0-based columns (src/jamma/lmm/likelihood.py:25-43)
    __host__ __device__ static constexpr int idx(int a, int b) {
        return a <= b ? (2 * R - (a + 1) + 2) * a / 2 + b - a
                      : (2 * R - (b + 1) + 2) * b / 2 + a - b;
    }
};

struct Params {
    int mode;
    int64_t n;
    int phi;
    int64_t m;
    const double* evals;
    const double* W;
    int64_t ldw;
    const double* Y;
    int64_t ldy;
    const double* G;
    int64_t ldg;
    const double* logl0;
    int n_grid;
    int n_iter;
    const double* loglam;  // n_grid
    const double* logdet;  // n_grid
    const double* H;       // (n_grid + phi) x n: grid rows, then null rows
    const double* S;       // (n_grid + 1 + phi) x phi x NS shared sums
    double c_reml, c_mle, df, n_d;
    jb_lmm_out out;
    // mixed form: Chebyshev expansions of the SNP-independent terms per grid bracket
    const double* cheb;    // [n_grid][1 + phi*NS][kChebN] coefficients (NULL: direct)
    const double* cheb_mid;
    const double* cheb_half;
    // Weighted x-sums of every table row r (grid rows, the ones row n_grid, the null rows
    // n_grid+1+f), produced for the whole chunk by two FP64 GEMMs:
    //   CL[j*ldcl + r*(C+phi) + a] = sum_i h_r,i x_ij w_a,i  (a < C)
    //   CL[j*ldcl + r*(C+phi) + C + f] = sum_i h_r,i x_ij y_f,i
    //   CQ[j*ldcq + r] = sum_i h_r,i x_ij^2
    // In the mixed form the rows are the ones row (r = 0) and the kChebG Chebyshev
    // coefficients (r = 1 + k) of the x-dependent sums over the whole log-lambda domain
    // [log 1e-5, log 1e5] (series_xsums), so no probe streams x.
    const double* CL;
    int64_t ldcl;
    const double* CQ;
    int64_t ldcq;
    const double* lam0;  // null-model lambda per phenotype (modes 2-4)
    double gmid, ginv;   // domain centre and 1 / half-width of the global series
};

constexpr int kChebN = 25;  // interpolation nodes (degree 24) per bracket
// Global series of the x-dependent sums: each term 1/(lambda e_i + 1) is analytic in
// t = log lambda in the strip |Im t| < pi, so over the 23-wide domain a Chebyshev series
// converges geometrically (Bernstein ellipse rho ~ 1.31): degree 95 leaves ~1e-13 of the
// sum's scale, far below the ~1e-9 relative error of the INT8-rotated genotypes the sums
// are formed from, and golden-section decisions match those of exact sums.
constexpr int kChebG = 96;
constexpr int kCoefPerLane = kChebG / 32;  // coefficients k = lane + 32 i held by each lane
static_assert(kChebG % 32 == 0, "series length must be a multiple of the warp size");
constexpr double kDomainLo = 1e-5, kDomainHi = 1e5;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double jnan() { return __longlong_as_double(0x7ff8000000000000ll); }
__device__ __forceinline__ double jmax(double a, double b) {  // jnp.maximum: NaN propagates
    return (isnan(a) || isnan(b)) ? jnan() : (a > b ? a : b);
}
__device__ __forceinline__ double clamp_pyy(double v) {
    return (v >= 0.0 && v < kPyyMin) ? kPyyMin : v;
}
__device__ __forceinline__ double rlog(double v) { return v > 0 ? log(v) : 0.0; }

// ---------------------------------------------------------------- special functions
// Regularised incomplete beta I_x(a, b) by the continued fraction of DLMF 8.17.22,
// evaluated with the modified Lentz method (Numerical Recipes 2nd ed. section 6.4):
// direct when x < (a+1)/(a+b+2), else through I_x(a,b) = 1 - I_{1-x}(b,a).
__device__ double betacf(double a, double b, double x) {
    const double tiny = 1e-300, eps = 1e-16;
    const double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (fabs(d) < tiny) d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int k = 1; k <= 4000; ++k) {
        const double k2 = 2.0 * k;
        double aa = k * (b - k) * x / ((qam + k2) * (a + k2));
        d = 1.0 + aa * d;
        if (fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c;
        if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        h *= d * c;
        aa = -(a + k) * (qab + k) * x / ((a + k2) * (qap + k2));
        d = 1.0 + aa * d;
        if (fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c;
        if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (fabs(del - 1.0) < eps) break;
    }
    return h;
}

// log Gamma(a + 1/2) - log Gamma(a) for a >= 25 from the Stirling series of both terms
// (log Gamma(z) = (z - 1/2) log z - z + log(2 pi)/2 + sum_k B_2k / (2k (2k-1) z^(2k-1)))
// expanded in 1/a: 1/2 log a - 1/(8a) + 1/(192 a^3) - 1/(640 a^5) + 17/(14336 a^7)
// - 31/(18432 a^9) + 691/(180224 a^11); the next term is below 1e-20 at a = 25.  The plain
// difference of the two log-gammas cancels ~5 digits at a = df/2 ~ 1e4.
__device__ double lgamma_ratio_half(double a) {
    const double t = 1.0 / a, t2 = t * t;
    const double s = t * (-1.0 / 8 + t2 * (1.0 / 192 + t2 * (-1.0 / 640 + t2 * (17.0 / 14336 +
                     t2 * (-31.0 / 18432 + t2 * (691.0 / 180224))))));
    return 0.5 * log(a) + s;
}

__device__ double betainc_reg(double a, double b, double x) {
    if (isnan(x)) return jnan();
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    // log(1 / B(a, b)); b = 1/2 (every F test here) with large a takes the series above
    const double lb = (b == 0.5 && a >= 25.0) ? lgamma_ratio_half(a) - 0.5723649429247001
                                              : lgamma(a + b) - lgamma(a) - lgamma(b);
    const double lbt = lb + a * log(x) + b * log1p(-x);
    if (x < (a + 1.0) / (a + b + 2.0)) return exp(lbt) * betacf(a, b, x) / a;
    return 1.0 - exp(lbt) * betacf(b, a, 1.0 - x) / b;
}

// F-test p-value as jamma writes it (likelihood_jax.py:668-673,765-771).
__device__ double f_pvalue(double f, double df, bool valid) {
    double z;
    if (isnan(f)) {
        z = jnan();
    } else {
        z = df / (df + (f > 1e-10 ? f : 1e-10));
        z = z < 0.0 ? 0.0 : (z > 1.0 ? 1.0 : z);
    }
    double p = betainc_reg(df / 2.0, 0.5, z);
    if (f <= 0.0) p = 1.0;
    return valid ? p : jnan();
}

// chi-square(1) survival function: P(X > s) = erfc(sqrt(s / 2)).
__device__ double chi2_1_sf(double s) {
    if (isnan(s)) return jnan();
    return erfc(sqrt(0.5 * s));
}

// ---------------------------------------------------------------- Pab
template <int C>
struct PabOut {
    double xx, xy, yy;  // level c (covariates projected out)
    double yy1;         // level c+1 (covariates and genotype projected out)
    double diag[C + 1]; // Pab[i, idx(i,i)], i = 0..c
};

// GEMMA CalcPab recursion (likelihood_jax.py:148-186); inverse of a zero pivot is 0.
template <int C>
__device__ __forceinline__ PabOut<C> pab_reduce(const double (&row0)[Lay<C>::NI]) {
    using L = Lay<C>;
    constexpr int R = L::R;
    double prev[L::NI], cur[L::NI];
    PabOut<C> o;
#pragma unroll
    for (int k = 0; k < L::NI; ++k) prev[k] = cur[k] = row0[k];
    o.diag[0] = prev[L::idx(0, 0)];
#pragma unroll
    for (int p = 1; p <= C + 1; ++p) {
        const int w = p - 1;
        const double ww = prev[L::idx(w, w)];
        const double inv = (ww != 0.0) ? 1.0 / ww : 0.0;
#pragma unroll
        for (int a = p; a < R; ++a) {
#pragma unroll
            for (int b = a; b < R; ++b) {
                const double t = __dmul_rn(__dmul_rn(prev[L::idx(a, w)], prev[L::idx(b, w)]), inv);
                cur[L::idx(a, b)] = __dsub_rn(prev[L::idx(a, b)], t);
            }
        }
        if (p <= C) o.diag[p] = cur[L::idx(p, p)];
        if (p == C) {
            o.xx = cur[L::idx(C, C)];
            o.xy = cur[L::idx(C, C + 1)];
            o.yy = cur[L::idx(C + 1, C + 1)];
        }
#pragma unroll
        for (int k = 0; k < L::NI; ++k) prev[k] = cur[k];
    }
    o.yy1 = prev[L::idx(C + 1, C + 1)];
    return o;
}

// REML log-likelihood (_reml_with_precomputed_iab, likelihood_jax.py:280-339).
template <int C>
__device__ __forceinline__ double reml_logl(const PabOut<C>& pb, const double (&log_iab)[C + 1],
                                            double logdet_h, const Params& p) {
    double ldw = 0.0;
#pragma unroll
    for (int i = 0; i <= C; ++i) {
        ldw = __dadd_rn(ldw, pb.diag[i] > 0 ? log(pb.diag[i]) : 0.0);
        ldw = __dsub_rn(ldw, log_iab[i]);
    }
    const double pyy = clamp_pyy(pb.yy1);
    double f = __dsub_rn(p.c_reml, __dmul_rn(0.5, logdet_h));
    f = __dsub_rn(f, __dmul_rn(0.5, ldw));
    return __dsub_rn(f, __dmul_rn(__dmul_rn(0.5, p.df), log(pyy)));
}

// MLE log-likelihood (mle_log_likelihood_jax, likelihood_jax.py:189-228).
template <int C>
__device__ __forceinline__ double mle_logl(const PabOut<C>& pb, double logdet_h, const Params& p) {
    const double pyy = clamp_pyy(pb.yy1);
    const double f = __dsub_rn(p.c_mle, __dmul_rn(0.5, logdet_h));
    return __dsub_rn(f, __dmul_rn(__dmul_rn(0.5, p.n_d), log(pyy)));
}

// Assemble a full row 0 from pre-reduced x-free sums and fresh x-dependent sums.
template <int C>
__device__ __forceinline__ void assemble(double (&row0)[Lay<C>::NI], const double* shared,
                                         const double (&xs)[Lay<C>::NX]) {
    using L = Lay<C>;
    int s = 0;
#pragma unroll
    for (int a = 0; a < L::R; ++a) {
#pragma unroll
        for (int b = a; b < L::R; ++b) {
            if (a == C || b == C) continue;
            row0[L::idx(a, b)] = shared[s++];
        }
    }
#pragma unroll
    for (int a = 0; a < C; ++a) row0[L::idx(a, C)] = xs[a];
    row0[L::idx(C, C)] = xs[C];
    row0[L::idx(C, C + 1)] = xs[C + 1];
}

// Full evaluation at a per-SNP lambda: H = 1/(lambda*eval + 1), all NI sums + logdet.
// Loads of UNR consecutive strided samples are issued together (memory-level parallelism).
constexpr int UNR = 4;

template <int C>
__device__ __forceinline__ void full_accumulate(double lam, double ev, double xv, double yv,
                                                const double (&w)[C > 0 ? C : 1],
                                                double (&acc)[Lay<C>::NI], double& ld) {
    using L = Lay<C>;
    const double v = __dadd_rn(__dmul_rn(lam, ev), 1.0);
    const double hi = __drcp_rn(v);  // correctly rounded, = 1.0 / v
    ld += log(fabs(v));
    double vec[L::R];
#pragma unroll
    for (int a = 0; a < C; ++a) vec[a] = w[a];
    vec[C] = xv;
    vec[C + 1] = yv;
#pragma unroll
    for (int a = 0; a < L::R; ++a) {
        const double t = hi * vec[a];
#pragma unroll
        for (int b = a; b < L::R; ++b) acc[L::idx(a, b)] = fma(t, vec[b], acc[L::idx(a, b)]);
    }
}

template <int C>
__device__ __forceinline__ void eval_full(const Params& p, const double* __restrict__ x,
                                          const double* __restrict__ y, double lam,
                                          double (&row0)[Lay<C>::NI], double& logdet) {
    using L = Lay<C>;
    double acc[L::NI];
#pragma unroll
    for (int k = 0; k < L::NI; ++k) acc[k] = 0.0;
    double ld = 0.0;
    const int lane = threadIdx.x & 31;
    int64_t i = lane;
    for (; i + 32 * (UNR - 1) < p.n; i += 32 * UNR) {
        double ev[UNR], xv[UNR], yv[UNR], w[UNR][C > 0 ? C : 1];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            ev[u] = __ldg(p.evals + i + 32 * u);
            xv[u] = x[i + 32 * u];
            yv[u] = __ldg(y + i + 32 * u);
#pragma unroll
            for (int a = 0; a < C; ++a) w[u][a] = __ldg(p.W + a * p.ldw + i + 32 * u);
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) full_accumulate<C>(lam, ev[u], xv[u], yv[u], w[u], acc, ld);
    }
    for (; i < p.n; i += 32) {
        double w[C > 0 ? C : 1];
#pragma unroll
        for (int a = 0; a < C; ++a) w[a] = __ldg(p.W + a * p.ldw + i);
        full_accumulate<C>(lam, __ldg(p.evals + i), x[i], __ldg(y + i), w, acc, ld);
    }
#pragma unroll
    for (int k = 0; k < L::NI; ++k) row0[k] = warp_sum(acc[k]);
    logdet = warp_sum(ld);
}

template <int C, bool REML>
__device__ __forceinline__ double eval_logl(const Params& p, const double* x, const double* y,
                                            double log_lam, const double (&log_iab)[C + 1],
                                            PabOut<C>* keep) {
    double row0[Lay<C>::NI];
    double logdet;
    eval_full<C>(p, x, y, exp(log_lam), row0, logdet);
    const PabOut<C> pb = pab_reduce<C>(row0);
    if (keep) *keep = pb;
    return REML ? reml_logl<C>(pb, log_iab, logdet, p) : mle_logl<C>(pb, logdet, p);
}

// Chebyshev series sum_j c_j T_j(t) by Clenshaw's recurrence.
__device__ __forceinline__ double cheb_eval(const double* __restrict__ c, double t) {
    double b1 = 0.0, b2 = 0.0;
    const double t2 = 2.0 * t;
#pragma unroll 5
    for (int j = kChebN - 1; j >= 1; --j) {
        const double b0 = fma(t2, b1, c[j] - b2);
        b2 = b1;
        b1 = b0;
    }
    return fma(t, b1, c[0] - b2);
}

// Mixed form: the c+2 x-dependent sums at log-lambda `s` from the SNP's global Chebyshev
// coefficients (chunk GEMM rows 1..kChebG), by Clenshaw's recurrence.  Every lane
// computes the same values (broadcast loads), so the warp stays uniform.
template <int C>
__device__ __forceinline__ void series_xsums(const Params& p, int64_t j, int f, double s,
                                             double (&xs)[Lay<C>::NX]) {
    using L = Lay<C>;
    const int64_t cp = C + p.phi;
    const double* __restrict__ cl = p.CL + j * p.ldcl;
    const double* __restrict__ cq = p.CQ + j * p.ldcq;
    const double tt = (s - p.gmid) * p.ginv;
    const double t2 = 2.0 * tt;
    double b1[L::NX], b2[L::NX];
#pragma unroll
    for (int q = 0; q < L::NX; ++q) b1[q] = b2[q] = 0.0;
#pragma unroll 4
    for (int k = kChebG - 1; k >= 1; --k) {
        const double* rl = cl + (1 + k) * cp;
        double c[L::NX];
#pragma unroll
        for (int a = 0; a < C; ++a) c[a] = __ldg(rl + a);
        c[C] = __ldg(cq + 1 + k);
        c[C + 1] = __ldg(rl + C + f);
#pragma unroll
        for (int q = 0; q < L::NX; ++q) {
            const double b0 = fma(t2, b1[q], c[q] - b2[q]);
            b2[q] = b1[q];
            b1[q] = b0;
        }
    }
    const double* rl = cl + cp;
    double c[L::NX];
#pragma unroll
    for (int a = 0; a < C; ++a) c[a] = __ldg(rl + a);
    c[C] = __ldg(cq + 1);
    c[C + 1] = __ldg(rl + C + f);
#pragma unroll
    for (int q = 0; q < L::NX; ++q) xs[q] = fma(tt, b1[q], c[q] - b2[q]);
}

// ---------------------------------------------------------------- warp-cooperative series
// Chebyshev values for a series summed across the warp: lane l gets T_l(x) (l = 0..31)
// and every lane T_32(x), by the doubling identity T_{a+b} = 2 T_a T_b - T_{a-b} (round r
// fills lanes 2^r+1 .. 2^(r+1) from lanes already known).
__device__ __forceinline__ void lane_cheb(double x, double& tl, double& t32) {
    const int lane = threadIdx.x & 31;
    tl = lane == 0 ? 1.0 : x;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int a = 1 << r;
        const bool act = lane > a && lane <= 2 * a;
        const double ta = __shfl_sync(0xffffffffu, tl, a);
        const double tb = __shfl_sync(0xffffffffu, tl, act ? lane - a : 0);
        const double tc = __shfl_sync(0xffffffffu, tl, act ? 2 * a - lane : 0);
        if (act) tl = fma(2.0 * ta, tb, -tc);
    }
    const double t16 = __shfl_sync(0xffffffffu, tl, 16);
    t32 = fma(2.0 * t16, t16, -1.0);
}

// T_k(x) for the coefficients a lane owns: k = lane + 32 i, i < kCoefPerLane.
struct LaneT {
    double t[kCoefPerLane];
};
__device__ __forceinline__ LaneT lane_cheb_global(double x) {
    const int lane = threadIdx.x & 31;
    double tl, t32;
    lane_cheb(x, tl, t32);
    const double tm = __shfl_sync(0xffffffffu, tl, (32 - lane) & 31);  // T_{32-l}
    LaneT r;
    r.t[0] = tl;
    r.t[1] = fma(2.0 * t32, tl, -(lane == 0 ? t32 : tm));  // T_{l+32}
#pragma unroll
    for (int i = 2; i < kCoefPerLane; ++i)
        r.t[i] = fma(2.0 * t32, r.t[i - 1], -r.t[i - 2]);   // T_{l+32i}
    return r;
}

// Per-(SNP, phenotype) coefficients of the global x-sum series, spread over the warp
// (lane l holds k = l + 32 i of every series), loaded once per SNP.
template <int C>
struct GlobalCoef {
    double c[Lay<C>::NX][kCoefPerLane];
};
template <int C>
__device__ __forceinline__ GlobalCoef<C> load_global_coef(const Params& p, int64_t j, int f) {
    const int lane = threadIdx.x & 31;
    const int64_t cp = C + p.phi;
    GlobalCoef<C> g;
#pragma unroll
    for (int i = 0; i < kCoefPerLane; ++i) {
        const int64_t r = 1 + lane + 32 * i;
        const double* rl = p.CL + j * p.ldcl + r * cp;
#pragma unroll
        for (int a = 0; a < C; ++a) g.c[a][i] = __ldg(rl + a);
        g.c[C][i] = __ldg(p.CQ + j * p.ldcq + r);
        g.c[C + 1][i] = __ldg(rl + C + f);
    }
    return g;
}

// The c+2 x-dependent sums at log-lambda s; identical bits in every lane.
template <int C>
__device__ __forceinline__ void coop_xsums(const Params& p, const GlobalCoef<C>& g, double s,
                                           double (&xs)[Lay<C>::NX]) {
    const LaneT T = lane_cheb_global((s - p.gmid) * p.ginv);
#pragma unroll
    for (int q = 0; q < Lay<C>::NX; ++q) {
        double v = g.c[q][0] * T.t[0];
#pragma unroll
        for (int i = 1; i < kCoefPerLane; ++i) v = fma(g.c[q][i], T.t[i], v);
        xs[q] = warp_sum(v);
    }
}

// Per-bracket expansions of log|H^-1| and the x-free sums of phenotype f (degree 24 over
// the golden bracket of grid index `best`): lane j < kChebN holds coefficient j.
template <int C>
struct BracketCoef {
    double c[1 + Lay<C>::NS];
    double mid, inv_half;
};
template <int C>
__device__ __forceinline__ BracketCoef<C> load_bracket_coef(const Params& p, int best, int f) {
    using L = Lay<C>;
    const int lane = threadIdx.x & 31;
    const int nf = 1 + p.phi * L::NS;
    const double* cb = p.cheb + (int64_t)best * nf * kChebN;
    BracketCoef<C> b;
    b.c[0] = lane < kChebN ? __ldg(cb + lane) : 0.0;
#pragma unroll
    for (int k = 0; k < L::NS; ++k)
        b.c[1 + k] = lane < kChebN ? __ldg(cb + (1 + f * L::NS + k) * kChebN + lane) : 0.0;
    b.mid = p.cheb_mid[best];
    b.inv_half = 1.0 / p.cheb_half[best];
    return b;
}

// log|H^-1| and the x-free sums at log-lambda s inside the bracket; identical bits in
// every lane.
template <int C>
__device__ __forceinline__ void coop_shared(const BracketCoef<C>& b, double s, double& logdet,
                                            double (&shared)[Lay<C>::NS]) {
    double tl, t32;
    lane_cheb((s - b.mid) * b.inv_half, tl, t32);
    logdet = warp_sum(b.c[0] * tl);
#pragma unroll
    for (int k = 0; k < Lay<C>::NS; ++k) shared[k] = warp_sum(b.c[1 + k] * tl);
}

// Mixed-form log-likelihood at log-lambda s with no length-n pass: the x-dependent sums
// from the SNP's global series, log|H^-1| and the x-free sums from the bracket's expansions
// (exact FP64 node values).  The golden-section probes use it; the final evaluation at
// the optimum takes the same steps in lmm_pairs_kernel, where direct_fix may replace the
// x-dependent sums by direct ones at large lambda.  pb receives the Pab rows.
template <int C, bool REML>
__device__ __forceinline__ double coop_eval(const Params& p, const GlobalCoef<C>& g,
                                            const BracketCoef<C>& b, double s,
                                            const double (&log_iab)[C + 1], PabOut<C>& pb) {
    using L = Lay<C>;
    double xs[L::NX], shared[L::NS], logdet;
    coop_xsums<C>(p, g, s, xs);
    coop_shared<C>(b, s, logdet, shared);
    double row0[L::NI];
    assemble<C>(row0, shared, xs);
    pb = pab_reduce<C>(row0);
    return REML ? reml_logl<C>(pb, log_iab, logdet, p) : mle_logl<C>(pb, logdet, p);
}

template <int C, bool REML>
__device__ __forceinline__ double coop_logl(const Params& p, const GlobalCoef<C>& g,
                                            const BracketCoef<C>& b, double s,
                                            const double (&log_iab)[C + 1]) {
    PabOut<C> pb;
    return coop_eval<C, REML>(p, g, b, s, log_iab, pb);
}

// Golden-section refinement (_golden_section_refine, likelihood_jax.py:419-488) on the
// mixed-form likelihood; returns the optimum's log-lambda (a + b) / 2 and the bracket's
// expansions for the final evaluation.
template <int C, bool REML>
__device__ double golden_coop(const Params& p, const GlobalCoef<C>& g, int best, int f,
                              const double (&log_iab)[C + 1], BracketCoef<C>& bc) {
    const int lo = best - 1 > 0 ? best - 1 : 0;
    const int hi = best + 1 < p.n_grid - 1 ? best + 1 : p.n_grid - 1;
    bc = load_bracket_coef<C>(p, best, f);
    auto probe = [&](double s) { return coop_logl<C, REML>(p, g, bc, s, log_iab); };
    double a = p.loglam[lo], b = p.loglam[hi];
    double c = __dsub_rn(b, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double d = __dadd_rn(a, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double fc = probe(c);
    double fd = probe(d);
    for (int it = 0; it < p.n_iter; ++it) {
        const bool keep_left = fc > fd;
        const double na = keep_left ? a : c;
        const double nb = keep_left ? d : b;
        const double nc = __dsub_rn(nb, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nd = __dadd_rn(na, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nl = probe(keep_left ? nc : nd);
        const double nfc = keep_left ? nl : fd;
        const double nfd = keep_left ? fc : nl;
        a = na; b = nb; c = nc; d = nd; fc = nfc; fd = nfd;
    }
    return __dmul_rn(__dadd_rn(a, b), 0.5);
}

// Grid bracket + golden section (_golden_section_refine, likelihood_jax.py:419-488).
template <int C, bool REML>
__device__ void golden(const Params& p, const double* x, const double* y, int best,
                       const double (&log_iab)[C + 1], double& lam_out, double& logl_out,
                       PabOut<C>& pb_out) {
    const int lo = best - 1 > 0 ? best - 1 : 0;
    const int hi = best + 1 < p.n_grid - 1 ? best + 1 : p.n_grid - 1;
    auto probe = [&](double s) { return eval_logl<C, REML>(p, x, y, s, log_iab, nullptr); };
    double a = p.loglam[lo], b = p.loglam[hi];
    double c = __dsub_rn(b, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double d = __dadd_rn(a, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double fc = probe(c);
    double fd = probe(d);
    for (int it = 0; it < p.n_iter; ++it) {
        const bool keep_left = fc > fd;
        const double na = keep_left ? a : c;
        const double nb = keep_left ? d : b;
        const double nc = __dsub_rn(nb, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nd = __dadd_rn(na, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nl = probe(keep_left ? nc : nd);
        const double nfc = keep_left ? nl : fd;
        const double nfd = keep_left ? fc : nl;
        a = na; b = nb; c = nc; d = nd; fc = nfc; fd = nfd;
    }
    const double log_opt = __dmul_rn(__dadd_rn(a, b), 0.5);
    lam_out = exp(log_opt);
    logl_out = eval_logl<C, REML>(p, x, y, log_opt, log_iab, &pb_out);
}

// ---------------------------------------------------------------- two pairs per warp
// The mixed-form search with one (SNP, phenotype) pair per half-warp and exactly the values
// of the one-pair-per-warp form above: lane l (< 16) of a half stands in for that form's
// lanes l ("v0") and l + 16 ("v1").  It holds both lanes' Chebyshev values, coefficients
// and partial sums, built by the same formulas from the same inputs, and folds them with
// the first (offset-16) step of the warp butterfly; the other four steps run across the
// half.  Every value and the order of every sum match, so results are bit-identical, while
// the per-probe scalar work (Pab recursion, logs, golden-section bookkeeping) that every
// lane repeats now serves two pairs per instruction.
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double fold_sum(double p0, double p1) {
    double v = __dadd_rn(p0, p1);  // offset 16: v_l + v_{l^16} (never contracted into an FMA)
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// lane_cheb's T_l and T_{l+16} (32-lane doubling rounds) and T_32.
__device__ __forceinline__ void lane_cheb_v(double x, double& t0, double& t1, double& t32) {
    const int lane = threadIdx.x & 15;
    double tl = lane == 0 ? 1.0 : x;
#pragma unroll
    for (int r = 0; r < 4; ++r) {  // a = 1, 2, 4, 8 (lanes above 16 are idle in these rounds)
        const int a = 1 << r;
        const bool act = lane > a && lane <= 2 * a;
        const double ta = __shfl_sync(kFull, tl, a, 16);
        const double tb = __shfl_sync(kFull, tl, act ? lane - a : 0, 16);
        const double tc = __shfl_sync(kFull, tl, act ? 2 * a - lane : 0, 16);
        if (act) tl = fma(2.0 * ta, tb, -tc);
    }
    const double t8 = __shfl_sync(kFull, tl, 8, 16);
    const double t16 = fma(2.0 * t8, t8, -1.0);  // lane 16 at a = 8: 2 T_8 T_8 - T_0
    const double tmir = __shfl_sync(kFull, tl, (16 - lane) & 15, 16);  // T_{16-l}
    t0 = tl;
    t1 = lane == 0 ? t16 : fma(2.0 * t16, tl, -tmir);  // lanes 17..31 at a = 16
    t32 = fma(2.0 * t16, t16, -1.0);
}

struct LaneTV {
    double t0[kCoefPerLane], t1[kCoefPerLane];
};
__device__ __forceinline__ LaneTV lane_cheb_global_v(double x) {
    const int lane = threadIdx.x & 15;
    double t0, t1, t32;
    lane_cheb_v(x, t0, t1, t32);
    const double a = __shfl_sync(kFull, t0, (16 - lane) & 15, 16);  // T_{16-l}
    const double b = __shfl_sync(kFull, t1, (16 - lane) & 15, 16);  // T_{32-l}
    LaneTV r;
    r.t0[0] = t0;
    r.t1[0] = t1;
    r.t0[1] = fma(2.0 * t32, t0, -(lane == 0 ? t32 : b));  // T_{l+32}
    r.t1[1] = fma(2.0 * t32, t1, -(lane == 0 ? t1 : a));   // T_{l+48}
#pragma unroll
    for (int i = 2; i < kCoefPerLane; ++i) {
        r.t0[i] = fma(2.0 * t32, r.t0[i - 1], -r.t0[i - 2]);
        r.t1[i] = fma(2.0 * t32, r.t1[i - 1], -r.t1[i - 2]);
    }
    return r;
}

template <int C>
struct GlobalCoefV {
    GlobalCoef<C> v0, v1;
};
template <int C>
__device__ __forceinline__ GlobalCoefV<C> load_global_coef_v(const Params& p, int64_t j, int f) {
    const int lane = threadIdx.x & 15;
    const int64_t cp = C + p.phi;
    GlobalCoefV<C> g;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        GlobalCoef<C>& gg = h ? g.v1 : g.v0;
#pragma unroll
        for (int i = 0; i < kCoefPerLane; ++i) {
            const int64_t r = 1 + lane + 16 * h + 32 * i;
            const double* rl = p.CL + j * p.ldcl + r * cp;
#pragma unroll
            for (int a = 0; a < C; ++a) gg.c[a][i] = __ldg(rl + a);
            gg.c[C][i] = __ldg(p.CQ + j * p.ldcq + r);
            gg.c[C + 1][i] = __ldg(rl + C + f);
        }
    }
    return g;
}

template <int C>
__device__ __forceinline__ void coop_xsums_v(const Params& p, const GlobalCoefV<C>& g, double s,
                                             double (&xs)[Lay<C>::NX]) {
    const LaneTV T = lane_cheb_global_v((s - p.gmid) * p.ginv);
#pragma unroll
    for (int q = 0; q < Lay<C>::NX; ++q) {
        double v0 = g.v0.c[q][0] * T.t0[0], v1 = g.v1.c[q][0] * T.t1[0];
#pragma unroll
        for (int i = 1; i < kCoefPerLane; ++i) {
            v0 = fma(g.v0.c[q][i], T.t0[i], v0);
            v1 = fma(g.v1.c[q][i], T.t1[i], v1);
        }
        xs[q] = fold_sum(v0, v1);
    }
}

template <int C>
struct BracketCoefV {
    BracketCoef<C> v0, v1;
};
template <int C>
__device__ __forceinline__ BracketCoefV<C> load_bracket_coef_v(const Params& p, int best, int f) {
    using L = Lay<C>;
    const int lane = threadIdx.x & 15;
    const int nf = 1 + p.phi * L::NS;
    const double* cb = p.cheb + (int64_t)best * nf * kChebN;
    BracketCoefV<C> b;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        BracketCoef<C>& bb = h ? b.v1 : b.v0;
        const int jj = lane + 16 * h;
        bb.c[0] = jj < kChebN ? __ldg(cb + jj) : 0.0;
#pragma unroll
        for (int k = 0; k < L::NS; ++k)
            bb.c[1 + k] = jj < kChebN ? __ldg(cb + (1 + f * L::NS + k) * kChebN + jj) : 0.0;
        bb.mid = p.cheb_mid[best];
        bb.inv_half = 1.0 / p.cheb_half[best];
    }
    return b;
}

template <int C>
__device__ __forceinline__ void coop_shared_v(const BracketCoefV<C>& b, double s, double& logdet,
                                              double (&shared)[Lay<C>::NS]) {
    double t0, t1, t32;
    lane_cheb_v((s - b.v0.mid) * b.v0.inv_half, t0, t1, t32);
    logdet = fold_sum(b.v0.c[0] * t0, b.v1.c[0] * t1);
#pragma unroll
    for (int k = 0; k < Lay<C>::NS; ++k) shared[k] = fold_sum(b.v0.c[1 + k] * t0, b.v1.c[1 + k] * t1);
}

template <int C, bool REML>
__device__ __forceinline__ double coop_eval_v(const Params& p, const GlobalCoefV<C>& g,
                                              const BracketCoefV<C>& b, double s,
                                              const double (&log_iab)[C + 1], PabOut<C>& pb) {
    using L = Lay<C>;
    double xs[L::NX], shared[L::NS], logdet;
    coop_xsums_v<C>(p, g, s, xs);
    coop_shared_v<C>(b, s, logdet, shared);
    double row0[L::NI];
    assemble<C>(row0, shared, xs);
    pb = pab_reduce<C>(row0);
    return REML ? reml_logl<C>(pb, log_iab, logdet, p) : mle_logl<C>(pb, logdet, p);
}

template <int C, bool REML>
__device__ __forceinline__ double coop_logl_v(const Params& p, const GlobalCoefV<C>& g,
                                              const BracketCoefV<C>& b, double s,
                                              const double (&log_iab)[C + 1]) {
    PabOut<C> pb;
    return coop_eval_v<C, REML>(p, g, b, s, log_iab, pb);
}

template <int C, bool REML>
__device__ double golden_coop_v(const Params& p, const GlobalCoefV<C>& g, int best, int f,
                                const double (&log_iab)[C + 1], BracketCoefV<C>& bc) {
    const int lo = best - 1 > 0 ? best - 1 : 0;
    const int hi = best + 1 < p.n_grid - 1 ? best + 1 : p.n_grid - 1;
    bc = load_bracket_coef_v<C>(p, best, f);
    auto probe = [&](double s) { return coop_logl_v<C, REML>(p, g, bc, s, log_iab); };
    double a = p.loglam[lo], b = p.loglam[hi];
    double c = __dsub_rn(b, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double d = __dadd_rn(a, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double fc = probe(c);
    double fd = probe(d);
    for (int it = 0; it < p.n_iter; ++it) {
        const bool keep_left = fc > fd;
        const double na = keep_left ? a : c;
        const double nb = keep_left ? d : b;
        const double nc = __dsub_rn(nb, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nd = __dadd_rn(na, __dmul_rn(kPhi, __dsub_rn(nb, na)));
        const double nl = probe(keep_left ? nc : nd);
        const double nfc = keep_left ? nl : fd;
        const double nfd = keep_left ? fc : nl;
        a = na; b = nb; c = nc; d = nd; fc = nfc; fd = nfd;
    }
    return __dmul_rn(__dadd_rn(a, b), 0.5);
}

// jnp.argmax semantics: first maximum, NaN wins (first NaN).
struct ArgMax {
    int idx = -1;
    double v = 0.0;
    __device__ void push(int i, double x) {
        if (idx < 0) { idx = i; v = x; return; }
        if (isnan(v)) return;
        if (isnan(x) || x > v) { idx = i; v = x; }
    }
    // Merge with a partial result over other indices (any order): the lowest-index NaN
    // if there is one, else the maximum with the lowest index among ties -- the same
    // pick as pushing every index in increasing order.
    __device__ void merge(int i, double x) {
        if (i < 0) return;
        if (idx < 0) { idx = i; v = x; return; }
        const bool na = isnan(v), nb = isnan(x);
        if (na || nb) {
            if (na && nb ? i < idx : nb) { idx = i; v = x; }
            return;
        }
        if (x > v || (x == v && i < idx)) { idx = i; v = x; }
    }
    template <int GW = 32>
    __device__ void warp_reduce() {  // over groups of GW lanes
#pragma unroll
        for (int o = GW / 2; o > 0; o >>= 1) {
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            merge(oi, ov);
        }
    }
};

template <int C>
__device__ __forceinline__ void beta_se(const PabOut<C>& pb, double px_yy, double df, bool& valid,
                                        double& beta, double& tau, double& se) {
    valid = pb.xx > 0;
    const double safe_xx = valid ? pb.xx : 1.0;
    beta = valid ? pb.xy / safe_xx : jnan();
    tau = df / px_yy;
    double var = valid ? 1.0 / (tau * safe_xx) : jnan();
    var = fabs(var) < 0.001 ? fabs(var) : var;
    se = valid ? sqrt(var) : jnan();
}

// Mixed form at large lambda.  The series' error in an x-dependent sum is fixed in absolute
// terms (a small fraction of the sum's size at small lambda, where every weight
// 1/(lambda e_i + 1) is near 1), while the sums the statistics use shrink like
// 1/(lambda e): at lambda = 1e5 the projected P_xy, P_xx are ~1e-5 of their small-lambda
// size and the score and LRT p-values moved by up to 2e-4 relative against the FP64 form
// (n = 20 000, 64 phenotypes whose null lambda sat on the upper bound).  The error grows
// about linearly in lambda (4e-8 at lambda = 10), so every final evaluation at
// lambda >= kDirectLam -- the score at the null lambda, the MLE and REML optima -- reduces
// its sums directly in FP64 over the rotated genotypes instead (one pass over x).  The
// search itself stays on the series.
constexpr double kDirectLam = 20.0;
constexpr double kLogDirectLam = 2.995732273553991;  // log(kDirectLam)

// The x-dependent sums of one pair at up to three lambdas (the score's null lambda, the
// MLE and REML optima; on[q] the same in every lane) in one warp-cooperative pass over the
// rotated genotypes, each term formed as full_accumulate forms it.
template <int C>
__device__ __forceinline__ void direct_xsums3(const Params& p, const double* __restrict__ x,
                                              const double* __restrict__ y,
                                              const double (&lam)[3], const bool (&on)[3],
                                              double (&xs)[3][Lay<C>::NX]) {
    using L = Lay<C>;
    double acc[3][L::NX];
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int k = 0; k < L::NX; ++k) acc[q][k] = 0.0;
    auto term = [&](double ev, double xv, double yv, const double (&w)[C > 0 ? C : 1]) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (!on[q]) continue;
            const double hi = __drcp_rn(__dadd_rn(__dmul_rn(lam[q], ev), 1.0));
#pragma unroll
            for (int a = 0; a < C; ++a) acc[q][a] = fma(hi * w[a], xv, acc[q][a]);
            const double t = hi * xv;
            acc[q][C] = fma(t, xv, acc[q][C]);
            acc[q][C + 1] = fma(t, yv, acc[q][C + 1]);
        }
    };
    // UNR consecutive strided samples' loads issued together (memory-level parallelism)
    int64_t i = threadIdx.x & 31;
    for (; i + 32 * (UNR - 1) < p.n; i += 32 * UNR) {
        double ev[UNR], xv[UNR], yv[UNR], w[UNR][C > 0 ? C : 1];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            ev[u] = __ldg(p.evals + i + 32 * u);
            xv[u] = x[i + 32 * u];
            yv[u] = __ldg(y + i + 32 * u);
#pragma unroll
            for (int a = 0; a < C; ++a) w[u][a] = __ldg(p.W + a * p.ldw + i + 32 * u);
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) term(ev[u], xv[u], yv[u], w[u]);
    }
    for (; i < p.n; i += 32) {
        double w[C > 0 ? C : 1];
#pragma unroll
        for (int a = 0; a < C; ++a) w[a] = __ldg(p.W + a * p.ldw + i);
        term(__ldg(p.evals + i), x[i], __ldg(y + i), w);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int k = 0; k < L::NX; ++k) xs[q][k] = on[q] ? warp_sum(acc[q][k]) : 0.0;
}

// Pairs with a final lambda >= kDirectLam: the whole warp takes each such pair of its
// 32 / GW groups in turn and reduces its x-dependent sums directly.  The score statistic
// is recomputed and rewritten here (the group's lane 0 overwrites the series value); the
// MLE / REML sums replace xs_m / xs_r of the owning group, which then evaluates them with
// its bracket-expanded x-free sums and log-determinant as before.
template <int C, int GW>
__device__ __forceinline__ void direct_fix(const Params& p, int64_t j, int f, bool valid_pair,
                                           bool need_score, bool need_mle, bool need_reml,
                                           double s_m, double s_r, double (&xs_m)[Lay<C>::NX],
                                           double (&xs_r)[Lay<C>::NX]) {
    using L = Lay<C>;
    const int mine = (int)(threadIdx.x & 31) / GW;
#pragma unroll 1
    for (int h = 0; h < 32 / GW; ++h) {
        const int src = h * GW;
        const int fh = __shfl_sync(kFull, f, src);
        const double sm = __shfl_sync(kFull, s_m, src), sr = __shfl_sync(kFull, s_r, src);
        const double lam0 = need_score ? p.lam0[fh] : 0.0;
        const bool on[3] = {need_score && lam0 >= kDirectLam, need_mle && sm >= kLogDirectLam,
                            need_reml && sr >= kLogDirectLam};
        if (!on[0] && !on[1] && !on[2]) continue;  // the same decision in every lane
        const long long jh = __shfl_sync(kFull, (long long)j, src);
        const bool vh = __shfl_sync(kFull, (int)valid_pair, src) != 0;
        const double lam[3] = {lam0, exp(sm), exp(sr)};
        double xs[3][L::NX];
        direct_xsums3<C>(p, p.G + jh * p.ldg, p.Y + (int64_t)fh * p.ldy, lam, on, xs);
        if (on[0]) {
            double row0[L::NI];
            assemble<C>(row0, p.S + (int64_t)(p.n_grid + 1 + fh) * p.phi * L::NS + (int64_t)fh * L::NS,
                        xs[0]);
            const PabOut<C> pb = pab_reduce<C>(row0);
            bool valid;
            double beta, tau, se;
            beta_se<C>(pb, clamp_pyy(pb.yy1), p.df, valid, beta, tau, se);
            const double fstat = p.n_d * (pb.xy * pb.xy) / (pb.yy * (valid ? pb.xx : 1.0));
            if ((int)(threadIdx.x & 31) == src && vh) {
                const int64_t o = (int64_t)fh * p.m + jh;
                if (p.out.p_score) p.out.p_score[o] = valid ? fstat : jnan();
                if (p.mode == 3) {
                    if (p.out.beta) p.out.beta[o] = beta;
                    if (p.out.se) p.out.se[o] = se;
                }
            }
        }
        if (mine == h) {
#pragma unroll
            for (int k = 0; k < L::NX; ++k) {
                if (on[1]) xs_m[k] = xs[1][k];
                if (on[2]) xs_r[k] = xs[2][k];
            }
        }
    }
}

// 4 warps per block; with one covariate at least 5 blocks per SM (<= 102 registers, 20
// resident warps to hide FP64 and shuffle latency), fewer for wider covariate sets whose
// per-warp state would otherwise spill.
constexpr int kPairsThreads = 128;
template <int C>
struct PairsOccupancy {
    static constexpr int kMinBlocks = C == 1 ? 4 : (C == 2 ? 3 : 2);  // C = 1: 125 registers, no spill
    // two pairs per warp: each lane holds two virtual lanes' state (C = 1: 160 registers,
    // no spill; 4 blocks at 128 registers measured within 0.5 %)
    static constexpr int kMinBlocksHalf = 3;
};

// One (SNP, phenotype) pair per group of GW lanes: a warp (GW = 32), or a half-warp in the
// mixed form with one covariate column (GW = 16, the bit-identical two-pairs-per-warp
// helpers above).  Every lane of a warp runs the same control flow: a group past the last
// pair repeats the last pair and writes nothing.
template <int C, bool INTERP, int GW>
__global__ void __launch_bounds__(kPairsThreads, GW == 16 ? PairsOccupancy<C>::kMinBlocksHalf
                                                            : PairsOccupancy<C>::kMinBlocks)
    lmm_pairs_kernel(const Params p) {
    using L = Lay<C>;
    static_assert(GW == 32 || (INTERP && GW == 16), "half-warp pairs are a mixed-form path");
    const int64_t npairs = p.m * p.phi;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if ((tid & ~31ll) / GW >= npairs) return;  // the whole warp is idle
    const bool valid_pair = tid / GW < npairs;
    const int64_t wid = valid_pair ? tid / GW : npairs - 1;
    const int lane = threadIdx.x & (GW - 1);
    const int64_t j = wid / p.phi;
    const int f = (int)(wid % p.phi);
    const double* __restrict__ x = p.G + j * p.ldg;
    const double* __restrict__ y = p.Y + (int64_t)f * p.ldy;
    const bool need_reml = p.mode == 1 || p.mode == 4;
    const bool need_mle = p.mode == 2 || p.mode == 4;
    const bool need_score = p.mode == 3 || p.mode == 4;
    const int64_t o = (int64_t)f * p.m + j;
    const int64_t srow = (int64_t)p.phi * L::NS;  // stride of one S row

    // Weighted x-sums of table row r for this (SNP, phenotype), from the chunk GEMMs.
    auto row_xsums = [&](int r, double (&xs)[L::NX]) {
        const double* cl = p.CL + j * p.ldcl + (int64_t)r * (C + p.phi);
#pragma unroll
        for (int a = 0; a < C; ++a) xs[a] = cl[a];
        xs[C] = p.CQ[j * p.ldcq + r];
        xs[C + 1] = cl[C + f];
    };

    // mixed form: this SNP's global series coefficients, spread over the warp
    GlobalCoef<C> gc;
    GlobalCoefV<C> gcv;
    if constexpr (INTERP && GW == 16)
        gcv = load_global_coef_v<C>(p, j, f);
    else if (INTERP)
        gc = load_global_coef<C>(p, j, f);

    // ---------------- phase 1: H = 1 (Iab) and H = H0 (score)
    double log_iab[C + 1];
#pragma unroll
    for (int i = 0; i <= C; ++i) log_iab[i] = 0.0;
    if (need_reml) {
        double xs[L::NX], row0[L::NI];
        row_xsums(INTERP ? 0 : p.n_grid, xs);
        assemble<C>(row0, p.S + (int64_t)p.n_grid * srow + (int64_t)f * L::NS, xs);
        const PabOut<C> pb = pab_reduce<C>(row0);
#pragma unroll
        for (int i = 0; i <= C; ++i) log_iab[i] = pb.diag[i] > 0 ? log(pb.diag[i]) : 0.0;
    }
    if (need_score) {
        double xs[L::NX], row0[L::NI];
        if constexpr (INTERP && GW == 16)
            coop_xsums_v<C>(p, gcv, log(p.lam0[f]), xs);
        else if (INTERP)
            coop_xsums<C>(p, gc, log(p.lam0[f]), xs);
        else
            row_xsums(p.n_grid + 1 + f, xs);
        assemble<C>(row0, p.S + (int64_t)(p.n_grid + 1 + f) * srow + (int64_t)f * L::NS, xs);
        const PabOut<C> pb = pab_reduce<C>(row0);
        bool valid;
        double beta, tau, se;
        beta_se<C>(pb, clamp_pyy(pb.yy1), p.df, valid, beta, tau, se);
        const double fstat = p.n_d * (pb.xy * pb.xy) / (pb.yy * (valid ? pb.xx : 1.0));
        if (lane == 0 && valid_pair) {
            // the F statistic (NaN: no test); lmm_fpvalue_kernel turns it into the p-value
            if (p.out.p_score) p.out.p_score[o] = valid ? fstat : jnan();
            if (p.mode == 3) {
                if (p.out.beta) p.out.beta[o] = beta;
                if (p.out.se) p.out.se[o] = se;
            }
        }
    }
    if (!need_reml && !need_mle) {
        if constexpr (INTERP) {  // score only: the large-lambda rewrite happens here
            double xs_m[L::NX], xs_r[L::NX];
            direct_fix<C, GW>(p, j, f, valid_pair, need_score, false, false, 0.0, 0.0, xs_m, xs_r);
        }
        return;
    }

    // ---------------- phase 2: shared lambda grid
    ArgMax best_reml, best_mle;
    // mixed form: lanes take grid points lane, lane+GW, ... from the series, then merge
    for (int g = INTERP ? lane : 0; g < p.n_grid; g += INTERP ? GW : 1) {
        double xs[L::NX], row0[L::NI];
        if (INTERP)
            series_xsums<C>(p, j, f, p.loglam[g], xs);
        else
            row_xsums(g, xs);
        assemble<C>(row0, p.S + (int64_t)g * srow + (int64_t)f * L::NS, xs);
        const PabOut<C> pb = pab_reduce<C>(row0);
        const double ldh = p.logdet[g];
        if (need_reml) best_reml.push(g, reml_logl<C>(pb, log_iab, ldh, p));
        if (need_mle) best_mle.push(g, mle_logl<C>(pb, ldh, p));
    }
    if (INTERP) {
        best_reml.warp_reduce<GW>();
        best_mle.warp_reduce<GW>();
    }

    // ---------------- phase 3: golden sections + statistics
    double lam_m = 0.0, logl_m = 0.0, lam_r = 0.0, logl_r = 0.0;
    double s_m = 0.0, s_r = 0.0;  // mixed form: log-lambda of the optima
    PabOut<C> pb_r;
    if constexpr (INTERP) {
        // final evaluations at the optima: x-dependent sums from the series (or, at large
        // lambda, directly), x-free sums and log|H^-1| from the bracket's expansions
        double xs_m[L::NX], xs_r[L::NX], sh_m[L::NS], sh_r[L::NS], ld_m = 0.0, ld_r = 0.0;
        if constexpr (GW == 16) {
            BracketCoefV<C> bm, br;
            if (need_mle) s_m = golden_coop_v<C, false>(p, gcv, best_mle.idx, f, log_iab, bm);
            if (need_reml) s_r = golden_coop_v<C, true>(p, gcv, best_reml.idx, f, log_iab, br);
            if (need_mle) {
                coop_xsums_v<C>(p, gcv, s_m, xs_m);
                coop_shared_v<C>(bm, s_m, ld_m, sh_m);
            }
            if (need_reml) {
                coop_xsums_v<C>(p, gcv, s_r, xs_r);
                coop_shared_v<C>(br, s_r, ld_r, sh_r);
            }
        } else {
            BracketCoef<C> bm, br;
            if (need_mle) s_m = golden_coop<C, false>(p, gc, best_mle.idx, f, log_iab, bm);
            if (need_reml) s_r = golden_coop<C, true>(p, gc, best_reml.idx, f, log_iab, br);
            if (need_mle) {
                coop_xsums<C>(p, gc, s_m, xs_m);
                coop_shared<C>(bm, s_m, ld_m, sh_m);
            }
            if (need_reml) {
                coop_xsums<C>(p, gc, s_r, xs_r);
                coop_shared<C>(br, s_r, ld_r, sh_r);
            }
        }
        lam_m = exp(s_m);
        lam_r = exp(s_r);
        direct_fix<C, GW>(p, j, f, valid_pair, need_score, need_mle, need_reml, s_m, s_r, xs_m,
                          xs_r);
        double row0[L::NI];
        if (need_mle) {
            assemble<C>(row0, sh_m, xs_m);
            const PabOut<C> pb = pab_reduce<C>(row0);
            logl_m = mle_logl<C>(pb, ld_m, p);
        }
        if (need_reml) {
            assemble<C>(row0, sh_r, xs_r);
            pb_r = pab_reduce<C>(row0);
            logl_r = reml_logl<C>(pb_r, log_iab, ld_r, p);
        }
    } else {
        if (need_mle) {
            PabOut<C> pb;
            golden<C, false>(p, x, y, best_mle.idx, log_iab, lam_m, logl_m, pb);
        }
        if (need_reml) golden<C, true>(p, x, y, best_reml.idx, log_iab, lam_r, logl_r, pb_r);
    }
    if (need_mle && lane == 0 && valid_pair) {
        if (p.out.lambda_mle) p.out.lambda_mle[o] = lam_m;
        if (p.out.logl_mle) p.out.logl_mle[o] = logl_m;
        const double stat = jmax(2.0 * (logl_m - p.logl0[f]), 0.0);
        if (p.out.p_lrt) p.out.p_lrt[o] = chi2_1_sf(stat);
    }
    if (need_reml) {
        bool valid;
        double beta, tau, se;
        const double px_yy = clamp_pyy(pb_r.yy1);
        beta_se<C>(pb_r, px_yy, p.df, valid, beta, tau, se);
        const double fstat = (pb_r.yy - px_yy) * tau;
        if (lane == 0 && valid_pair) {
            if (p.out.lambda_remle) p.out.lambda_remle[o] = lam_r;
            if (p.out.logl_h1) p.out.logl_h1[o] = logl_r;
            if (p.out.beta) p.out.beta[o] = beta;
            if (p.out.se) p.out.se[o] = se;
            if (p.out.p_wald) p.out.p_wald[o] = valid ? fstat : jnan();  // F, as for p_score
        }
    }
}

// ---------------------------------------------------------------- tables
// H rows: grid lambda_g = exp(loglam[g]) for g < n_grid, then the null lambda0[f];
// logdet[g] = sum_i log|lambda_g * eval_i + 1| for grid rows.
__global__ void lmm_table_kernel(int64_t n, int n_grid, int phi, const double* __restrict__ evals,
                                 const double* __restrict__ loglam, const double* __restrict__ lam0,
                                 double* __restrict__ H, double* __restrict__ logdet) {
    const int r = blockIdx.x;
    const double lam = r < n_grid ? exp(loglam[r]) : lam0[r - n_grid];
    double ld = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = __dadd_rn(__dmul_rn(lam, evals[i]), 1.0);
        H[(int64_t)r * n + i] = 1.0 / v;
        ld += log(fabs(v));
    }
    if (r >= n_grid) return;
    __shared__ double red[32];
    ld = warp_sum(ld);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ld;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
        logdet[r] = s;
    }
}

// x-free weighted sums S[row][f][s] = sum_i h_row,i * v_a,i * v_b,i over pairs without X,
// rows: grid (H), ones, null rows (H0_f).
template <int C>
__global__ void lmm_shared_kernel(int64_t n, int n_grid, int phi, const double* __restrict__ W,
                                  int64_t ldw, const double* __restrict__ Y, int64_t ldy,
                                  const double* __restrict__ H, double* __restrict__ S) {
    using L = Lay<C>;
    const int r = blockIdx.x;
    const int f = blockIdx.y;
    const double* h = r < n_grid ? H + (int64_t)r * n
                                 : (r == n_grid ? nullptr : H + (int64_t)(r - 1) * n);
    double acc[L::NS];
#pragma unroll
    for (int s = 0; s < L::NS; ++s) acc[s] = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double hi = h ? h[i] : 1.0;
        double vec[L::R];
#pragma unroll
        for (int a = 0; a < C; ++a) vec[a] = W[a * ldw + i];
        vec[C] = 0.0;
        vec[C + 1] = Y[(int64_t)f * ldy + i];
        int s = 0;
#pragma unroll
        for (int a = 0; a < L::R; ++a) {
#pragma unroll
            for (int b = a; b < L::R; ++b) {
                if (a == C || b == C) continue;
                acc[s] = fma(hi * vec[a], vec[b], acc[s]);
                ++s;
            }
        }
    }
    __shared__ double red[L::NS][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < L::NS; ++s) {
        const double v = warp_sum(acc[s]);
        if (lane == 0) red[s][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < L::NS) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[threadIdx.x][k];
        S[((int64_t)r * phi + f) * L::NS + threadIdx.x] = t;
    }
}

// GEMM operands for the per-chunk weighted x-sums: for every table row r (grid rows, the
// ones row, the null rows) A_sq[r] = h_r and A_lin[r*(C+phi) + a] = h_r * w_a (a < C),
// A_lin[r*(C+phi) + C + f] = h_r * y_f; each row has n entries.
template <int C>
__global__ void lmm_gemm_tables_kernel(int64_t n, int n_grid, int phi, const double* __restrict__ W,
                                       int64_t ldw, const double* __restrict__ Y, int64_t ldy,
                                       const double* __restrict__ H, double* __restrict__ Alin,
                                       double* __restrict__ Asq) {
    const int r = blockIdx.x;
    const double* h = r < n_grid ? H + (int64_t)r * n
                                 : (r == n_grid ? nullptr : H + (int64_t)(r - 1) * n);
    const int64_t base = (int64_t)r * (C + phi);
    for (int64_t i = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.y * blockDim.x) {
        const double hv = h ? h[i] : 1.0;
        Asq[(int64_t)r * n + i] = hv;
#pragma unroll
        for (int a = 0; a < C; ++a) Alin[(base + a) * n + i] = hv * W[a * ldw + i];
        for (int f = 0; f < phi; ++f) Alin[(base + C + f) * n + i] = hv * Y[(int64_t)f * ldy + i];
    }
}

// ---------------------------------------------------------------- squared x-sums
// CQ[j*ldcq + r] = sum_i A[i, r] x_ij^2 (r < rows) for every SNP j of a rotated chunk X
// (column-major, ld ldx): the squared weighted sums of every table row.  One fused kernel
// reads each rotated genotype once, squares it in shared memory and forms the product with
// the row table on the FP64 tensor cores (mma.sync m8n8k4 .f64), so X^2 never goes to HBM.
//   * A is held transposed, AT[i*ldt + r] (ldt a multiple of the row tile, zero for
//     r >= rows), so a slice of kSqTK samples is one contiguous block per row tile;
//   * a CTA owns TR rows x kSqTN SNPs for one range of samples; warp w owns SNPs
//     16w..16w+15 (two 8-column MMA tiles) for all TR/8 row tiles of the CTA;
//   * shared layouts As[k][TR] (TR = 8 mod 16 doubles) and Xs[j][kSqXLD] (kSqXLD = 4 mod
//     16) make every 32-lane fragment load two conflict-free wavefronts;
//   * slices are double-buffered with cp.async; out-of-range samples and SNPs read as zero;
//   * the samples are split over kz = blockIdx.z ranges when the SNP tiles alone cannot
//     fill the GPU; partial sums go to P[(kz*m + j)*ldt + r] and sq_reduce_kernel adds
//     them in kz order, so every sum has a fixed order (bit-reproducible).
constexpr int kSqTK = 16;   // samples per slice
constexpr int kSqTN = 64;   // SNPs per CTA (4 warps x 16)
constexpr int kSqXLD = 20;  // padded sample stride of a slice's SNP
constexpr int kSqThreads = 128;
constexpr int kSqSlots = 148 * 3;  // CTAs resident at once on a B200 (3 per SM)

template <int TR>
struct SqCfg {
    static_assert(TR % 16 == 8, "row tile must be 8 mod 16 doubles (conflict-free fragments)");
    static constexpr int RT = TR / 8;              // 8-row MMA tiles
    static constexpr int A_ELEMS = kSqTK * TR;
    static constexpr int X_ELEMS = kSqTN * kSqXLD;
    static constexpr int STAGE = A_ELEMS + X_ELEMS;  // doubles (even: stages stay 16-byte aligned)
    static constexpr int SMEM = 2 * STAGE * 8;
};

// Row tile for a table of `rows` rows and the matching padded leading dimension of AT.
inline int sq_tile_rows(int64_t rows) { return rows <= 56 ? 56 : 104; }
inline int64_t sq_ldt(int64_t rows) {
    const int tr = sq_tile_rows(rows);
    return ceil_div(rows, tr) * tr;
}
// Sample-range split: at least four waves of CTAs, and among the splits up to twice that
// the one whose last wave is fullest (every CTA does the same work, so a part-filled last
// wave is idle hardware); each range at least four slices long.
inline int sq_split(int64_t n, int64_t m, int64_t rows) {
    const int64_t tiles = ceil_div(m, kSqTN) * (sq_ldt(rows) / sq_tile_rows(rows));
    const int64_t kmax = ceil_div(n, 4 * kSqTK);
    int64_t k0 = ceil_div(4 * kSqSlots, tiles);
    if (k0 > kmax) k0 = kmax;
    if (k0 < 1) k0 = 1;
    int64_t best = k0;
    double best_eff = 0.0;
    for (int64_t ks = k0; ks <= 2 * k0 && ks <= kmax; ++ks) {
        const int64_t units = tiles * ks;
        const double eff = (double)units / (double)(ceil_div(units, kSqSlots) * kSqSlots);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = ks;
        }
    }
    return (int)best;
}

__device__ __forceinline__ void cp_async16(double* dst, const double* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src),
                 "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// D (8 x 8) += A (8 x 4) B (4 x 8) in FP64; lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <int TR>
__global__ void __launch_bounds__(kSqThreads, 3)
    sq_sums_kernel(const double* __restrict__ AT, int64_t ldt, const double* __restrict__ X,
                   int64_t ldx, int64_t n, int64_t m, int64_t klen, int rows,
                   double* __restrict__ out, int64_t ldo, int64_t zstride) {
    using Cfg = SqCfg<TR>;
    extern __shared__ __align__(16) double sq_smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t j0 = (int64_t)blockIdx.x * kSqTN;
    const int64_t r0 = (int64_t)blockIdx.y * TR;
    const int64_t kbeg = (int64_t)blockIdx.z * klen;
    const int64_t kend = kbeg + klen < n ? kbeg + klen : n;
    const int nsl = kend > kbeg ? (int)((kend - kbeg + kSqTK - 1) / kSqTK) : 0;

    auto issue = [&](int st, int64_t k) {
        double* As = sq_smem + st * Cfg::STAGE;
        double* Xs = As + Cfg::A_ELEMS;
        for (int e = tid; e < kSqTK * (TR / 2); e += kSqThreads) {  // A: 16-byte chunks
            const int kk = e / (TR / 2), c = e % (TR / 2);
            const bool ok = k + kk < kend;
            cp_async16(As + kk * TR + 2 * c, AT + (ok ? (k + kk) * ldt : 0) + r0 + 2 * c, ok);
        }
        for (int e = tid; e < kSqTN * kSqTK; e += kSqThreads) {  // X: one double per copy
            const int jj = e / kSqTK, kk = e % kSqTK;
            const bool ok = (k + kk < kend) && (j0 + jj < m);
            cp_async8(Xs + jj * kSqXLD + kk, X + (ok ? (j0 + jj) * ldx + k + kk : 0), ok);
        }
        cp_async_commit();
    };

    double acc[Cfg::RT][2][2];
#pragma unroll
    for (int a = 0; a < Cfg::RT; ++a)
#pragma unroll
        for (int q = 0; q < 2; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;

    const int fr = lane >> 2, fk = lane & 3;  // fragment row (or column) and k of this lane
    if (nsl > 0) issue(0, kbeg);
    for (int s = 0; s < nsl; ++s) {
        if (s + 1 < nsl) {
            issue((s + 1) & 1, kbeg + (int64_t)(s + 1) * kSqTK);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const double* As = sq_smem + (s & 1) * Cfg::STAGE;
        double* Xs = sq_smem + (s & 1) * Cfg::STAGE + Cfg::A_ELEMS;
        // square the X elements this thread copied (its own copies have landed)
        for (int e = tid; e < kSqTN * kSqTK; e += kSqThreads) {
            double* v = Xs + (e / kSqTK) * kSqXLD + e % kSqTK;
            *v = *v * *v;
        }
        __syncthreads();
        const double* xb = Xs + (warp * 16 + fr) * kSqXLD + fk;
        const double* ab = As + fk * TR + fr;
#pragma unroll
        for (int k0 = 0; k0 < kSqTK; k0 += 4) {
            const double b0 = xb[k0], b1 = xb[8 * kSqXLD + k0];
#pragma unroll
            for (int rt = 0; rt < Cfg::RT; ++rt) {
                const double a = ab[k0 * TR + rt * 8];
                dmma_8x8x4(acc[rt][0][0], acc[rt][0][1], a, b0);
                dmma_8x8x4(acc[rt][1][0], acc[rt][1][1], a, b1);
            }
        }
        __syncthreads();  // the next issue overwrites this stage
    }
    double* o = out + (int64_t)blockIdx.z * zstride;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int64_t j = j0 + warp * 16 + nt * 8 + 2 * fk + e;
            if (j >= m) continue;
#pragma unroll
            for (int rt = 0; rt < Cfg::RT; ++rt) {
                const int64_t r = r0 + rt * 8 + fr;
                if (r < rows) o[j * ldo + r] = acc[rt][nt][e];
            }
        }
    }
}

// CQ[j*ldcq + r] = sum over kz = 0..ks-1 of P[(kz*m + j)*ldt + r], in kz order.
__global__ void sq_reduce_kernel(const double* __restrict__ P, int64_t ldt, int64_t m, int rows,
                                 int ks, double* __restrict__ CQ, int64_t ldcq) {
    const int64_t total = m * rows;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / rows, r = t - j * rows;
        double v = 0.0;
        for (int z = 0; z < ks; ++z) v += P[((int64_t)z * m + j) * ldt + r];
        CQ[j * ldcq + r] = v;
    }
}

// AT[i*ldt + r] = A[r*n + i] for r < rows, 0 for rows <= r < ldt.
__global__ void sq_table_kernel(const double* __restrict__ A, int64_t n, int rows, int64_t ldt,
                                double* __restrict__ AT) {
    const int64_t total = n * ldt;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ldt, r = t - i * ldt;
        AT[t] = r < rows ? A[r * n + i] : 0.0;
    }
}

// Mixed form, global series over t = log lambda in [lo, hi]: node j of kChebG at
// t_j = mid + half * cos(pi (j + 1/2) / kChebG); hn[j * n + i] = 1 / (exp(t_j) e_i + 1).
__global__ void lmm_series_nodes_kernel(int64_t n, double mid, double half,
                                        const double* __restrict__ evals, double* __restrict__ hn) {
    const int j = blockIdx.y;
    const double lam = exp(mid + half * cos(M_PI * (j + 0.5) / kChebG));
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        hn[(int64_t)j * n + i] = __drcp_rn(__dadd_rn(__dmul_rn(lam, evals[i]), 1.0));
}

// Chebyshev transform of the node values, column-major kChebG x kChebG:
// ccos[k + j * kChebG] = (2 / kChebG) cos(pi k (j + 1/2) / kChebG), row k = 0 halved, so
// coefficient k of any per-sample weight is sum_j ccos[k, j] * value_j.
__global__ void lmm_series_dct_kernel(double* __restrict__ ccos) {
    const int j = blockIdx.x, k = threadIdx.x;
    const double c = (2.0 / kChebG) * cos(M_PI * k * (j + 0.5) / kChebG);
    ccos[k + (int64_t)j * kChebG] = k == 0 ? 0.5 * c : c;
}

// GEMM operands of the mixed form: row 0 is the ones row (h = 1), row 1 + k holds the
// Chebyshev coefficient k of h_i(t) (already in Asq rows 1..kChebG from the transform
// GEMM); A_lin[r*(C+phi) + a] = Asq[r] * w_a, A_lin[r*(C+phi) + C + f] = Asq[r] * y_f.
template <int C>
__global__ void lmm_series_tables_kernel(int64_t n, int phi, const double* __restrict__ W,
                                         int64_t ldw, const double* __restrict__ Y, int64_t ldy,
                                         double* __restrict__ Alin, double* __restrict__ Asq) {
    const int r = blockIdx.x;
    const int64_t base = (int64_t)r * (C + phi);
    for (int64_t i = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.y * blockDim.x) {
        double hv = 1.0;
        if (r == 0)
            Asq[i] = 1.0;
        else
            hv = Asq[(int64_t)r * n + i];
#pragma unroll
        for (int a = 0; a < C; ++a) Alin[(base + a) * n + i] = hv * W[a * ldw + i];
        for (int f = 0; f < phi; ++f) Alin[(base + C + f) * n + i] = hv * Y[(int64_t)f * ldy + i];
    }
}

// Chebyshev node values for the mixed form: block (bracket b, node k) x phenotype f
// evaluates log|H^-1| (f == 0) and the x-free weighted sums of phenotype f exactly in
// FP64 at lambda = exp(s_k), s_k the k-th Chebyshev node of bracket b.
template <int C>
__global__ void lmm_cheb_nodes_kernel(int64_t n, int n_grid, int phi,
                                      const double* __restrict__ evals, const double* __restrict__ W,
                                      int64_t ldw, const double* __restrict__ Y, int64_t ldy,
                                      const double* __restrict__ loglam, double* __restrict__ vals,
                                      double* __restrict__ mid, double* __restrict__ half) {
    using L = Lay<C>;
    const int b = blockIdx.x / kChebN, k = blockIdx.x % kChebN, f = blockIdx.y;
    const int lo = b - 1 > 0 ? b - 1 : 0, hi = b + 1 < n_grid - 1 ? b + 1 : n_grid - 1;
    const double A = loglam[lo], B = loglam[hi];
    const double m = 0.5 * (A + B), h = 0.5 * (B - A);
    const double s = m + h * cos(M_PI * (k + 0.5) / kChebN);
    const double lam = exp(s);
    double acc[L::NS];
#pragma unroll
    for (int q = 0; q < L::NS; ++q) acc[q] = 0.0;
    double ld = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = __dadd_rn(__dmul_rn(lam, evals[i]), 1.0);
        const double hv = __drcp_rn(v);
        if (f == 0) ld += log(fabs(v));
        double vec[L::R];
#pragma unroll
        for (int a = 0; a < C; ++a) vec[a] = W[a * ldw + i];
        vec[C] = 0.0;
        vec[C + 1] = Y[(int64_t)f * ldy + i];
        int q = 0;
#pragma unroll
        for (int a = 0; a < L::R; ++a) {
#pragma unroll
            for (int bb = a; bb < L::R; ++bb) {
                if (a == C || bb == C) continue;
                acc[q] = fma(hv * vec[a], vec[bb], acc[q]);
                ++q;
            }
        }
    }
    __shared__ double red[L::NS + 1][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < L::NS; ++q) {
        const double v = warp_sum(acc[q]);
        if (lane == 0) red[q][w] = v;
    }
    {
        const double v = warp_sum(ld);
        if (lane == 0) red[L::NS][w] = v;
    }
    __syncthreads();
    const int nf = 1 + phi * L::NS;
    double* out = vals + ((int64_t)b * kChebN + k) * nf;
    if (threadIdx.x <= L::NS) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[threadIdx.x][q];
        if (threadIdx.x < L::NS)
            out[1 + f * L::NS + threadIdx.x] = t;
        else if (f == 0)
            out[0] = t;
    }
    if (threadIdx.x == 0 && k == 0 && f == 0) {
        mid[b] = m;
        half[b] = h;
    }
}

// Chebyshev coefficients c_j = (2/N) sum_k f(s_k) cos(pi j (k + 1/2) / N), c_0 halved.
__global__ void lmm_cheb_coef_kernel(int nf, const double* __restrict__ vals,
                                     double* __restrict__ coef) {
    const int b = blockIdx.x, fi = blockIdx.y, j = threadIdx.x;
    if (j >= kChebN) return;
    double c = 0.0;
    for (int k = 0; k < kChebN; ++k)
        c += vals[((int64_t)b * kChebN + k) * nf + fi] * cos(M_PI * j * (k + 0.5) / kChebN);
    c *= 2.0 / kChebN;
    if (j == 0) c *= 0.5;
    coef[((int64_t)b * nf + fi) * kChebN + j] = c;
}

// ---------------------------------------------------------------- null model
// One CTA per phenotype runs _golden_section_minimize (likelihood.py:395-474) over
// -mle_log_likelihood_null (349-392): all threads evaluate, thread-uniform control.
template <int C>
__device__ double null_mle_eval(int64_t n, const double* W, int64_t ldw, const double* y,
                                const double* evals, double lam, double c_mle, double* red) {
    using L = Lay<C>;
    double acc[L::NS];
#pragma unroll
    for (int s = 0; s < L::NS; ++s) acc[s] = 0.0;
    double ld = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = __dadd_rn(__dmul_rn(lam, evals[i]), 1.0);
        const double hi = 1.0 / v;
        ld += log(fabs(v));
        double vec[L::R];
#pragma unroll
        for (int a = 0; a < C; ++a) vec[a] = W[a * ldw + i];
        vec[C] = 0.0;
        vec[C + 1] = y[i];
        int s = 0;
#pragma unroll
        for (int a = 0; a < L::R; ++a) {
#pragma unroll
            for (int b = a; b < L::R; ++b) {
                if (a == C || b == C) continue;
                acc[s] = fma(hi * vec[a], vec[b], acc[s]);
                ++s;
            }
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
#pragma unroll
    for (int s = 0; s < L::NS; ++s) {
        const double v = warp_sum(acc[s]);
        if (lane == 0) red[s * 32 + w] = v;
    }
    {
        const double v = warp_sum(ld);
        if (lane == 0) red[L::NS * 32 + w] = v;
    }
    __syncthreads();
    double tot[L::NS + 1];
#pragma unroll
    for (int s = 0; s <= L::NS; ++s) {
        double t = 0.0;
        for (int k = 0; k < nw; ++k) t += red[s * 32 + k];
        tot[s] = t;
    }
    double row0[L::NI];
    double xs[L::NX];
#pragma unroll
    for (int k = 0; k < L::NX; ++k) xs[k] = 0.0;
    assemble<C>(row0, tot, xs);
    const PabOut<C> pb = pab_reduce<C>(row0);
    const double pyy = clamp_pyy(pb.yy);  // level n_cvt for the null model
    const double f = __dsub_rn(c_mle, __dmul_rn(0.5, tot[L::NS]));
    return __dsub_rn(f, __dmul_rn(__dmul_rn(0.5, (double)n), log(pyy)));
}

template <int C>
__global__ void null_mle_kernel(int64_t n, const double* W, int64_t ldw, const double* Y,
                                int64_t ldy, const double* evals, double lo, double step,
                                int n_grid, int n_iter, double log_hi, double c_mle, double* lam0,
                                double* logl0) {
    __shared__ double red[(Lay<C>::NS + 1) * 32];
    const int f = blockIdx.x;
    const double* y = Y + (int64_t)f * ldy;
    auto func = [&](double lam) {
        return -null_mle_eval<C>(n, W, ldw, y, evals, lam, c_mle, red);
    };
    int best_i = 0;
    double best_v = func(exp(lo));
    for (int i = 1; i < n_grid; ++i) {
        const double v = func(exp(__dadd_rn(lo, __dmul_rn((double)i, step))));
        if (v < best_v) {
            best_v = v;
            best_i = i;
        }
    }
    const int il = best_i - 1 > 0 ? best_i - 1 : 0;
    const int ih = best_i + 1 < n_grid - 1 ? best_i + 1 : n_grid - 1;
    double a = __dadd_rn(lo, __dmul_rn((double)il, step));
    double b = __dadd_rn(lo, __dmul_rn((double)ih, step));
    double c = __dsub_rn(b, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double d = __dadd_rn(a, __dmul_rn(kPhi, __dsub_rn(b, a)));
    double fc = func(exp(c)), fd = func(exp(d));
    for (int it = 0; it < n_iter; ++it) {
        if (fc < fd) {
            b = d;
            d = c;
            fd = fc;
            c = __dsub_rn(b, __dmul_rn(kPhi, __dsub_rn(b, a)));
            fc = func(exp(c));
        } else {
            a = c;
            c = d;
            fc = fd;
            d = __dadd_rn(a, __dmul_rn(kPhi, __dsub_rn(b, a)));
            fd = func(exp(d));
        }
    }
    const double opt = exp(__dmul_rn(__dadd_rn(a, b), 0.5));
    const double v = func(opt);
    if (threadIdx.x == 0) {
        lam0[f] = opt;
        logl0[f] = -v;
    }
}

// ---------------------------------------------------------------- host helpers
struct WsLayout {
    int64_t loglam, logdet, H, S, cheb, cmid, chalf, cvals, alin, asq, asqt, hn, ccos, blas, total;
};

inline int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }

inline int ns_of(int c) { return (c + 2) * (c + 1) / 2; }

// Table rows of the chunk GEMMs: grid rows + ones row + null rows (FP64 form) or the ones
// row + kChebG series coefficients (mixed form); sized for whichever is larger.
inline int64_t table_rows(int phi, int n_grid) {
    const int64_t direct = (int64_t)n_grid + 1 + phi, series = 1 + kChebG;
    return direct > series ? direct : series;
}

inline WsLayout ws_layout(int64_t n, int c, int phi, int n_grid) {
    WsLayout w;
    int64_t off = 0;
    w.loglam = off;
    off += align256(8 * (int64_t)n_grid);
    w.logdet = off;
    off += align256(8 * (int64_t)n_grid);
    w.H = off;
    off += align256(8 * (int64_t)(n_grid + phi) * n);
    w.S = off;
    off += align256(8 * (int64_t)(n_grid + 1 + phi) * phi * ns_of(c));
    const int64_t nf = 1 + (int64_t)phi * ns_of(c);
    w.cheb = off;
    off += align256(8 * (int64_t)n_grid * nf * kChebN);
    w.cmid = off;
    off += align256(8 * (int64_t)n_grid);
    w.chalf = off;
    off += align256(8 * (int64_t)n_grid);
    w.cvals = off;
    off += align256(8 * (int64_t)n_grid * nf * kChebN);
    const int64_t rows = table_rows(phi, n_grid);
    w.alin = off;
    off += align256(8 * rows * (c + phi) * n);
    w.asq = off;
    off += align256(8 * rows * n);
    {  // the squared-sum table transposed for sq_sums_kernel, for either form's row count
        const int64_t r1 = (int64_t)n_grid + 1 + phi, r2 = 1 + kChebG;
        const int64_t ldt = sq_ldt(r1) > sq_ldt(r2) ? sq_ldt(r1) : sq_ldt(r2);
        w.asqt = off;
        off += align256(8 * ldt * n);
    }
    w.hn = off;
    off += align256(8 * (int64_t)kChebG * n);
    w.ccos = off;
    off += align256(8 * (int64_t)kChebG * kChebG);
    w.blas = off;
    off += kCublasWorkspaceBytes;
    w.total = off;
    return w;
}

struct ChunkLayout {
    int64_t sqp, cl, cq, blas, total;
};

// Partial squared sums of sq_sums_kernel's sample ranges: the largest over the row counts a
// chunk can use (FP64 form with and without null rows, mixed form).
inline int64_t sq_partial_doubles(int64_t n, int64_t m, int phi, int n_grid) {
    const int64_t cand[3] = {(int64_t)n_grid + 1 + phi, (int64_t)n_grid + 1, 1 + (int64_t)kChebG};
    int64_t best = 0;
    for (int64_t r : cand) {
        const int ks = sq_split(n, m, r);
        const int64_t v = ks > 1 ? (int64_t)ks * m * sq_ldt(r) : 0;
        if (v > best) best = v;
    }
    return best;
}

inline ChunkLayout chunk_layout(int64_t n, int c, int phi, int n_grid, int64_t m) {
    ChunkLayout L;
    const int64_t rows = table_rows(phi, n_grid);
    int64_t off = 0;
    L.sqp = off;
    off += align256(8 * sq_partial_doubles(n, m, phi, n_grid));
    L.cl = off;
    off += align256(8 * rows * (c + phi) * m);
    L.cq = off;
    off += align256(8 * rows * m);
    L.blas = off;  // cuBLAS workspace of this chunk's DGEMMs (fixed size: same kernels alone or
    off += kCublasWorkspaceBytes;  // beside other streams' work, so results do not depend on it)
    L.total = off;
    return L;
}

// Mixed form, genotype-side linear x-sums: the chunk GEMM  CL = A_lin x~  with x~ = U^T g
// equals  (U A_lin^T)^T g, so the basis  V = U A_lin^T  (n x rows_lin, column q = basis of
// CL row q) is formed once per cohort and split into INT8 digit planes; every chunk then
// gets CL from the decoded calls on the INT8 rotation core (V has rows_lin ~ 1 % of U's n
// columns), instead of an FP64 DGEMM over the rotated chunk.
struct SeriesLayout {
    int64_t rows_lin, basis, ozaki, total;
};

inline SeriesLayout series_layout(int64_t n, int c, int phi) {
    SeriesLayout L;
    L.rows_lin = (int64_t)(1 + kChebG) * (c + phi);
    int64_t off = 0;
    L.basis = off;
    off += align256(8 * n * L.rows_lin);
    L.ozaki = off;
    off += align256(tc::ozaki_layout(L.rows_lin, n).total);
    L.total = off;
    return L;
}

// numpy.linspace(start, stop, num): start + i*step, last element = stop.
__global__ void linspace_kernel(double* out, double start, double stop, int num) {
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= num) return;
    if (num == 1) {
        out[0] = start;
        return;
    }
    const double step = (stop - start) / (double)(num - 1);
    out[i] = (i == num - 1) ? stop : __dadd_rn(__dmul_rn((double)i, step), start);
}

// F statistics (NaN where there is no test) -> F-test p-values, in place, one thread per
// value, for up to two arrays of `count` values (Wald and score) in one launch.  The
// continued fraction of betainc_reg takes up to ~100 steps for F above ~3 at df ~ 2e4;
// inside the search kernel every lane of a pair's group would repeat it, and a warp would
// wait for the slower of its pairs.
__global__ void lmm_fpvalue_kernel(double* __restrict__ v0, double* __restrict__ v1,
                                   int64_t count, double df) {
    const int64_t total = v1 ? 2 * count : count;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        double* v = i < count ? v0 + i : v1 + (i - count);
        *v = f_pvalue(*v, df, true);
    }
}

// Squared x-sums of a rotated chunk: sq_sums_kernel (+ sq_reduce_kernel when the samples
// are split into ranges).  AT: the transposed table (ld sq_ldt(rows)); P: partial sums
// (sq_partial_doubles); CQ: rows x m, ld ldcq.
int32_t launch_sq_sums(const double* AT, int64_t rows, const double* X, int64_t ldx, int64_t n,
                       int64_t m, double* P, double* CQ, int64_t ldcq, cudaStream_t st) {
    const int tr = sq_tile_rows(rows);
    const int64_t ldt = sq_ldt(rows);
    const int ks = sq_split(n, m, rows);
    const int64_t klen = ceil_div(ceil_div(n, ks), kSqTK) * kSqTK;
    const int64_t gx = ceil_div(m, kSqTN);
    if (gx > 0x7fffffffll || ldt / tr > 65535) {
        set_error("squared x-sums: chunk too large");
        return JB_E_INVALID;
    }
    dim3 grid((unsigned)gx, (unsigned)(ldt / tr), (unsigned)ks);
    double* out = ks > 1 ? P : CQ;
    const int64_t ldo = ks > 1 ? ldt : ldcq;
    if (tr == 56) {
        JB_CUDA(cudaFuncSetAttribute(sq_sums_kernel<56>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     SqCfg<56>::SMEM));
        sq_sums_kernel<56><<<grid, kSqThreads, SqCfg<56>::SMEM, st>>>(
            AT, ldt, X, ldx, n, m, klen, (int)rows, out, ldo, m * ldt);
    } else {
        JB_CUDA(cudaFuncSetAttribute(sq_sums_kernel<104>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     SqCfg<104>::SMEM));
        sq_sums_kernel<104><<<grid, kSqThreads, SqCfg<104>::SMEM, st>>>(
            AT, ldt, X, ldx, n, m, klen, (int)rows, out, ldo, m * ldt);
    }
    JB_LAUNCH_CHECK("sq_sums_kernel");
    if (ks > 1) {
        const int64_t blocks = ceil_div(m * rows, 256) < 4096 ? ceil_div(m * rows, 256) : 4096;
        sq_reduce_kernel<<<(unsigned)blocks, 256, 0, st>>>(P, ldt, m, (int)rows, ks, CQ, ldcq);
        JB_LAUNCH_CHECK("sq_reduce_kernel");
    }
    return JB_OK;
}

template <int C>
int32_t launch_pairs(const Params& p, cudaStream_t st) {
    const int64_t pairs = p.m * p.phi;
    if constexpr (C == 1) {
        if (p.cheb)  // two pairs per warp (bit-identical to one per warp)
            lmm_pairs_kernel<C, true, 16>
                <<<(unsigned)ceil_div(pairs * 16, kPairsThreads), kPairsThreads, 0, st>>>(p);
        else
            lmm_pairs_kernel<C, false, 32>
                <<<(unsigned)ceil_div(pairs * 32, kPairsThreads), kPairsThreads, 0, st>>>(p);
    } else if (p.cheb)
        lmm_pairs_kernel<C, true, 32><<<(unsigned)ceil_div(pairs * 32, kPairsThreads), kPairsThreads, 0, st>>>(p);
    else
        lmm_pairs_kernel<C, false, 32><<<(unsigned)ceil_div(pairs * 32, kPairsThreads), kPairsThreads, 0, st>>>(p);
    JB_LAUNCH_CHECK("lmm_pairs_kernel");
    // p-values of the tests this mode ran (other outputs stay untouched)
    double* v0 = (p.mode == 1 || p.mode == 4) ? p.out.p_wald : nullptr;
    double* v1 = (p.mode == 3 || p.mode == 4) ? p.out.p_score : nullptr;
    if (!v0) {
        v0 = v1;
        v1 = nullptr;
    }
    if (v0) {
        const int64_t total = v1 ? 2 * pairs : pairs;
        const int64_t blocks = ceil_div(total, 128) < 8192 ? ceil_div(total, 128) : 8192;
        lmm_fpvalue_kernel<<<(unsigned)blocks, 128, 0, st>>>(v0, v1, pairs, p.df);
        JB_LAUNCH_CHECK("lmm_fpvalue_kernel");
    }
    return JB_OK;
}

template <int C>
int32_t launch_prepare(int64_t n, int phi, int n_grid, const double* evals, const double* W,
                       int64_t ldw, const double* Y, int64_t ldy, const double* lam0,
                       double l_min, double l_max, uint8_t* ws, cudaStream_t st, bool interp) {
    const WsLayout L = ws_layout(n, C, phi, n_grid);
    double* loglam = reinterpret_cast<double*>(ws + L.loglam);
    double* logdet = reinterpret_cast<double*>(ws + L.logdet);
    double* H = reinterpret_cast<double*>(ws + L.H);
    double* S = reinterpret_cast<double*>(ws + L.S);
    linspace_kernel<<<(n_grid + 127) / 128, 128, 0, st>>>(loglam, std::log(l_min), std::log(l_max),
                                                        n_grid);
    JB_LAUNCH_CHECK("linspace_kernel");
    const int rows_h = n_grid + (lam0 ? phi : 0);
    lmm_table_kernel<<<rows_h, 256, 0, st>>>(n, n_grid, phi, evals, loglam, lam0, H, logdet);
    JB_LAUNCH_CHECK("lmm_table_kernel");
    const int rows_s = n_grid + 1 + (lam0 ? phi : 0);
    lmm_shared_kernel<C><<<dim3(rows_s, phi), 256, 0, st>>>(n, n_grid, phi, W, ldw, Y, ldy, H, S);
    JB_LAUNCH_CHECK("lmm_shared_kernel");
    const unsigned ny = (unsigned)(ceil_div(n, 256) < 64 ? ceil_div(n, 256) : 64);
    double* Alin = reinterpret_cast<double*>(ws + L.alin);
    double* Asq = reinterpret_cast<double*>(ws + L.asq);
    if (!interp) {
        lmm_gemm_tables_kernel<C><<<dim3(rows_s, ny), 256, 0, st>>>(n, n_grid, phi, W, ldw, Y, ldy,
                                                                   H, Alin, Asq);
        JB_LAUNCH_CHECK("lmm_gemm_tables_kernel");
    } else {
        // global series tables: node values -> coefficients (one DGEMM) -> A_lin / A_sq
        const double lo = std::log(kDomainLo), hi = std::log(kDomainHi);
        double* hn = reinterpret_cast<double*>(ws + L.hn);
        double* ccos = reinterpret_cast<double*>(ws + L.ccos);
        lmm_series_nodes_kernel<<<dim3(ny, kChebG), 256, 0, st>>>(n, 0.5 * (lo + hi), 0.5 * (hi - lo),
                                                                   evals, hn);
        JB_LAUNCH_CHECK("lmm_series_nodes_kernel");
        lmm_series_dct_kernel<<<kChebG, kChebG, 0, st>>>(ccos);
        JB_LAUNCH_CHECK("lmm_series_dct_kernel");
        cublasHandle_t h = cublas_handle();
        if (!h) {
            set_error("cuBLAS handle creation failed");
            return JB_E_LIBRARY;
        }
        cublasStatus_t cs = bind_cublas(h, st, ws + L.blas, kCublasWorkspaceBytes);
        if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasSetStream/Workspace");
        const double one = 1.0, zero = 0.0;
        // (n x K, column-major, ld n) = hn (n x K) * ccos^T: coefficient rows 1..K of Asq
        cs = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, kChebG, kChebG, &one, hn, (int)n,
                         ccos, kChebG, &zero, Asq + n, (int)n);
        if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasDgemm (series transform)");
        lmm_series_tables_kernel<C><<<dim3(1 + kChebG, ny), 256, 0, st>>>(n, phi, W, ldw, Y, ldy,
                                                                         Alin, Asq);
        JB_LAUNCH_CHECK("lmm_series_tables_kernel");
    }
    {  // the squared-sum rows transposed for sq_sums_kernel
        const int64_t rows_sq = interp ? 1 + kChebG : (int64_t)rows_s;
        const int64_t ldt = sq_ldt(rows_sq);
        const int64_t blocks = ceil_div(n * ldt, 256) < 8192 ? ceil_div(n * ldt, 256) : 8192;
        sq_table_kernel<<<(unsigned)blocks, 256, 0, st>>>(Asq, n, (int)rows_sq, ldt,
                                                          reinterpret_cast<double*>(ws + L.asqt));
        JB_LAUNCH_CHECK("sq_table_kernel");
    }
    if (interp) {
        const int nf = 1 + phi * Lay<C>::NS;
        double* vals = reinterpret_cast<double*>(ws + L.cvals);
        double* coef = reinterpret_cast<double*>(ws + L.cheb);
        lmm_cheb_nodes_kernel<C><<<dim3(n_grid * kChebN, phi), 256, 0, st>>>(
            n, n_grid, phi, evals, W, ldw, Y, ldy, loglam, vals,
            reinterpret_cast<double*>(ws + L.cmid), reinterpret_cast<double*>(ws + L.chalf));
        JB_LAUNCH_CHECK("lmm_cheb_nodes_kernel");
        lmm_cheb_coef_kernel<<<dim3(n_grid, nf), 32, 0, st>>>(nf, vals, coef);
        JB_LAUNCH_CHECK("lmm_cheb_coef_kernel");
    }
    return JB_OK;
}

}  // namespace lmm
}  // namespace jb

using namespace jb;
using namespace jb::lmm;

extern "C" {

int64_t jb_lmm_workspace_size(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid) {
    if (n <= 0 || n_cvt < 1 || phi < 1 || n_grid < 1) return -1;
    return ws_layout(n, n_cvt, phi, n_grid).total;
}

int32_t jb_lmm_prepare(int32_t lmm_mode, int32_t precision, int64_t n, int32_t n_cvt,
                       int32_t phi, const double* evals, const double* UtW, int64_t ldw,
                       const double* Uty, int64_t ldy, const double* lam0, double l_min,
                       double l_max, int32_t n_grid, void* workspace, int64_t workspace_bytes,
                       uintptr_t stream) {
    JB_CHECK_ARG(precision == 0 || precision == 1, "jb_lmm_prepare: precision must be 0 or 1");
    JB_CHECK_ARG(lmm_mode >= 1 && lmm_mode <= 4, "jb_lmm_prepare: lmm_mode must be 1..4");
    JB_CHECK_ARG(n > 0 && phi >= 1 && n_grid >= 2, "jb_lmm_prepare: bad sizes");
    JB_CHECK_ARG(n_cvt >= 1 && n_cvt <= kMaxCvt, "jb_lmm_prepare: n_cvt must be in 1..%d", kMaxCvt);
    JB_CHECK_ARG(n > n_cvt + 1, "jb_lmm_prepare: n must exceed n_cvt + 1");
    JB_CHECK_ARG(ldw >= n && ldy >= n, "jb_lmm_prepare: bad leading dimension");
    JB_CHECK_ARG(l_min > 0 && l_max > l_min, "jb_lmm_prepare: need 0 < l_min < l_max");
    JB_CHECK_ARG(lmm_mode == 1 || lam0, "jb_lmm_prepare: modes 2-4 need lam0");
    JB_CHECK_ARG(workspace_bytes >= jb_lmm_workspace_size(n, n_cvt, phi, n_grid),
                 "jb_lmm_prepare: workspace too small");
    JB_CHECK_ARG(phi <= 65535, "jb_lmm_prepare: too many phenotypes");
    JB_CHECK_ARG(precision == 0 || (l_min >= kDomainLo * (1 - 1e-12) && l_max <= kDomainHi * (1 + 1e-12)),
                 "jb_lmm_prepare: the mixed form needs 1e-5 <= l_min < l_max <= 1e5");
    cudaStream_t st = as_stream(stream);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    const double* l0 = lmm_mode == 1 ? nullptr : lam0;
    switch (n_cvt) {
        case 1: return launch_prepare<1>(n, phi, n_grid, evals, UtW, ldw, Uty, ldy, l0, l_min, l_max, ws, st, precision == 1);
        case 2: return launch_prepare<2>(n, phi, n_grid, evals, UtW, ldw, Uty, ldy, l0, l_min, l_max, ws, st, precision == 1);
        case 3: return launch_prepare<3>(n, phi, n_grid, evals, UtW, ldw, Uty, ldy, l0, l_min, l_max, ws, st, precision == 1);
        case 4: return launch_prepare<4>(n, phi, n_grid, evals, UtW, ldw, Uty, ldy, l0, l_min, l_max, ws, st, precision == 1);
    }
    return JB_E_UNSUPPORTED;
}

int64_t jb_lmm_chunk_workspace_size(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid,
                                    int64_t m) {
    if (n <= 0 || n_cvt < 1 || phi < 1 || n_grid < 1 || m < 0) return -1;
    return chunk_layout(n, n_cvt, phi, n_grid, m > 0 ? m : 1).total;
}

int32_t jb_lmm_series_rows(void) { return 1 + kChebG; }

int64_t jb_lmm_series_workspace_size(int64_t n, int32_t n_cvt, int32_t phi) {
    if (n <= 0 || n_cvt < 1 || n_cvt > kMaxCvt || phi < 1) return -1;
    return series_layout(n, n_cvt, phi).total;
}

int32_t jb_lmm_series_prepare(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid,
                              const void* workspace, int64_t workspace_bytes, const double* U,
                              int64_t ldu, void* series_ws, int64_t series_bytes,
                              uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && n_cvt >= 1 && n_cvt <= kMaxCvt && phi >= 1 && n_grid >= 2,
                 "jb_lmm_series_prepare: bad sizes");
    JB_CHECK_ARG(U && ldu >= n, "jb_lmm_series_prepare: bad eigenvector matrix");
    JB_CHECK_ARG(workspace && workspace_bytes >= jb_lmm_workspace_size(n, n_cvt, phi, n_grid),
                 "jb_lmm_series_prepare: workspace too small");
    const SeriesLayout SL = series_layout(n, n_cvt, phi);
    JB_CHECK_ARG(series_ws && series_bytes >= SL.total, "jb_lmm_series_prepare: series workspace too small");
    JB_CHECK_ARG(SL.rows_lin <= 65535, "jb_lmm_series_prepare: too many phenotypes");
    const WsLayout L = ws_layout(n, n_cvt, phi, n_grid);
    uint8_t* ws = const_cast<uint8_t*>(static_cast<const uint8_t*>(workspace));
    uint8_t* sws = static_cast<uint8_t*>(series_ws);
    cudaStream_t st = as_stream(stream);
    cublasHandle_t h = cublas_handle();
    if (!h) {
        set_error("cuBLAS handle creation failed");
        return JB_E_LIBRARY;
    }
    cublasStatus_t cs = bind_cublas(h, st, ws + L.blas, kCublasWorkspaceBytes);
    if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasSetStream/Workspace");
    const double one = 1.0, zero = 0.0;
    double* V = reinterpret_cast<double*>(sws + SL.basis);
    // V (n x rows_lin) = U (n x n) * A_lin^T, A_lin stored as rows of n (column-major n x rows_lin)
    cs = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)SL.rows_lin, (int)n, &one, U, (int)ldu,
                     reinterpret_cast<const double*>(ws + L.alin), (int)n, &zero, V, (int)n);
    if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasDgemm (series basis)");
    return tc::ozaki_split(V, n, SL.rows_lin, n, sws + SL.ozaki, st);
}

int32_t jb_lmm_chunk_series_i8(int64_t n, int32_t n_cvt, int32_t phi, int32_t n_grid, int64_t m,
                               const void* series_ws, int64_t series_bytes, const int8_t* codes,
                               int64_t ld_codes, const double* mean, int32_t has_missing,
                               void* rot_ws, int64_t rot_bytes, void* chunk_workspace,
                               int64_t chunk_bytes, uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && n_cvt >= 1 && n_cvt <= kMaxCvt && phi >= 1 && n_grid >= 2 && m >= 0,
                 "jb_lmm_chunk_series_i8: bad sizes");
    if (m == 0) return JB_OK;
    const SeriesLayout SL = series_layout(n, n_cvt, phi);
    JB_CHECK_ARG(series_ws && series_bytes >= SL.total, "jb_lmm_chunk_series_i8: series workspace too small");
    const tc::RotChunkLayout RL = tc::rot_chunk_layout(n, m);
    JB_CHECK_ARG(rot_ws && rot_bytes >= RL.total, "jb_lmm_chunk_series_i8: rotation workspace too small");
    JB_CHECK_ARG(ceil_div(SL.rows_lin, 32) <= ceil_div(n, 32),
                 "jb_lmm_chunk_series_i8: more series rows than samples");
    JB_CHECK_ARG(codes && ld_codes >= n && (!has_missing || mean), "jb_lmm_chunk_series_i8: bad genotype input");
    const ChunkLayout CLy = chunk_layout(n, n_cvt, phi, n_grid, m);
    JB_CHECK_ARG(chunk_workspace && chunk_bytes >= CLy.total, "jb_lmm_chunk_series_i8: chunk workspace too small");
    uint8_t* rws = static_cast<uint8_t*>(rot_ws);
    double* CL = reinterpret_cast<double*>(static_cast<uint8_t*>(chunk_workspace) + CLy.cl);
    const uint8_t* ows = static_cast<const uint8_t*>(series_ws) + SL.ozaki;
    tc::Tile* tiles = reinterpret_cast<tc::Tile*>(rws + RL.tiles);
    int* status = reinterpret_cast<int*>(rws + RL.status);
    cudaStream_t st = as_stream(stream);
    if (has_missing) {  // the [calls | masks] pairs packed by jb_rotate_i8 for these codes
        const int64_t NB = ceil_div(m, 128);
        return tc::rotate_i8_gemm(ows, SL.rows_lin, n, reinterpret_cast<const int8_t*>(rws + RL.b_off),
                                  NB * 256, RL.ldb, true, m, mean, CL, SL.rows_lin, tiles, status, st);
    }
    return tc::rotate_i8_gemm(ows, SL.rows_lin, n, codes, m, ld_codes, false, m, nullptr, CL,
                              SL.rows_lin, tiles, status, st);
}

int32_t jb_lmm_chunk(int32_t lmm_mode, int32_t precision, int64_t n, int32_t n_cvt, int32_t phi,
                     int64_t m,
                     const double* evals, const double* UtW, int64_t ldw, const double* Uty,
                     int64_t ldy, const double* UtG, int64_t ldg, const double* lam0,
                     const double* logl0, double l_min, double l_max, int32_t n_grid,
                     int32_t n_iter, jb_lmm_out out, void* workspace, int64_t workspace_bytes,
                     void* chunk_workspace, int64_t chunk_bytes, uintptr_t stream) {
    JB_CHECK_ARG(lmm_mode >= 1 && lmm_mode <= 4, "jb_lmm_chunk: lmm_mode must be 1..4");
    JB_CHECK_ARG(n > 0 && phi >= 1 && m >= 0 && n_grid >= 2 && n_iter >= 0, "jb_lmm_chunk: bad sizes");
    JB_CHECK_ARG(n_cvt >= 1 && n_cvt <= kMaxCvt, "jb_lmm_chunk: n_cvt must be in 1..%d", kMaxCvt);
    JB_CHECK_ARG(n > n_cvt + 1, "jb_lmm_chunk: n must exceed n_cvt + 1");
    JB_CHECK_ARG(ldw >= n && ldy >= n && ldg >= n, "jb_lmm_chunk: bad leading dimension");
    JB_CHECK_ARG(l_min > 0 && l_max > l_min, "jb_lmm_chunk: need 0 < l_min < l_max");
    JB_CHECK_ARG(lmm_mode != 2 && lmm_mode != 4 ? true : logl0 != nullptr,
                 "jb_lmm_chunk: modes 2 and 4 need logl0");
    JB_CHECK_ARG(workspace_bytes >= jb_lmm_workspace_size(n, n_cvt, phi, n_grid),
                 "jb_lmm_chunk: workspace too small");
    if (m == 0) return JB_OK;
    const WsLayout L = ws_layout(n, n_cvt, phi, n_grid);
    uint8_t* ws = static_cast<uint8_t*>(workspace);
    Params p;
    p.mode = lmm_mode;
    p.n = n;
    p.phi = phi;
    p.m = m;
    p.evals = evals;
    p.W = UtW;
    p.ldw = ldw;
    p.Y = Uty;
    p.ldy = ldy;
    p.G = UtG;
    p.ldg = ldg;
    p.logl0 = logl0;
    p.n_grid = n_grid;
    p.n_iter = n_iter;
    p.loglam = reinterpret_cast<const double*>(ws + L.loglam);
    p.logdet = reinterpret_cast<const double*>(ws + L.logdet);
    p.H = reinterpret_cast<const double*>(ws + L.H);
    p.S = reinterpret_cast<const double*>(ws + L.S);
    const double df = (double)(n - n_cvt - 1);
    p.df = df;
    p.n_d = (double)n;
    p.c_reml = 0.5 * df * (std::log(df) - std::log(2 * M_PI) - 1.0);
    p.c_mle = 0.5 * (double)n * (std::log((double)n) - std::log(2 * M_PI) - 1.0);
    p.out = out;
    JB_CHECK_ARG(precision >= 0 && precision <= 2, "jb_lmm_chunk: precision must be 0, 1 or 2");
    p.cheb = precision >= 1 ? reinterpret_cast<const double*>(ws + L.cheb) : nullptr;
    p.cheb_mid = reinterpret_cast<const double*>(ws + L.cmid);
    p.cheb_half = reinterpret_cast<const double*>(ws + L.chalf);
    p.lam0 = lam0;
    JB_CHECK_ARG(precision == 0 || lmm_mode == 1 || lam0 != nullptr,
                 "jb_lmm_chunk: the mixed form needs lam0 in modes 2-4");
    JB_CHECK_ARG(precision == 0 || (l_min >= kDomainLo * (1 - 1e-12) && l_max <= kDomainHi * (1 + 1e-12)),
                 "jb_lmm_chunk: the mixed form needs 1e-5 <= l_min < l_max <= 1e5");
    {
        const double lo = std::log(kDomainLo), hi = std::log(kDomainHi);
        p.gmid = 0.5 * (lo + hi);
        p.ginv = 1.0 / (0.5 * (hi - lo));
    }
    cudaStream_t st = as_stream(stream);
    // chunk GEMMs: weighted x-sums of every table row (grid, ones, null) for all SNPs
    const ChunkLayout CLy = chunk_layout(n, n_cvt, phi, n_grid, m);
    JB_CHECK_ARG(chunk_workspace && chunk_bytes >= CLy.total, "jb_lmm_chunk: chunk workspace too small");
    uint8_t* cws = static_cast<uint8_t*>(chunk_workspace);
    double* CL = reinterpret_cast<double*>(cws + CLy.cl);
    double* CQ = reinterpret_cast<double*>(cws + CLy.cq);
    // FP64 form: grid rows, ones row, null rows (only when prepared); mixed: ones + series
    const int rows = precision >= 1 ? 1 + kChebG : n_grid + 1 + (lmm_mode == 1 ? 0 : phi);
    const int rows_lin = rows * (n_cvt + phi);
    {
        if (precision != 2) {  // precision 2: CL already formed by jb_lmm_chunk_series_i8
            cublasHandle_t h = cublas_handle();
            if (!h) {
                set_error("cuBLAS handle creation failed");
                return JB_E_LIBRARY;
            }
            cublasStatus_t cs = bind_cublas(h, st, cws + CLy.blas, kCublasWorkspaceBytes);
            if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasSetStream/Workspace");
            const double one = 1.0, zero = 0.0;
            cs = cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, rows_lin, (int)m, (int)n, &one,
                             reinterpret_cast<const double*>(ws + L.alin), (int)n, UtG, (int)ldg,
                             &zero, CL, rows_lin);
            if (cs != CUBLAS_STATUS_SUCCESS) return cublas_status(cs, "cublasDgemm (linear x-sums)");
        }
        const int32_t rc = launch_sq_sums(reinterpret_cast<const double*>(ws + L.asqt), rows, UtG,
                                          ldg, n, m, reinterpret_cast<double*>(cws + CLy.sqp), CQ,
                                          rows, st);
        if (rc) return rc;
    }
    p.CL = CL;
    p.ldcl = rows_lin;
    p.CQ = CQ;
    p.ldcq = rows;
    switch (n_cvt) {
        case 1: return launch_pairs<1>(p, st);
        case 2: return launch_pairs<2>(p, st);
        case 3: return launch_pairs<3>(p, st);
        case 4: return launch_pairs<4>(p, st);
    }
    return JB_E_UNSUPPORTED;
}

int32_t jb_null_mle(int64_t n, int32_t n_cvt, int32_t phi, const double* evals, const double* UtW,
                    int64_t ldw, const double* Uty, int64_t ldy, double l_min, double l_max,
                    int32_t n_grid, int32_t n_iter, double* lam0, double* logl0,
                    uintptr_t stream) {
    JB_CHECK_ARG(n > 0 && phi >= 1 && n_grid >= 2 && n_iter >= 0, "jb_null_mle: bad sizes");
    JB_CHECK_ARG(n_cvt >= 1 && n_cvt <= kMaxCvt, "jb_null_mle: n_cvt must be in 1..%d", kMaxCvt);
    JB_CHECK_ARG(ldw >= n && ldy >= n, "jb_null_mle: bad leading dimension");
    JB_CHECK_ARG(l_min > 0 && l_max > l_min, "jb_null_mle: need 0 < l_min < l_max");
    const double lo = std::log(l_min), hi = std::log(l_max);
    const double step = (hi - lo) / (double)(n_grid - 1);
    const double c_mle = 0.5 * (double)n * (std::log((double)n) - std::log(2 * M_PI) - 1.0);
    cudaStream_t st = as_stream(stream);
    switch (n_cvt) {
#define JB_NULL_CASE(CC)                                                                     \
    case CC:                                                                                 \
        null_mle_kernel<CC><<<phi, 256, 0, st>>>(n, UtW, ldw, Uty, ldy, evals, lo, step,     \
                                                 n_grid, n_iter, hi, c_mle, lam0, logl0);    \
        JB_LAUNCH_CHECK("null_mle_kernel");                                                  \
        return JB_OK;
        JB_NULL_CASE(1)
        JB_NULL_CASE(2)
        JB_NULL_CASE(3)
        JB_NULL_CASE(4)
#undef JB_NULL_CASE
    }
    return JB_E_UNSUPPORTED;
}

}  // extern "C"
