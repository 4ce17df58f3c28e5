"""Oracle restatement of jamma's per-SNP LMM association math (FP64, NumPy/SciPy).

All arrays are float64.  Shapes: n samples, m SNPs in a chunk, c = n_cvt covariate
columns, ni = n_index = (c+3)(c+2)/2 Uab pairs, r = c+2 projection levels.

The golden-section refinement is the *JAX* variant
(``src/jamma/lmm/likelihood_jax.py:419-488``), which recomputes both probe points
from the new bracket every step; the scalar null-model search is the *Python*
variant (``src/jamma/lmm/likelihood.py:395-474``), which carries one probe over.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy import special, stats

PHI = 0.6180339887498949
P_YY_MIN = 1e-8


# --------------------------------------------------------------------------- indices
def get_ab_index(a: int, b: int, n_cvt: int) -> int:
    """GEMMA GetabIndex, 1-based upper-triangular packing (``likelihood.py:25-43``)."""
    cols = n_cvt + 2
    a1, b1 = (a, b) if a <= b else (b, a)
    return (2 * cols - a1 + 2) * (a1 - 1) // 2 + b1 - a1


def index_table(n_cvt: int) -> dict:
    """Index mappings of ``build_index_table`` (``likelihood_jax.py:40-109``)."""
    ni = (n_cvt + 3) * (n_cvt + 2) // 2
    pairs = [
        (a - 1, b - 1, get_ab_index(a, b, n_cvt))
        for a in range(1, n_cvt + 3)
        for b in range(a, n_cvt + 3)
    ]
    rec = {}
    for p in range(1, n_cvt + 2):
        rec[p] = [
            (
                get_ab_index(a, b, n_cvt),
                get_ab_index(a, p, n_cvt),
                get_ab_index(b, p, n_cvt),
                get_ab_index(p, p, n_cvt),
            )
            for a in range(p + 1, n_cvt + 3)
            for b in range(a, n_cvt + 3)
        ]
    return {
        "n_index": ni,
        "idx_yy": get_ab_index(n_cvt + 2, n_cvt + 2, n_cvt),
        "idx_xx": get_ab_index(n_cvt + 1, n_cvt + 1, n_cvt),
        "idx_xy": get_ab_index(n_cvt + 2, n_cvt + 1, n_cvt),
        "pairs": pairs,
        "rec": rec,
        "diag": [(i, get_ab_index(i + 1, i + 1, n_cvt)) for i in range(n_cvt + 1)],
    }


# --------------------------------------------------------------------------- Uab / Pab
def build_uab(UtW: np.ndarray, Uty: np.ndarray, UtG: np.ndarray) -> np.ndarray:
    """(m, n, ni) products v_a*v_b of [W_1..W_c, x, y] (``batch_compute_uab``, 342-393)."""
    n, m = UtG.shape
    c = UtW.shape[1]
    t = index_table(c)
    uab = np.empty((m, n, t["n_index"]))
    xt = UtG.T
    for a, b, idx in t["pairs"]:
        va = UtW[:, a][None, :] if a < c else (xt if a == c else Uty[None, :])
        vb = UtW[:, b][None, :] if b < c else (xt if b == c else Uty[None, :])
        uab[:, :, idx] = va * vb
    return uab


def pab_recursion(n_cvt: int, row0: np.ndarray) -> np.ndarray:
    """Rows 1..c+1 of Pab from row 0 (``calc_pab_jax``, ``likelihood_jax.py:148-186``).

    ``P[p,ab] = P[p-1,ab] - P[p-1,aw] P[p-1,bw] / P[p-1,ww]`` with the inverse taken as
    0 when ``P[p-1,ww] == 0``.  ``row0`` has shape (..., ni).
    """
    t = index_table(n_cvt)
    out = np.zeros(row0.shape[:-1] + (n_cvt + 2, t["n_index"]))
    out[..., 0, :] = row0
    for p in range(1, n_cvt + 2):
        prev = out[..., p - 1, :]
        for i_ab, i_aw, i_bw, i_ww in t["rec"][p]:
            ww = prev[..., i_ww]
            with np.errstate(divide="ignore", invalid="ignore"):
                inv = np.where(ww != 0, 1.0 / np.where(ww != 0, ww, 1.0), 0.0)
            out[..., p, i_ab] = prev[..., i_ab] - prev[..., i_aw] * prev[..., i_bw] * inv
    return out


def calc_pab(n_cvt: int, hi: np.ndarray, uab: np.ndarray) -> np.ndarray:
    """Pab for every SNP; ``hi`` is (n,) shared or (m, n) per SNP."""
    if hi.ndim == 1:
        row0 = np.tensordot(uab, hi, axes=([1], [0]))
    else:
        row0 = np.matmul(hi[:, None, :], uab)[:, 0, :]
    return pab_recursion(n_cvt, row0)


# --------------------------------------------------------------------------- likelihoods
def _clamp_pyy(p):
    return np.where((p >= 0.0) & (p < P_YY_MIN), P_YY_MIN, p)


def _logdet_h(lam: np.ndarray, evals: np.ndarray) -> np.ndarray:
    v = lam[:, None] * evals[None, :] + 1.0
    return np.sum(np.log(np.abs(v)), axis=1), 1.0 / v


def reml_alt(n_cvt, lam, evals, uab, iab):
    """REML logl per SNP at per-SNP ``lam`` (``_reml_with_precomputed_iab``, 280-339)."""
    n = evals.shape[0]
    df = n - n_cvt - 1
    t = index_table(n_cvt)
    logdet_h, hi = _logdet_h(np.asarray(lam, dtype=np.float64), evals)
    pab = calc_pab(n_cvt, hi, uab)
    logdet_hiw = np.zeros(pab.shape[0])
    for row, col in t["diag"]:
        dp = pab[:, row, col]
        di = iab[:, row, col]
        with np.errstate(divide="ignore", invalid="ignore"):
            logdet_hiw = logdet_hiw + np.where(dp > 0, np.log(np.where(dp > 0, dp, 1.0)), 0.0)
            logdet_hiw = logdet_hiw - np.where(di > 0, np.log(np.where(di > 0, di, 1.0)), 0.0)
    pyy = _clamp_pyy(pab[:, n_cvt + 1, t["idx_yy"]])
    c = 0.5 * df * (np.log(df) - np.log(2 * np.pi) - 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        return c - 0.5 * logdet_h - 0.5 * logdet_hiw - 0.5 * df * np.log(pyy)


def mle_alt(n_cvt, lam, evals, uab):
    """MLE logl per SNP (``mle_log_likelihood_jax``, ``likelihood_jax.py:189-228``)."""
    n = evals.shape[0]
    t = index_table(n_cvt)
    logdet_h, hi = _logdet_h(np.asarray(lam, dtype=np.float64), evals)
    pab = calc_pab(n_cvt, hi, uab)
    pyy = _clamp_pyy(pab[:, n_cvt + 1, t["idx_yy"]])
    c = 0.5 * n * (np.log(n) - np.log(2 * np.pi) - 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        return c - 0.5 * logdet_h - 0.5 * n * np.log(pyy)


def _grid_logls(kind, n_cvt, lambdas, evals, uab, iab):
    """(g, m) logls on the shared grid (``_batch_grid_reml_with_iab`` 565-598, ``_batch_grid_mle`` 801-827)."""
    m = uab.shape[0]
    out = np.empty((lambdas.shape[0], m))
    for g, lam in enumerate(lambdas):
        lam_v = np.full(m, lam)
        out[g] = reml_alt(n_cvt, lam_v, evals, uab, iab) if kind == "reml" else mle_alt(
            n_cvt, lam_v, evals, uab
        )
    return out


def golden_refine(compute, all_logls, log_lambdas, n_grid, n_iter):
    """Grid bracket + JAX-style golden section (``_golden_section_refine``, 419-488).

    ``argmax`` picks the first maximum; the bracket is clamped to the grid; each step
    keeps the left part when ``fc > fd``, recomputes both probes from the new bracket,
    evaluates only the new one and carries the other value.  Returns exp of the bracket
    midpoint and the likelihood re-evaluated there.
    """
    best = np.argmax(all_logls, axis=0)
    lo = np.maximum(best - 1, 0)
    hi = np.minimum(best + 1, n_grid - 1)
    a = log_lambdas[lo]
    b = log_lambdas[hi]
    c = b - PHI * (b - a)
    d = a + PHI * (b - a)
    fc = compute(c)
    fd = compute(d)
    for _ in range(n_iter):
        keep_left = fc > fd
        na = np.where(keep_left, a, c)
        nb = np.where(keep_left, d, b)
        nc = nb - PHI * (nb - na)
        nd = na + PHI * (nb - na)
        new = compute(np.where(keep_left, nc, nd))
        fc, fd = np.where(keep_left, new, fd), np.where(keep_left, fc, new)
        a, b, c, d = na, nb, nc, nd
    log_opt = (a + b) / 2
    return np.exp(log_opt), compute(log_opt)


def grid_log_lambdas(l_min, l_max, n_grid):
    """``jnp.linspace(log(l_min), log(l_max), n_grid)`` (``likelihood_jax.py:540-543``)."""
    return np.linspace(np.log(l_min), np.log(l_max), n_grid)


def optimize_reml(n_cvt, evals, uab, iab, l_min=1e-5, l_max=1e5, n_grid=50, n_iter=20):
    """``golden_section_optimize_lambda`` (``likelihood_jax.py:491-562``)."""
    ll = grid_log_lambdas(l_min, l_max, n_grid)
    grid = _grid_logls("reml", n_cvt, np.exp(ll), evals, uab, iab)
    return golden_refine(
        lambda lg: reml_alt(n_cvt, np.exp(lg), evals, uab, iab), grid, ll, n_grid, n_iter
    )


def optimize_mle(n_cvt, evals, uab, l_min=1e-5, l_max=1e5, n_grid=50, n_iter=20):
    """``golden_section_optimize_lambda_mle`` (``likelihood_jax.py:830-883``)."""
    ll = grid_log_lambdas(l_min, l_max, n_grid)
    grid = _grid_logls("mle", n_cvt, np.exp(ll), evals, uab, None)
    return golden_refine(
        lambda lg: mle_alt(n_cvt, np.exp(lg), evals, uab), grid, ll, n_grid, n_iter
    )


# --------------------------------------------------------------------------- statistics
def _beta_se(pxx, pxy, px_yy, df):
    valid = pxx > 0
    safe_pxx = np.where(valid, pxx, 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        beta = np.where(valid, pxy / safe_pxx, np.nan)
        tau = df / px_yy
        var = np.where(valid, 1.0 / (tau * safe_pxx), np.nan)
        var = np.where(np.abs(var) < 0.001, np.abs(var), var)
        se = np.where(valid, np.sqrt(var), np.nan)
    return valid, beta, tau, se


def f_pvalue(f_stat, df, valid):
    """betainc(df/2, 1/2, clip(df/(df+max(F,1e-10)))) with F<=0 -> 1, invalid -> NaN."""
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.clip(df / (df + np.maximum(f_stat, 1e-10)), 0.0, 1.0)
        p = special.betainc(df / 2.0, 0.5, z)
    p = np.where(f_stat <= 0, 1.0, p)
    return np.where(valid, p, np.nan)


def wald_stats(n_cvt, lam, evals, uab, n_samples):
    """(beta, se, p_wald) per SNP (``calc_wald_stats_jax``, ``likelihood_jax.py:601-675``)."""
    df = n_samples - n_cvt - 1
    t = index_table(n_cvt)
    hi = 1.0 / (np.asarray(lam)[:, None] * evals[None, :] + 1.0)
    pab = calc_pab(n_cvt, hi, uab)
    pxx = pab[:, n_cvt, t["idx_xx"]]
    pxy = pab[:, n_cvt, t["idx_xy"]]
    pyy = pab[:, n_cvt, t["idx_yy"]]
    px_yy = _clamp_pyy(pab[:, n_cvt + 1, t["idx_yy"]])
    valid, beta, tau, se = _beta_se(pxx, pxy, px_yy, df)
    with np.errstate(invalid="ignore"):
        f = (pyy - px_yy) * tau
    return beta, se, f_pvalue(f, df, valid)


def score_stats(n_cvt, hi_null, uab, n_samples):
    """(beta, se, p_score) at the null H^-1 (``calc_score_stats_jax``, 706-798)."""
    df = n_samples - n_cvt - 1
    t = index_table(n_cvt)
    pab = calc_pab(n_cvt, hi_null, uab)
    pyy = pab[:, n_cvt, t["idx_yy"]]
    pxx = pab[:, n_cvt, t["idx_xx"]]
    pxy = pab[:, n_cvt, t["idx_xy"]]
    px_yy = _clamp_pyy(pab[:, n_cvt + 1, t["idx_yy"]])
    valid, beta, _tau, se = _beta_se(pxx, pxy, px_yy, df)
    with np.errstate(divide="ignore", invalid="ignore"):
        f = n_samples * (pxy * pxy) / (pyy * np.where(valid, pxx, 1.0))
    return beta, se, f_pvalue(f, df, valid)


def lrt_pvalue(logl_h1, logl_h0):
    """chi2_1 survival of max(2(l1-l0), 0) (``calc_lrt_pvalue_jax``, 231-251)."""
    return stats.chi2.sf(np.maximum(2.0 * (logl_h1 - logl_h0), 0.0), df=1)


# --------------------------------------------------------------------------- null model
def _mle_null(lam, evals, uab_null, n_cvt):
    """Scalar null MLE logl (``mle_log_likelihood_null``, ``likelihood.py:349-392``)."""
    n = evals.shape[0]
    v = lam * evals + 1.0
    hi = 1.0 / v
    logdet_h = np.sum(np.log(np.abs(v)))
    pab = pab_recursion(n_cvt, hi @ uab_null)
    pyy = pab[n_cvt, get_ab_index(n_cvt + 2, n_cvt + 2, n_cvt)]
    if 0.0 <= pyy < P_YY_MIN:
        pyy = P_YY_MIN
    c = 0.5 * n * (np.log(n) - np.log(2 * np.pi) - 1.0)
    return c - 0.5 * logdet_h - 0.5 * n * np.log(pyy)


def golden_minimize(func, l_min=1e-5, l_max=1e5, n_grid=50, n_iter=20):
    """Scalar grid + golden minimiser (``_golden_section_minimize``, ``likelihood.py:395-474``)."""
    lo_l, hi_l = math.log(l_min), math.log(l_max)
    step = (hi_l - lo_l) / (n_grid - 1)
    lls = [lo_l + i * step for i in range(n_grid)]
    best_i, best_v = 0, func(math.exp(lls[0]))
    for i in range(1, n_grid):
        v = func(math.exp(lls[i]))
        if v < best_v:
            best_v, best_i = v, i
    a = lls[max(best_i - 1, 0)]
    b = lls[min(best_i + 1, n_grid - 1)]
    c = b - PHI * (b - a)
    d = a + PHI * (b - a)
    fc, fd = func(math.exp(c)), func(math.exp(d))
    for _ in range(n_iter):
        if fc < fd:
            b, d, fd = d, c, fc
            c = b - PHI * (b - a)
            fc = func(math.exp(c))
        else:
            a, c, fc = c, d, fd
            d = a + PHI * (b - a)
            fd = func(math.exp(d))
    opt = math.exp((a + b) / 2.0)
    return opt, -func(opt)


def null_uab(UtW, Uty):
    """Uab without the genotype columns (``compute_Uab(..., Utx=None)``, ``likelihood.py:46-142``)."""
    n, c = UtW.shape
    t = index_table(c)
    vec = np.column_stack([UtW, np.zeros(n), Uty])
    u = np.zeros((n, t["n_index"]))
    for a, b, idx in t["pairs"]:
        if a == c or b == c:
            continue
        u[:, idx] = vec[:, a] * vec[:, b]
    return u


def null_model_mle(evals, UtW, Uty, l_min=1e-5, l_max=1e5):
    """(lambda0_mle, logl_H0) (``compute_null_model_mle``, ``likelihood.py:571-607``)."""
    c = UtW.shape[1]
    u = null_uab(UtW, Uty)
    return golden_minimize(lambda lam: -_mle_null(lam, evals, u, c), l_min, l_max)


# --------------------------------------------------------------------------- eigen
def eigh_threshold(k: np.ndarray, threshold: float = 1e-10):
    """``np.linalg.eigh`` then |lambda| < threshold -> 0 (``src/jamma/lmm/eigen.py:94,118``)."""
    w, u = np.linalg.eigh(k)
    return np.where(np.abs(w) < threshold, 0.0, w), u


# --------------------------------------------------------------------------- chunk + runner
def lmm_chunk(mode, evals, UtW, Uty, UtG, logl_h0=None, lam0=None, l_min=1e-5, l_max=1e5,
              n_grid=50, n_refine=10):
    """All statistics of one rotated SNP chunk, per ``lmm_mode`` (``runner_streaming.py:469-554``).

    Returns a dict with keys lambda_remle, logl_h1, beta, se, p_wald, lambda_mle,
    logl_mle, p_lrt, p_score (arrays of length m; NaN where the mode has no value).
    """
    n, m = UtG.shape
    c = UtW.shape[1]
    n_iter = max(n_refine, 20)
    nan = np.full(m, np.nan)
    out = {k: nan.copy() for k in ("lambda_remle", "logl_h1", "beta", "se", "p_wald",
                                   "lambda_mle", "logl_mle", "p_lrt", "p_score")}
    uab = build_uab(UtW, Uty, UtG)
    if mode in (3, 4):
        hi0 = 1.0 / (lam0 * evals + 1.0)
        b, s, p = score_stats(c, hi0, uab, n)
        out["p_score"] = p
        if mode == 3:
            out["beta"], out["se"] = b, s
    if mode in (2, 4):
        lm, llm = optimize_mle(c, evals, uab, l_min, l_max, n_grid, n_iter)
        out["lambda_mle"], out["logl_mle"] = lm, llm
        out["p_lrt"] = lrt_pvalue(llm, logl_h0)
    if mode in (1, 4):
        iab = pab_recursion(c, uab.sum(axis=1))
        lr, llr = optimize_reml(c, evals, uab, iab, l_min, l_max, n_grid, n_iter)
        b, s, p = wald_stats(c, lr, evals, uab, n)
        out.update(lambda_remle=lr, logl_h1=llr, beta=b, se=s, p_wald=p)
    return out


@dataclass
class LmmOracleResult:
    snp_indices: np.ndarray
    af: np.ndarray
    n_miss: np.ndarray
    lam0: float | None
    logl_h0: float | None
    stats: dict = field(default_factory=dict)


def lmm_association(g, phenotypes, kinship=None, covariates=None, eigenvalues=None,
                    eigenvectors=None, lmm_mode=1, maf_threshold=0.01, miss_threshold=0.05,
                    l_min=1e-5, l_max=1e5, n_grid=50, n_refine=10, chunk=2000):
    """``run_lmm_association_streaming`` on an in-memory (n, p) genotype matrix.

    Restates ``src/jamma/lmm/runner_streaming.py:94-628``: valid-sample mask
    (188-198), float32 pass-1 statistics (224-256), filter (286-290), eigh (332-341),
    W (``prepare.py:41-74``), rotations UtW/Uty (349-352), null MLE for modes 2/3/4
    (``prepare.py:114-155``), then per chunk: impute NaN with the float32 pass-1 mean
    (no centering, 427-434), rotate ``UT @ G`` and run :func:`lmm_chunk`.
    """
    y = np.asarray(phenotypes, dtype=np.float64)
    valid = ~np.isnan(y) & (y != -9.0)
    if covariates is not None:
        valid &= np.all(~np.isnan(covariates), axis=1)
    y = y[valid]
    g = np.asarray(g)[valid]
    if kinship is not None:
        kinship = kinship[np.ix_(valid, valid)]
    W = np.ones((y.shape[0], 1)) if covariates is None else np.asarray(covariates, np.float64)[valid]
    n = y.shape[0]
    from oracle.kinship import filter_mask, stream_pass1_means

    mean32, miss, var = stream_pass1_means(g)
    mask, af = filter_mask(mean32, miss, var, n, maf_threshold, miss_threshold)
    idx = np.where(mask)[0]
    if eigenvalues is None:
        eigenvalues, eigenvectors = eigh_threshold(kinship)
    UT = np.ascontiguousarray(eigenvectors.T)
    UtW = UT @ W
    Uty = UT @ y
    lam0 = logl0 = None
    if lmm_mode in (2, 3, 4):
        lam0, logl0 = null_model_mle(eigenvalues, UtW, Uty, l_min, l_max)
    res = LmmOracleResult(idx, af[idx], miss[idx].astype(int), lam0, logl0)
    parts = []
    means = np.asarray(mean32, dtype=np.float64)
    for s in range(0, idx.size, chunk):
        cols = idx[s : s + chunk]
        gc = np.asarray(g[:, cols], dtype=np.float64)
        gc = np.where(np.isnan(gc), means[cols][None, :], gc)
        parts.append(lmm_chunk(lmm_mode, eigenvalues, UtW, Uty, UT @ gc, logl0, lam0,
                               l_min, l_max, n_grid, n_refine))
    keys = parts[0].keys() if parts else []
    res.stats = {k: np.concatenate([p[k] for p in parts]) for k in keys}
    return res


def loco_association(g, phenotypes, chroms, covariates=None, lmm_mode=1, maf_threshold=0.01,
                     miss_threshold=0.05, chunk=2000):
    """``run_lmm_loco`` (``src/jamma/lmm/loco.py:54-252``): per chromosome (sorted names)
    the LOCO kinship (filtered with the association's MAF / missing thresholds over all
    samples) is restricted to the analysed samples and eigendecomposed; that chromosome's
    SNPs are tested with float64 statistics and imputation means over the analysed
    samples (``_run_lmm_for_chromosome``, 255-593).  Returns a list of
    (chr, snp_indices, af, n_miss, stats) in output order.
    """
    from oracle.kinship import filter_mask, loco_kinships, snp_stats

    chroms = np.asarray(chroms).astype(str)
    y = np.asarray(phenotypes, dtype=np.float64)
    valid = ~np.isnan(y) & (y != -9.0)
    if covariates is not None:
        valid &= np.all(~np.isnan(covariates), axis=1)
    yv = y[valid]
    W = np.ones((yv.size, 1)) if covariates is None else np.asarray(covariates, np.float64)[valid]
    n = yv.size
    out = []
    for c, K in loco_kinships(g, chroms, maf_threshold, miss_threshold):
        evals, U = eigh_threshold(K[np.ix_(valid, valid)])
        cols = np.where(chroms == c)[0]
        gc = np.asarray(g[np.ix_(valid, cols)], dtype=np.float64)
        mean, miss, var = snp_stats(gc)
        mask, af = filter_mask(mean, miss, var, n, maf_threshold, miss_threshold)
        loc = np.where(mask)[0]
        if loc.size == 0:
            continue
        UT = np.ascontiguousarray(U.T)
        UtW, Uty = UT @ W, UT @ yv
        lam0 = l0 = None
        if lmm_mode in (2, 3, 4):
            lam0, l0 = null_model_mle(evals, UtW, Uty)
        parts = []
        for s in range(0, loc.size, chunk):
            sub = loc[s:s + chunk]
            gs = gc[:, sub]
            gs = np.where(np.isnan(gs), mean[sub][None, :], gs)
            parts.append(lmm_chunk(lmm_mode, evals, UtW, Uty, UT @ gs, l0, lam0))
        stats = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
        out.append((c, cols[loc], af[loc], miss[loc].astype(int), stats))
    return out
