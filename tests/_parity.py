"""Comparison helpers for the GPU parity tests (device results against the CPU oracle).

Plain FP64 form: lambda 1e-9 relative and other fields 1e-8 relative for at least
``min_frac`` of SNPs, lambda always within the golden section's final bracket (1e-4),
every p-value within 1e-6 relative or 1e-12 absolute, identical calls at 0.05 / 1e-3 /
5e-8.  Mixed form: identical NaN pattern, every |log10 p| error below 1e-4 and identical
calls (lambda is not compared: a golden-section step on a flat likelihood may resolve
differently).
"""

from __future__ import annotations

import numpy as np

FIELDS = {"l_remle": "lambda_remle", "logl_H1": "logl_h1", "beta": "beta", "se": "se",
          "p_wald": "p_wald", "l_mle": "lambda_mle", "p_lrt": "p_lrt", "p_score": "p_score"}


def _arrays(results):
    out = {}
    for field, key in FIELDS.items():
        vals = [getattr(r, field) for r in results]
        if all(v is not None for v in vals):
            out[key] = np.array(vals, dtype=float)
    return out


def _rel(a, b):
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def _finite_pair(got, ref, k):
    a, b = np.asarray(got[k], float), np.asarray(ref[k], float)
    assert a.shape == b.shape, k
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    np.testing.assert_array_equal(nan_a, nan_b, err_msg=f"{k}: NaN pattern")
    return a[~nan_a], b[~nan_b]


def assert_assoc_parity(got: dict, ref: dict, keys, min_frac: float = 0.99):
    for k in keys:
        a, b = _finite_pair(got, ref, k)
        if a.size == 0:
            continue
        r = _rel(a, b)
        tight = 1e-9 if k.startswith("lambda") else 1e-8
        frac = np.mean(r <= tight)
        assert frac >= min_frac, f"{k}: only {frac:.4f} within {tight}; worst {r.max():.3e}"
        if k.startswith("lambda"):
            assert r.max() <= 1e-4, f"{k}: worst {r.max():.3e}"
        if k.startswith("p_"):
            ok = (r <= 1e-6) | (np.abs(a - b) <= 1e-12)
            assert ok.mean() >= 0.999, f"{k}: worst {r.max():.3e}"
            for t in (0.05, 1e-3, 5e-8):
                np.testing.assert_array_equal(a < t, b < t, err_msg=f"{k}: calls at {t}")


def assert_mixed_parity(got: dict, ref: dict, keys):
    for k in keys:
        a, b = _finite_pair(got, ref, k)
        if a.size == 0 or not k.startswith("p_"):
            continue
        with np.errstate(divide="ignore", invalid="ignore"):  # p = 0 on both sides
            dlog = np.abs(np.log10(a) - np.log10(b))
        dlog = np.where(a == b, 0.0, dlog)
        assert dlog.max() < 1e-4, f"{k}: |dlog10 p| {dlog.max():.2e}"
        for t in (0.05, 1e-3, 5e-8):
            np.testing.assert_array_equal(a < t, b < t, err_msg=f"{k}: calls at {t}")


def strict_fp64_report(got: dict, ref: dict, keys=("beta", "se", "logl_h1", "p_wald"),
                       lam_key: str = "lambda_remle", lam_tol: float = 1e-12,
                       tol: float = 1e-10, tols: dict | None = None) -> dict:
    """The plain FP64 form at the north-star tolerance: on every SNP whose REML lambda
    matches the oracle's to ``lam_tol`` relative (every golden-section decision taken the
    same way), each field in ``keys`` must agree to ``tol`` relative (``tols`` overrides it
    per field).  Returns the fraction of SNPs that qualify and the worst error among them
    per field.

    The rest of the SNPs took a golden-section step differently: in the last steps the two
    probes' log-likelihoods differ by less than the FP64 rounding of their length-n sums,
    so any two FP64 implementations (GPU and NumPy, or jamma's own NumPy and JAX paths)
    can branch differently there; lambda then stays within the final bracket."""
    la, lb = np.asarray(got[lam_key], float), np.asarray(ref[lam_key], float)
    same = np.isfinite(la) & np.isfinite(lb) & (_rel(la, lb) <= lam_tol)
    out = {"frac_lambda_matched": float(np.mean(same)), "n": int(same.size)}
    for k in keys:
        if k not in got or k not in ref:
            continue
        a, b = np.asarray(got[k], float)[same], np.asarray(ref[k], float)[same]
        ok = np.isfinite(a) & np.isfinite(b)
        np.testing.assert_array_equal(np.isfinite(a), np.isfinite(b), err_msg=f"{k}: NaN pattern")
        r = _rel(a[ok], b[ok])
        worst = float(r.max()) if r.size else 0.0
        out[k] = worst
        t = (tols or {}).get(k, tol)
        if worst > t:
            out.setdefault("violations", []).append(
                f"{k}: {worst:.3e} > {t} on a SNP whose lambda matches the oracle")
    return out


def assert_strict(rep: dict, min_frac: float = 0.5, label: str = "") -> None:
    """Fail on a report of :func:`strict_fp64_report` with violations, or with fewer than
    ``min_frac`` of the SNPs taking every golden-section step as the oracle."""
    assert not rep.get("violations"), f"{label} {rep['violations']}"
    assert rep["frac_lambda_matched"] >= min_frac, f"{label} {rep}"
