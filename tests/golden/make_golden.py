"""Generate the committed golden fixtures under tests/golden/ (run in a container that
has the jamma reference checkout; the GPU test machines only read the outputs).

Two kinds of vectors are produced:

1. ``gemma_fixtures.npz`` -- the GEMMA 0.96/0.98 reference outputs that ship with
   jamma's test-suite (``tests/fixtures/gemma_synthetic``, ``gemma_covariate``,
   ``gemma_score``, ``gemma_all_tests``): packed genotypes, phenotypes, covariates,
   the GEMMA kinship and the numeric columns of each ``.assoc.txt``, plus the
   null-model log-likelihoods printed in the ``.log.txt`` files.

2. ``reference_likelihood.npz`` -- outputs of jamma's own NumPy module
   ``src/jamma/lmm/likelihood.py`` (importable without JAX), loaded by file path and
   evaluated on the gemma_synthetic cohort: Pab matrices, REML / MLE
   log-likelihoods of the alternative model at several lambdas for several SNPs,
   and both null-model optimisers.

Usage: python tests/golden/make_golden.py [/path/to/jamma/checkout]
"""

from __future__ import annotations

import importlib.util
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")
FX = REF / "tests" / "fixtures"
sys.path.insert(0, str(HERE.parents[1]))

from oracle.plink import read_bed_packed  # noqa: E402


def _assoc_columns(path: Path) -> dict:
    arr = np.genfromtxt(path, names=True, dtype=None, encoding=None)
    out = {}
    for name in arr.dtype.names:
        if name in ("chr", "rs", "allele1", "allele0"):
            continue
        out[name] = np.asarray(arr[name], dtype=np.float64)
    return out


def _null_logls(path: Path) -> tuple[float, float]:
    txt = path.read_text()
    reml = float(re.search(r"REMLE log-likelihood in the null model = (\S+)", txt).group(1))
    mle = float(re.search(r"## MLE log-likelihood in the null model = (\S+)", txt).group(1))
    return reml, mle


def make_gemma_fixtures() -> None:
    packed, n, p = read_bed_packed(FX / "gemma_synthetic" / "test")
    fam = [line.split() for line in (FX / "gemma_synthetic" / "test.fam").read_text().splitlines()]
    y = np.array([float(r[5]) for r in fam])
    cov = np.loadtxt(FX / "gemma_covariate" / "covariates.txt")
    kin = np.loadtxt(FX / "gemma_synthetic" / "gemma_kinship.cXX.txt")
    out = {"packed": packed, "n": n, "p": p, "pheno": y, "covariates": cov, "kinship": kin}
    cases = {
        "wald": FX / "gemma_synthetic" / "gemma_assoc.assoc.txt",
        "lrt": FX / "gemma_synthetic" / "gemma_lrt.assoc.txt",
        "score": FX / "gemma_score" / "gemma_score.assoc.txt",
        "all": FX / "gemma_all_tests" / "gemma_all.assoc.txt",
        "cov_wald": FX / "gemma_covariate" / "gemma_covariate.assoc.txt",
        "cov_lrt": FX / "gemma_covariate" / "gemma_covariate_lrt.assoc.txt",
        "cov_score": FX / "gemma_covariate" / "gemma_covariate_score.assoc.txt",
        "cov_all": FX / "gemma_all_tests" / "gemma_all_covar.assoc.txt",
    }
    for key, path in cases.items():
        for col, vals in _assoc_columns(path).items():
            out[f"{key}__{col}"] = vals
    logs = {
        "lrt": FX / "gemma_synthetic" / "gemma_lrt.log.txt",
        "cov_lrt": FX / "gemma_covariate" / "gemma_covariate_lrt.log.txt",
    }
    for key, path in logs.items():
        reml, mle = _null_logls(path)
        out[f"{key}__null_reml"] = np.float64(reml)
        out[f"{key}__null_mle"] = np.float64(mle)
    np.savez_compressed(HERE / "gemma_fixtures.npz", **out)


def _load_reference_likelihood():
    path = REF / "src" / "jamma" / "lmm" / "likelihood.py"
    spec = importlib.util.spec_from_file_location("jamma_ref_likelihood", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_reference_likelihood() -> None:
    lk = _load_reference_likelihood()
    g = np.load(HERE / "gemma_fixtures.npz")
    from oracle.plink import decode_packed

    geno = decode_packed(g["packed"], int(g["n"]))
    y = g["pheno"]
    kin = g["kinship"]
    evals, U = np.linalg.eigh(kin)
    evals = np.where(np.abs(evals) < 1e-10, 0.0, evals)
    UT = U.T
    out = {"evals": evals, "U": U}
    snps = np.array([0, 1, 7, 42, 123, 250, 499])
    lambdas = np.array([1e-5, 3e-3, 0.1, 0.6059673, 1.0, 7.5, 1e3, 1e5])
    for tag, W in (("ic", np.ones((y.size, 1))), ("cov", g["covariates"])):
        c = W.shape[1]
        UtW, Uty = UT @ W, UT @ y
        UtG = UT @ geno[:, snps]
        out[f"{tag}__UtW"], out[f"{tag}__Uty"], out[f"{tag}__UtG"] = UtW, Uty, UtG
        reml = np.zeros((snps.size, lambdas.size))
        mle = np.zeros_like(reml)
        pab = np.zeros((snps.size, lambdas.size, c + 2, (c + 3) * (c + 2) // 2))
        for j in range(snps.size):
            uab = lk.compute_Uab(UtW, Uty, UtG[:, j])
            for k, lam in enumerate(lambdas):
                reml[j, k] = lk.reml_log_likelihood(lam, evals, uab, c)
                mle[j, k] = lk.mle_log_likelihood(lam, evals, uab, c)
                pab[j, k] = lk.calc_pab(c, 1.0 / (lam * evals + 1.0), uab)
        out[f"{tag}__reml"], out[f"{tag}__mle"], out[f"{tag}__pab"] = reml, mle, pab
        lam_reml0, logl_reml0 = lk.compute_null_model_lambda(evals, UtW, Uty, c)
        lam_mle0, logl_mle0 = lk.compute_null_model_mle(evals, UtW, Uty, c)
        out[f"{tag}__null_reml"] = np.array([lam_reml0, logl_reml0])
        out[f"{tag}__null_mle"] = np.array([lam_mle0, logl_mle0])
    out["snps"], out["lambdas"] = snps, lambdas
    np.savez_compressed(HERE / "reference_likelihood.npz", **out)


if __name__ == "__main__":
    make_gemma_fixtures()
    make_reference_likelihood()
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)
