"""One-call GWAS pipeline with jamma's ``gwas()`` signature (src/jamma/gwas.py:40-167).

Steps follow ``PipelineRunner.run`` (src/jamma/pipeline.py:426-609): phenotypes from
the .fam column, kinship from file or computed from the .bed (all samples, streamed),
covariates, then the streaming association written to ``{output_dir}/{prefix}.assoc.txt``.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from jamma_b200.io import (
    AssocResult,
    get_plink_metadata,
    read_covariate_file,
    read_eigen_files,
    read_kinship_matrix,
    read_phenotypes,
    read_snp_list_file,
    resolve_snp_list_to_indices,
    write_eigen_files,
    write_kinship_matrix,
)
from jamma_b200.kinship import compute_kinship_from_bed
from jamma_b200.lmm import run_lmm_association_streaming


@dataclass
class GWASResult:
    associations: list[AssocResult]
    n_samples: int
    n_snps_tested: int
    timing: dict[str, float] = field(default_factory=dict)


def gwas(bfile, *, kinship_file=None, covariate_file=None, lmm_mode: int = 1, maf: float = 0.01,
         miss: float = 0.05, output_dir="output", output_prefix: str = "result",
         save_kinship: bool = False, check_memory: bool = True, show_progress: bool = True,
         loco: bool = False, eigenvalue_file=None, eigenvector_file=None, write_eigen: bool = False,
         phenotype_column: int = 1, snps_file=None, ksnps_file=None, hwe: float = 0.0,
         precision: str = "fp64") -> GWASResult:
    """Kinship (or eigen files), then the streaming association written to
    ``{output_dir}/{output_prefix}.assoc.txt``, with jamma's arguments and defaults.

    ``precision`` picks the form of every device step: ``"fp64"`` (default) is FP64
    throughout and reproduces jamma's results; ``"mixed"`` computes the kinship with the
    exact INT8 tensor-core Gram plus FP64 corrections, rotates genotypes on the INT8
    tensor cores (four base-254 digit planes of the eigenvectors, exact int32 products) and
    runs the series-interpolated lambda search, with FP64 likelihoods and statistics.
    """
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
    kin_precision = "int8" if precision == "mixed" else "fp64"
    if lmm_mode not in (1, 2, 3, 4):
        raise ValueError(f"lmm_mode must be 1, 2, 3 or 4, got {lmm_mode}")
    if loco and kinship_file is not None:
        raise ValueError("kinship_file and loco are mutually exclusive")
    if (eigenvalue_file is None) != (eigenvector_file is None):
        raise ValueError("eigenvalue_file and eigenvector_file must be provided together")
    t0 = time.perf_counter()
    bfile = Path(bfile)
    meta = get_plink_metadata(bfile)
    n = meta["n_samples"]
    y = read_phenotypes(bfile, phenotype_column)
    n_analyzed = int(np.sum(~np.isnan(y) & (y != -9.0)))
    if n_analyzed == 0:  # pipeline.py:286-291
        raise ValueError("No samples with valid phenotypes")
    sid = list(meta["sid"])
    snps_idx = None
    if snps_file is not None:
        snps_idx = resolve_snp_list_to_indices(read_snp_list_file(snps_file), sid)
    cov = None
    if covariate_file is not None:
        cov, _ = read_covariate_file(covariate_file)
        if cov.shape[0] != n:
            raise ValueError(f"Covariate file has {cov.shape[0]} rows but .fam has {n} samples")
    ks = None
    if ksnps_file is not None:
        ks = resolve_snp_list_to_indices(read_snp_list_file(ksnps_file), sid)
    evals = evecs = K = None
    if loco:
        pass
    elif eigenvalue_file is not None:
        evals, evecs = read_eigen_files(eigenvalue_file, eigenvector_file, n_samples=n_analyzed)
    else:
        if kinship_file is not None:
            K = read_kinship_matrix(kinship_file, n_samples=n)
        else:
            K = compute_kinship_from_bed(bfile, ksnps_indices=ks, precision=kin_precision)
            if save_kinship:
                write_kinship_matrix(K, Path(output_dir) / f"{output_prefix}.cXX.txt")
        if write_eigen:  # eigen files of the analysed samples (pipeline.py:549-566)
            from jamma_b200.eigen import eigendecompose_kinship

            valid = ~np.isnan(y) & (y != -9.0)
            Kv = K if np.all(valid) else K[np.ix_(valid, valid)]
            evals, evecs = eigendecompose_kinship(Kv, check_memory=check_memory)
            write_eigen_files(evals, evecs, output_dir, output_prefix)
    t_k = time.perf_counter()
    out = Path(output_dir) / f"{output_prefix}.assoc.txt"
    timing: dict = {}
    if loco:
        from jamma_b200.loco import run_lmm_loco

        res = run_lmm_loco(bfile, y, covariates=cov, maf_threshold=maf, miss_threshold=miss,
                           lmm_mode=lmm_mode, output_path=out, save_kinship=save_kinship,
                           kinship_output_dir=Path(output_dir), kinship_output_prefix=output_prefix,
                           snps_indices=snps_idx, ksnps_indices=ks, precision=precision,
                           kinship_precision=kin_precision)
        t_end = time.perf_counter()
        n_valid = int(np.sum(~np.isnan(y) & (y != -9.0)))
        return GWASResult(res, n_valid, meta["n_snps"],
                          {"kinship_s": 0.0, "lmm_s": t_end - t0, "total_s": t_end - t0})
    res = run_lmm_association_streaming(
        bfile, y, kinship=K, covariates=cov, eigenvalues=evals, eigenvectors=evecs,
        maf_threshold=maf, miss_threshold=miss, output_path=out, lmm_mode=lmm_mode,
        snps_indices=snps_idx, hwe_threshold=hwe, timing=timing, precision=precision)
    t_end = time.perf_counter()
    n_valid = int(np.sum(~np.isnan(y) & (y != -9.0)))
    return GWASResult(res, n_valid, meta["n_snps"],
                      {"kinship_s": t_k - t0, "lmm_s": t_end - t_k, "total_s": t_end - t0, **timing})
