"""Command line with jamma's GEMMA-style flags (src/jamma/cli.py:54-524).

    python -m jamma_b200.cli [-outdir D] [-o P] gk -bfile B [-gk 1|2] [-maf M] [-miss R]
                             [-loco] [-eigen] [-n N] [-ksnps FILE] [-precision fp64|mixed]
    python -m jamma_b200.cli [-outdir D] [-o P] lmm -bfile B [-k K | -d D -u U | -loco]
                             [-c C] [-lmm 1-4] [-maf M] [-miss R] [-eigen] [-n N]
                             [-snps FILE] [-ksnps FILE] [-hwe P] [-precision fp64|mixed]

``-precision`` (not a GEMMA flag) selects the form of the device steps: ``fp64`` (the
default) reproduces jamma's FP64 results; ``mixed`` runs the INT8 tensor-core kinship
Gram, the INT8 digit-plane rotation and the series-interpolated lambda search (-gk 1 only;
-gk 2 stays FP64).

Both commands write ``{outdir}/{prefix}.log.txt`` in GEMMA's ``##`` layout.  Errors are
reported as ``Error: ...`` with exit status 1 (cli.py:485-487).
"""

from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path


def _snp_indices(path, sid) -> "np.ndarray":
    from jamma_b200.io import read_snp_list_file, resolve_snp_list_to_indices

    return resolve_snp_list_to_indices(read_snp_list_file(path), sid)


def _gk(a, command_line: str) -> None:
    from jamma_b200.io import get_plink_metadata, write_eigen_files, write_gemma_log, write_kinship_matrix
    from jamma_b200.kinship import compute_kinship_from_bed

    t0 = time.perf_counter()
    if a.gk not in (1, 2):
        raise ValueError(f"invalid kinship mode {a.gk}. Use -gk 1 or -gk 2.")
    out = Path(a.outdir)
    meta = get_plink_metadata(a.bfile)
    ks = _snp_indices(a.ksnps, meta["sid"]) if a.ksnps else None
    kin_precision = "int8" if a.precision == "mixed" else "fp64"
    if a.gk == 2 and a.precision == "mixed":
        raise ValueError("-gk 2 (standardized) is computed in FP64 only; drop -precision mixed")
    if a.loco:
        if a.gk == 2:
            raise ValueError("-gk 2 (standardized) is not supported with -loco; LOCO kinship "
                             "uses centered mode (-gk 1)")
        from jamma_b200.io import write_kinship_matrix as _w
        from jamma_b200.loco import compute_loco_kinship

        n_chr = 0
        for chrom, K in compute_loco_kinship(a.bfile, a.maf, a.miss, ksnps_indices=ks,
                                             precision=kin_precision):
            _w(K.cpu().numpy(), out / f"{a.prefix}.loco.cXX.chr{chrom}.txt")
            n_chr += 1
        elapsed = time.perf_counter() - t0
        write_gemma_log(out, a.prefix, {"kinship_mode": "loco", "n_chromosomes": n_chr,
                                        "maf_threshold": a.maf, "miss_threshold": a.miss},
                        {"total": elapsed, "kinship": elapsed}, command_line)
        print(f"wrote {n_chr} LOCO kinship matrices to {out}")
        return
    K = compute_kinship_from_bed(a.bfile, a.maf, a.miss, kinship_mode=a.gk, ksnps_indices=ks,
                                 precision=kin_precision)
    t_k = time.perf_counter() - t0
    kpath = out / f"{a.prefix}.cXX.txt"
    write_kinship_matrix(K, kpath)
    print(f"wrote {kpath}")
    if a.eigen:
        from jamma_b200.eigen import eigendecompose_kinship

        evals, evecs = eigendecompose_kinship(K)
        d, u = write_eigen_files(evals, evecs, out, a.prefix)
        print(f"wrote {d} and {u}")
    write_gemma_log(out, a.prefix, {"n_samples": meta["n_samples"], "n_snps": meta["n_snps"],
                                    "kinship_mode": a.gk, "kinship_file": str(kpath),
                                    "maf_threshold": a.maf, "miss_threshold": a.miss},
                    {"total": time.perf_counter() - t0, "kinship": t_k}, command_line)


def _lmm(a, command_line: str) -> None:
    from jamma_b200.gwas import gwas
    from jamma_b200.io import write_gemma_log

    if (a.eigenD is None) != (a.eigenU is None):
        raise ValueError("-d and -u must be given together")
    if a.kinship is None and a.eigenD is None and not a.loco:
        raise ValueError("lmm needs -k, -d/-u or -loco")
    r = gwas(a.bfile, kinship_file=a.kinship, covariate_file=a.covar, lmm_mode=a.mode,
             maf=a.maf, miss=a.miss, output_dir=a.outdir, output_prefix=a.prefix,
             loco=a.loco, eigenvalue_file=a.eigenD, eigenvector_file=a.eigenU,
             write_eigen=a.eigen, phenotype_column=a.pheno_col, snps_file=a.snps,
             ksnps_file=a.ksnps, hwe=a.hwe, precision=a.precision)
    write_gemma_log(a.outdir, a.prefix, {"n_samples": r.n_samples, "n_snps": r.n_snps_tested,
                                         "lmm_mode": a.mode, "maf_threshold": a.maf,
                                         "miss_threshold": a.miss, "precision": a.precision},
                    {k.removesuffix("_s"): v for k, v in r.timing.items()}, command_line)
    print(f"{r.n_snps_tested} SNPs, {r.timing['total_s']:.2f}s -> "
          f"{Path(a.outdir) / (a.prefix + '.assoc.txt')}")


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    ap = argparse.ArgumentParser(prog="jamma_b200")
    ap.add_argument("-outdir", default="output")
    ap.add_argument("-o", dest="prefix", default="result")
    ap.add_argument("-v", dest="verbose", action="store_true")
    sub = ap.add_subparsers(dest="cmd", required=True)
    gk = sub.add_parser("gk")
    gk.add_argument("-bfile", required=True)
    gk.add_argument("-gk", type=int, default=1)
    gk.add_argument("-maf", type=float, default=0.0)
    gk.add_argument("-miss", type=float, default=1.0)
    gk.add_argument("-loco", action="store_true")
    gk.add_argument("-eigen", action="store_true")
    gk.add_argument("-n", dest="pheno_col", type=int, default=1)
    gk.add_argument("-ksnps")
    gk.add_argument("-precision", choices=("fp64", "mixed"), default="fp64")
    gk.add_argument("--check-memory", dest="check_memory", action="store_true", default=True)
    gk.add_argument("--no-check-memory", dest="check_memory", action="store_false")
    lm = sub.add_parser("lmm")
    lm.add_argument("-bfile", required=True)
    lm.add_argument("-k", dest="kinship")
    lm.add_argument("-c", dest="covar")
    lm.add_argument("-lmm", dest="mode", type=int, default=1)
    lm.add_argument("-maf", type=float, default=0.01)
    lm.add_argument("-miss", type=float, default=0.05)
    lm.add_argument("-loco", action="store_true")
    lm.add_argument("-d", dest="eigenD")
    lm.add_argument("-u", dest="eigenU")
    lm.add_argument("-eigen", action="store_true")
    lm.add_argument("-n", dest="pheno_col", type=int, default=1)
    lm.add_argument("-snps")
    lm.add_argument("-ksnps")
    lm.add_argument("-hwe", type=float, default=0.0)
    lm.add_argument("-precision", choices=("fp64", "mixed"), default="fp64")
    lm.add_argument("--check-memory", dest="check_memory", action="store_true", default=True)
    lm.add_argument("--no-check-memory", dest="check_memory", action="store_false")
    a = ap.parse_args(argv)
    command_line = "jamma " + " ".join(argv)
    try:
        if a.cmd == "gk":
            _gk(a, command_line)
        else:
            _lmm(a, command_line)
    except (ValueError, FileNotFoundError, MemoryError, NotImplementedError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
