"""Command line with jamma's GEMMA-style flags (src/jamma/cli.py:54-524).

    python -m jamma_b200.cli [-outdir D] [-o P] gk -bfile B [-gk 1]
    python -m jamma_b200.cli [-outdir D] [-o P] lmm -bfile B -k K [-c C] [-lmm N]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="jamma_b200")
    ap.add_argument("-outdir", default="output")
    ap.add_argument("-o", dest="prefix", default="result")
    sub = ap.add_subparsers(dest="cmd", required=True)
    gk = sub.add_parser("gk")
    gk.add_argument("-bfile", required=True)
    gk.add_argument("-gk", type=int, default=1)
    gk.add_argument("-maf", type=float, default=0.0)
    gk.add_argument("-miss", type=float, default=1.0)
    lm = sub.add_parser("lmm")
    lm.add_argument("-bfile", required=True)
    lm.add_argument("-k", dest="kinship")
    lm.add_argument("-c", dest="covar")
    lm.add_argument("-lmm", dest="mode", type=int, default=1)
    lm.add_argument("-maf", type=float, default=0.01)
    lm.add_argument("-miss", type=float, default=0.05)
    lm.add_argument("-n", dest="pheno_col", type=int, default=1)
    lm.add_argument("-d", dest="eigenD")
    lm.add_argument("-u", dest="eigenU")
    lm.add_argument("-hwe", type=float, default=0.0)
    a = ap.parse_args(argv)
    try:
        if a.cmd == "gk":
            if a.gk != 1:
                raise ValueError("only -gk 1 (centered kinship) is available")
            from jamma_b200.io import write_kinship_matrix
            from jamma_b200.kinship import compute_kinship_from_bed

            K = compute_kinship_from_bed(a.bfile, a.maf, a.miss)
            out = Path(a.outdir) / f"{a.prefix}.cXX.txt"
            write_kinship_matrix(K, out)
            print(f"wrote {out}")
        else:
            from jamma_b200.gwas import gwas

            r = gwas(a.bfile, kinship_file=a.kinship, covariate_file=a.covar, lmm_mode=a.mode,
                     maf=a.maf, miss=a.miss, output_dir=a.outdir, output_prefix=a.prefix,
                     eigenvalue_file=a.eigenD, eigenvector_file=a.eigenU,
                     phenotype_column=a.pheno_col, hwe=a.hwe)
            print(f"{r.n_snps_tested} SNPs, {r.timing['total_s']:.2f}s -> "
                  f"{Path(a.outdir) / (a.prefix + '.assoc.txt')}")
    except (ValueError, FileNotFoundError, MemoryError, NotImplementedError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
