"""CPU oracle for the LMM association hot path (test infrastructure only).

This package is a NumPy/SciPy restatement of jamma's GEMMA-style linear mixed
model path: PLINK decoding, pass-1 SNP statistics and filters, centered
kinship, eigendecomposition, rotation, the Uab/Pab projections, REML/MLE
likelihoods, the grid + golden-section variance-ratio search and the
Wald / likelihood-ratio / score statistics.  Every function cites the
reference file and line it restates (paths inside the jamma project).

It is the *checker*: only the test-suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it.  The product package
``jamma_b200`` never imports it and has no CPU fallback.

Pinning: the restatement is checked against GEMMA fixtures shipped with the
reference (kinship ``.cXX.txt``, Wald/LRT/Score/all-tests ``.assoc.txt``,
null-model log-likelihoods in ``.log.txt``) and against golden vectors
produced by the reference's own NumPy module ``jamma/lmm/likelihood.py``
(see ``tests/golden/make_golden.py``).
"""

from oracle.plink import read_bed, read_bim, read_fam, write_plink  # noqa: F401
from oracle.kinship import centered_kinship, snp_stats  # noqa: F401
from oracle.lmm import (  # noqa: F401
    LmmOracleResult,
    eigh_threshold,
    lmm_association,
    null_model_mle,
)
