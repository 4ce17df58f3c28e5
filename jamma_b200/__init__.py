"""jamma_b200: jamma's GEMMA-style LMM association hot path on NVIDIA B200 (sm_100a).

Public API (same names, arguments and error behaviour as jamma 2.0.1):

- :func:`compute_centered_kinship` -- GEMMA -gk 1 relatedness matrix
- :func:`compute_standardized_kinship` -- GEMMA -gk 2 relatedness matrix
- :func:`eigendecompose_kinship` -- FP64 eigendecomposition with jamma's thresholding
- :func:`run_lmm_association_streaming`, :func:`run_lmm_association_jax` -- -lmm 1..4
- :func:`gwas` -- one-call pipeline (kinship -> eigen -> association -> .assoc.txt)

All arithmetic runs in ``libjamma_b200.so`` (hand-written CUDA for sm_100a plus
cuBLAS / cuSOLVER); PyTorch only owns device buffers and streams.
"""

from jamma_b200.eigen import eigendecompose_kinship
from jamma_b200.io import (
    AssocResult,
    IncrementalAssocWriter,
    read_covariate_file,
    read_eigen_files,
    read_kinship_matrix,
    write_assoc_results,
    write_eigen_files,
    write_kinship_matrix,
)
from jamma_b200.kinship import (
    compute_centered_kinship,
    compute_kinship_from_bed,
    compute_standardized_kinship,
)
from jamma_b200.lmm import run_lmm_association_jax, run_lmm_association_streaming

__version__ = "0.1.0"

# Imported eagerly: importing the submodule later would rebind the package attribute
# ``gwas`` to the module and break a second call of the function.
from jamma_b200.gwas import gwas  # noqa: E402


__all__ = [
    "AssocResult",
    "IncrementalAssocWriter",
    "compute_centered_kinship",
    "compute_kinship_from_bed",
    "compute_standardized_kinship",
    "eigendecompose_kinship",
    "gwas",
    "read_covariate_file",
    "read_eigen_files",
    "read_kinship_matrix",
    "run_lmm_association_jax",
    "run_lmm_association_streaming",
    "write_assoc_results",
    "write_eigen_files",
    "write_kinship_matrix",
]
