"""Continuous-batching server: jobs run concurrently give the same results as alone.

Each job's arithmetic is the ordinary association path with its own buffers and a fixed
chunk width, and the kinship / eigendecomposition are deterministic, so the results of
a job served in a mix of concurrent jobs must equal those of the job served alone.  The
stated tolerance is 1e-12 relative (it holds bit-exactly on one device).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from jamma_b200 import synth
from oracle import plink as OP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jamma_b200 import _build

    _build.build()


def _jobs():
    from jamma_b200.serve import GwasJob

    specs = [  # (cohort, n, p, phenotypes, mode, seed)
        ("A", 300, 1200, 1, 4, 1), ("B", 450, 900, 2, 1, 2), ("A", 300, 1200, 3, 2, 3),
        ("C", 200, 1500, 1, 3, 4), ("B", 450, 900, 1, 4, 5),
    ]
    geno = {}
    jobs = []
    for i, (cid, n, p, phi, mode, seed) in enumerate(specs):
        if cid not in geno:
            geno[cid] = synth.genotypes(n, p, 0.01, seed=100 + n)
        g = geno[cid]
        y = synth.phenotypes(np.nan_to_num(g, nan=1.0), seed=seed, n_pheno=phi)
        cov = synth.covariates(n, 1, seed=seed) if i % 2 else None
        jobs.append(GwasJob(f"job{i}", cid, OP.encode_genotypes(g), n, y, cov, mode))
    return jobs


def _serve(jobs, max_active, capture_graphs=True):
    from jamma_b200.serve import GwasServer

    srv = GwasServer(hbm_budget_bytes=8 << 30, max_active=max_active, chunk=512,
                     capture_graphs=capture_graphs)
    for j in jobs:
        srv.submit(j)
    done = srv.run()
    return {j.job_id: j for j in done}, srv


def test_results_are_the_same_alone_and_in_the_mix():
    mixed, srv = _serve(_jobs(), max_active=4)
    assert len(mixed) == 5
    summary = srv.latency_summary()
    assert summary["p99_s"] >= summary["p50_s"] > 0
    for job in _jobs():
        alone, _ = _serve([job], max_active=1)
        a, b = alone[job.job_id], mixed[job.job_id]
        np.testing.assert_array_equal(a.snp_indices, b.snp_indices)
        for k in a.results:
            np.testing.assert_allclose(a.results[k], b.results[k], rtol=1e-12, atol=0,
                                       err_msg=f"{job.job_id}:{k}")


def test_eager_chunks_equal_graph_replays():
    """capture_graphs=False issues each chunk's launches eagerly: the same results, bit for
    bit, as replaying the captured graphs."""
    graphs, _ = _serve(_jobs(), max_active=4)
    eager, _ = _serve(_jobs(), max_active=4, capture_graphs=False)
    for jid, a in graphs.items():
        b = eager[jid]
        np.testing.assert_array_equal(a.snp_indices, b.snp_indices)
        for k in a.results:
            np.testing.assert_array_equal(a.results[k], b.results[k], err_msg=f"{jid}:{k}")


def test_server_matches_the_streaming_runner(tmp_path):
    """A served job equals run_lmm_association_streaming on the same cohort (mixed form)."""
    from jamma_b200 import eigendecompose_kinship, run_lmm_association_streaming
    from jamma_b200.kinship import compute_centered_kinship

    job = _jobs()[1]
    g = OP.decode_packed(job.packed, job.n_samples)
    OP.write_plink(tmp_path / "s", g)
    served, srv = _serve([job], max_active=1)
    res = srv.cohorts[job.cohort_id]
    evals = res.evals.cpu().numpy()
    U = res.U.cpu().numpy().T
    y = job.phenotypes[:, 0]
    out = run_lmm_association_streaming(tmp_path / "s", y, eigenvalues=evals, eigenvectors=U,
                                        covariates=job.covariates, lmm_mode=job.lmm_mode,
                                        precision="mixed", chunk_size=512)
    got = np.array([r.p_wald for r in out])
    # the two paths use different chunk widths (cuBLAS shapes): allow rare golden near-ties
    rel = np.abs(served[job.job_id].results["p_wald"][0] - got) / np.abs(got)
    assert np.mean(rel < 1e-9) >= 0.99, rel.max()
    del compute_centered_kinship, eigendecompose_kinship


def test_over_budget_job_is_rejected():
    from jamma_b200.serve import GwasServer

    job = _jobs()[0]
    srv = GwasServer(hbm_budget_bytes=1 << 20, max_active=2)
    srv.submit(job)
    with pytest.raises(MemoryError):
        srv.run()
