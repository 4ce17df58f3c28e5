"""Seeded synthetic cohorts with the shapes and distributions of the benchmark configs.

Genotypes x_ij ~ Binomial(2, p_j) with p_j ~ U(0.05, 0.5), i.i.d. missing calls at a
given rate; phenotype y = X_causal beta + g + e with beta ~ N(0, 0.3^2), a polygenic
term g scaled to heritability h2 and e ~ N(0, 1); covariates are an intercept plus
N(0, 1) columns.  Real cohorts (mouse_hs1940 and the like) are not reproduced; these
seeded stand-ins only share their sizes and value distributions.
"""

from __future__ import annotations

import numpy as np
import torch


def genotypes(n: int, p: int, miss_rate: float = 0.01, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    af = rng.uniform(0.05, 0.5, p)
    g = rng.binomial(2, af, size=(n, p)).astype(np.float64)
    if miss_rate > 0:
        g[rng.random((n, p)) < miss_rate] = np.nan
    return g


def phenotypes(g: np.ndarray, n_causal: int = 20, h2: float = 0.5, seed: int = 1,
               n_pheno: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n, p = g.shape
    x = np.where(np.isnan(g), np.nanmean(g, axis=0, keepdims=True), g)
    x = x - x.mean(0, keepdims=True)
    ys = []
    for _ in range(n_pheno):
        causal = rng.choice(p, size=min(n_causal, p), replace=False)
        fixed = x[:, causal] @ rng.normal(0, 0.3, causal.size)
        poly = x @ rng.normal(0, 1, p) / np.sqrt(p)
        poly *= np.sqrt(h2 / max(1 - h2, 1e-6) / max(poly.var(), 1e-12))
        ys.append(fixed + poly + rng.normal(0, 1, n))
    y = np.stack(ys, 1)
    return y[:, 0] if n_pheno == 1 else y


def covariates(n: int, n_extra: int = 2, seed: int = 2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.column_stack([np.ones(n), rng.normal(0, 1, (n, n_extra))])


def packed_records_device(n: int, p: int, miss_rate: float, seed: int,
                          device: str = "cuda") -> torch.Tensor:
    """(p, ceil(n/4)) packed .bed records generated directly in device memory.

    Same distribution as :func:`genotypes` (different random stream): used for
    benchmark-sized cohorts that would take minutes to draw on the host.
    """
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    bps = (n + 3) // 4
    out = torch.empty((p, bps), dtype=torch.uint8, device=device)
    step = max(1, (1 << 28) // max(n, 1))
    for s in range(0, p, step):
        e = min(p, s + step)
        af = torch.rand((e - s, 1), generator=gen, device=device, dtype=torch.float32) * 0.45 + 0.05
        u1 = torch.rand((e - s, bps * 4), generator=gen, device=device)
        u2 = torch.rand((e - s, bps * 4), generator=gen, device=device)
        cnt = (u1 < af).to(torch.uint8) + (u2 < af).to(torch.uint8)
        code = torch.where(cnt == 2, 0, torch.where(cnt == 1, 2, 3)).to(torch.uint8)
        if miss_rate > 0:
            miss = torch.rand((e - s, bps * 4), generator=gen, device=device) < miss_rate
            code = torch.where(miss, torch.ones_like(code), code)
        code[:, n:] = 3
        c = code.view(e - s, bps, 4)
        out[s:e] = c[:, :, 0] | (c[:, :, 1] << 2) | (c[:, :, 2] << 4) | (c[:, :, 3] << 6)
    return out
