"""FP64 scipy restatement of the event likelihood of example_full.jl:338-449
(poisson_dist_per_module, shape_mixture_per_module,
extended_llh_per_module).  TEST INFRASTRUCTURE ONLY: the checker of the
library's event-likelihood kernel."""
from __future__ import annotations

import numpy as np
from scipy import special, stats


def module_llh(params, x, photons=None, mode="shifted"):
    """params [n_sources, 6] (A, w, a1, a2, theta, shift) of one module; x the
    module's hit times."""
    p = np.asarray(params, dtype=np.float64)
    A, w, a1, a2, th, sh = p.T
    n_src = np.ones(len(p)) if photons is None else np.asarray(photons, dtype=np.float64)
    mu = float(np.sum(A * n_src))
    q = A / A.sum() if mode == "reference" else A * n_src / mu
    n = len(x)
    pois = stats.poisson.logpmf(n, mu) if n else -mu
    if n == 0:
        return pois
    y = np.asarray(x, dtype=np.float64)[:, None] - sh[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        g1 = np.where(y > 0, stats.gamma.pdf(np.maximum(y, 1e-300), a1, scale=th), 0.0)
        g2 = np.where((y > 0) & (a2 > 0), stats.gamma.pdf(np.maximum(y, 1e-300), np.where(a2 > 0, a2, 1.0),
                                                             scale=th), 0.0)
    f = np.sum(q * (w * g1 + (1 - w) * g2), axis=1)
    return pois + float(np.sum(np.log(f)))


def poisson_logpmf(n, mu):
    return n * np.log(mu) - mu - special.gammaln(n + 1)
