"""The CPU oracle of the learned preconditioner's network: its hand-written
gradient against central finite differences (float64), on a random graph
with nonzero output weights so that every layer receives gradient."""
import numpy as np

import gnn_oracle as G


def _random_case(n=40, K=6, C=8, seed=0):
    rng = np.random.default_rng(seed)
    nbr = np.empty((n, K), dtype=np.int64)
    for i in range(n):
        nbr[i, 0] = i
        nbr[i, 1:] = rng.choice([j for j in range(n) if j != i], K - 1, replace=False)
    x = rng.standard_normal((n, G.FIN))
    ef = rng.standard_normal((n, K, G.EF))
    w = rng.random((n, K))
    w[:, 0] = 0.0
    w /= w.sum(1, keepdims=True)
    Y = rng.standard_normal((n, C))
    T = rng.standard_normal((n, C))
    p = rng.standard_normal(G.n_params()) * 0.2
    return p, x, ef, w, nbr, Y, T


def test_oracle_gradient_matches_finite_differences():
    p, x, ef, w, nbr, Y, T = _random_case()
    loss, g = G.loss_grad(p, x, ef, w, nbr, Y, T)
    assert np.isclose(loss, G.loss_only(p, x, ef, w, nbr, Y, T), rtol=1e-14)
    rng = np.random.default_rng(1)
    # every parameter block: W0, b0, each layer's Ws Wn b, u, c
    idx = np.concatenate([rng.choice(G.n_params() - 68, 60, replace=False),
                          np.arange(G.n_params() - 68, G.n_params())])
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (G.loss_only(pp, x, ef, w, nbr, Y, T) - G.loss_only(pm, x, ef, w, nbr, Y, T)) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_untrained_output_is_jacobi():
    p, x, ef, w, nbr, Y, T = _random_case(seed=3)
    p[-(G.H + G.EF):] = 0.0  # u = 0, c = 0
    o, _ = G.forward(p, x, ef, w, nbr)
    assert np.all(o == 0.0)
    dinv = np.linspace(0.5, 2.0, nbr.shape[0])
    v = np.arange(nbr.shape[0], dtype=np.float64)
    assert np.allclose(G.apply_precond(o, dinv, nbr, v), dinv * v)
