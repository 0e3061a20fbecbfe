"""Learned preconditioner on the GPU.

* The gradient of the library's hand-written backward kernels against the
  CPU oracle (oracle/gnn_oracle.py) on a stored moving-body system, with
  random weights (nonzero output weights so every layer gets gradient):
  loss within 1e-4 relative, gradient within 2e-3 (L2, relative; FP32 and
  atomic accumulation order).
* Training on systems of a rotating rotor over a fuselage (the plain LU
  solves them) lowers the loss, and on azimuths not seen in training the
  GMRES with the trained network needs fewer iterations than with the
  untrained one (Jacobi), with solutions equal to LU's within 1e-9.
* Without a network attached the GMRES mode falls back to LU.
"""
import numpy as np
import pytest

import gnn_oracle as G
from dust_b200 import abi, linsys, precond, synth
from dust_b200.params import FmmParams

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _system(phase, n_fus=600, n_span=10, n_chord=4):
    els, nst = synth.rotor_fuselage(n_fus=n_fus, n_span=n_span, n_chord=n_chord, phase=phase)
    return els, nst


PRM = FmmParams(u_inf=(2.0, 0.0, -1.0), rankine_rad=0.1)


def _solve_lu(ls, els):
    ls.assemble_linsys(els)
    x, _ = ls.solve_linsys(abi.DUST_SOLVE_LU64)
    return x


def test_gnn_gradient_matches_oracle():
    els, nst = _system(0.1, n_fus=300, n_span=6, n_chord=3)
    ls = linsys.initialize_linsys(PRM, els.n, nst, els)
    x = _solve_lu(ls, els)
    ls.assemble_linsys(els)
    pc = precond.Precond(els.ver.mean(axis=1), k=8, seed=1)
    pc.add_sample(ls, x, seed=5)
    rng = np.random.default_rng(2)
    p = (rng.standard_normal(pc.num_params()) * 0.15).astype(np.float32)
    pc.set_params(p)
    loss, g = pc.loss_grad(0)
    xs, ef, w, nbr, Y, T = pc.get_sample(0)
    lo, go = G.loss_grad(p.astype(np.float64), xs.astype(np.float64), ef.astype(np.float64),
                         w.astype(np.float64), nbr.astype(np.int64), Y.astype(np.float64),
                         T.astype(np.float64))
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    assert rel(g.astype(np.float64), go) < 2e-3
    # the sample's columns: M b targets the solution, M A z the probe
    assert np.allclose(T[:, -1], x.astype(np.float32))


def test_trained_preconditioner_beats_jacobi():
    train_phases = np.linspace(0.0, np.pi / 2, 10, endpoint=False)
    test_phases = [0.05, 0.52, 1.31]
    els0, nst = _system(0.0)
    ls = linsys.initialize_linsys(PRM, els0.n, nst, els0)
    pc = precond.Precond(els0.ver.mean(axis=1), k=8, seed=3)
    for q, ph in enumerate(train_phases):
        els, _ = _system(ph)
        x = _solve_lu(ls, els)
        ls.assemble_linsys(els)
        pc.add_sample(ls, x, seed=100 + q)
    l0 = np.mean([pc.loss_grad(i, with_grad=False)[0] for i in range(pc.num_samples)])
    l1 = pc.train(600, lr=2e-3)
    assert l1 < 0.7 * l0
    untrained = precond.Precond(els0.ver.mean(axis=1), k=8, seed=3)
    its = {}
    for name, p in (("jacobi", untrained), ("trained", pc)):
        p.attach(ls)
        its[name] = []
        for ph in test_phases:
            els, _ = _system(ph)
            xl = _solve_lu(ls, els)
            ls.assemble_linsys(els)
            xg, rep = ls.solve_linsys(abi.DUST_SOLVE_GMRES_NN)
            assert rep["mode_used"] == abi.DUST_SOLVE_GMRES_NN and rep["fell_back"] == 0
            assert rep["residual"] <= 1e-11
            assert rel(xg, xl) < 1e-9
            its[name].append(rep["iterations"])
    assert sum(its["trained"]) < sum(its["jacobi"]), its


def test_gmres_without_network_falls_back_to_lu():
    els, nst = _system(0.3, n_fus=300, n_span=6, n_chord=3)
    ls = linsys.initialize_linsys(PRM, els.n, nst, els)
    xl = _solve_lu(ls, els)
    ls.assemble_linsys(els)
    xg, rep = ls.solve_linsys(abi.DUST_SOLVE_GMRES_NN)
    assert rep["fell_back"] == 1 and rep["mode_used"] == abi.DUST_SOLVE_LU64
    assert rel(xg, xl) < 1e-12
