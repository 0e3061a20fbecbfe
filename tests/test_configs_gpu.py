"""GPU parity at the named workload sizes.

Standalone wake FMM (1M ring + 100k background particles, core 0.02,
p = 4/6/8) and the dense solve (16,384-panel ellipsoid, 64 right-hand
sides).  Where the oracle cannot finish at full size in seconds, the check
uses a size-independent property or a seeded sample:

* FMM, 110k particles (ring + background, leaves <= 64): FP64 against the
  oracle at 1e-10 (relative L2, all particles); FP32C within 3e-6.
* FMM, 1.1M particles: the GPU direct sum is pinned to the oracle's direct
  sum on 256 seeded targets (1e-10); the FP64 FMM error against that direct
  sum on 4,096 targets falls with p; FP32C differs from FP64 FMM by < 3e-6.
* Dense, 16,384 panels: 24 seeded rows of the assembled matrix and
  right-hand side against the oracle (1e-10); LU64 and the mixed solve
  (FP32 LU, tensor-core trailing updates, FP64 refinement) reach a normwise
  backward error of 1e-12 on all 64 right-hand sides and agree to 1e-9.
"""
import numpy as np
import pytest

import oracle as O
from dust_b200 import abi, linsys, octree, synth

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 3e-6  # FP32C FMM (FP32 pair sums per tile, FP64 across tiles) vs FP64


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def ring110k():
    return synth.RingCase(n_ring=100_000, n_bg=10_000, seed=3)


@pytest.mark.parametrize("p", [4, 6])
def test_ring_110k_fp64_matches_oracle(ring110k, p):
    c = ring110k
    prm = c.fmm_params(p)
    ov, os_, orr, cnt = O.fmm_apply(prm, c.cen, c.dir, c.mag, c.r_vortex)
    oc = octree.initialize_octree(prm)
    v, s, r = oc.apply_multipole(c.cen, c.dir, c.mag, c.r_vortex)
    st = oc.stats()
    assert st["n_leaves"] == cnt[0] and st["n_active_cells"] == cnt[1]
    assert rel(v, ov) < TOL64 and rel(s, os_) < TOL64 and rel(r, orr) < TOL64
    prm32 = prm.replace(precision=abi.DUST_PREC_FP32C)
    v3, s3, r3 = octree.initialize_octree(prm32).apply_multipole(c.cen, c.dir, c.mag,
                                                                 c.r_vortex)
    assert rel(v3, ov) < TOL32 and rel(s3, os_) < TOL32 and rel(r3, orr) < TOL32


@pytest.fixture(scope="module")
def ring_full():
    c = synth.RingCase(seed=0)
    return c.permuted(c.truth_order(4096))


def test_ring_full_direct_sum_pinned(ring_full):
    c = ring_full
    prm = c.fmm_params(4)
    dv, ds, dr = O.direct_particles(prm, c.cen, c.dir, c.mag, c.r_vortex, n_tgt=256)
    gv, gs, gr = octree.direct_particles(prm, c.cen, c.dir, c.mag, c.r_vortex, n_tgt=256)
    assert rel(gv, dv) < TOL64 and rel(gs, ds) < TOL64 and rel(gr, dr) < TOL64


def test_ring_full_fmm_converges_and_fp32c(ring_full):
    c = ring_full
    nt = 4096
    tv, ts, _ = octree.direct_particles(c.fmm_params(4), c.cen, c.dir, c.mag, c.r_vortex,
                                        n_tgt=nt)
    errs = []
    for p in (4, 6, 8):
        prm = c.fmm_params(p)
        v, s, _ = octree.initialize_octree(prm).apply_multipole(c.cen, c.dir, c.mag,
                                                                c.r_vortex)
        errs.append((rel(v[:nt], tv), rel(s[:nt], ts)))
        if p == 4:
            prm32 = prm.replace(precision=abi.DUST_PREC_FP32C)
            v3, s3, _ = octree.initialize_octree(prm32).apply_multipole(c.cen, c.dir, c.mag,
                                                                        c.r_vortex)
            assert rel(v3, v) < TOL32 and rel(s3, s) < TOL32
    assert errs[1][0] < errs[0][0] and errs[2][0] < errs[1][0]
    assert errs[0][0] < 1e-3


@pytest.fixture(scope="module")
def ellipsoid16k():
    case = synth.EllipsoidCase(n_target=16384, nrhs=64, seed=0)
    n = case.n
    body = case.body
    rng = np.random.default_rng(4)
    body.uvort = rng.standard_normal((n, 3)) * 0.05
    prm = case.fmm_params().replace(u_inf=(1.0, 0.2, -0.1))
    ls = linsys.Linsys(prm, n, 0, body)
    ls.assemble_linsys(body)
    A, b = ls.get_system()
    ls.close()
    return case, prm, A, b


def test_ellipsoid_16k_rows_match_oracle(ellipsoid16k):
    case, prm, A, b = ellipsoid16k
    rows = np.sort(np.random.default_rng(7).choice(case.n, 24, replace=False))
    Ar, br = O.linsys_rows(prm, case.body, rows)
    assert rel(A[rows], Ar) < TOL64 and rel(b[rows], br) < TOL64
    # closed body: doublet rows sum to the full solid angle (4 pi)
    assert np.max(np.abs(A.sum(axis=1) - 4 * np.pi)) < 0.05 * 4 * np.pi


def test_ellipsoid_16k_64rhs_lu64_and_mixed(ellipsoid16k):
    import torch
    case, prm, A, b = ellipsoid16k
    n = case.n
    rng = np.random.default_rng(9)
    B = rng.standard_normal((n, 64)) * np.abs(b).max()
    Ad = torch.as_tensor(np.ascontiguousarray(A.T), device="cuda")
    Bd = torch.as_tensor(np.ascontiguousarray(B.T), device="cuda")
    X64, X32 = torch.empty_like(Bd), torch.empty_like(Bd)
    r64 = linsys.dense_solve_device(Ad, Bd, X64, abi.DUST_SOLVE_LU64)
    r32 = linsys.dense_solve_device(Ad, Bd, X32, abi.DUST_SOLVE_MIXED, tol=1e-12)
    assert r64["mode_used"] == abi.DUST_SOLVE_LU64
    assert r32["mode_used"] == abi.DUST_SOLVE_MIXED and r32["residual"] <= 1e-12
    # the doublet system needs no interchange, and the factors certify it
    assert r64["pivoted"] == 0 and r32["pivoted"] == 0
    Anorm = float(Ad.abs().sum(dim=0).max())

    def berr(X):
        R = Bd - X @ Ad
        return float((R.abs().amax(dim=1) / (Anorm * X.abs().amax(dim=1))).max())
    assert berr(X64) <= 1e-12 and berr(X32) <= 1e-12
    assert float(torch.linalg.norm(X32 - X64) / torch.linalg.norm(X64)) < 1e-9
    # the device entry point leaves A as it was (a second solve agrees)
    X2 = torch.empty_like(Bd)
    linsys.dense_solve_device(Ad, Bd, X2, abi.DUST_SOLVE_LU64)
    assert torch.equal(X2, X64)
