"""Parity at the full sizes of the benchmark configurations.

* The 192x64x64 Hex8 cantilever (2,446,275 DOF, densities U[0.01,1] from seed
  2024): every solver against the oracle's LinearAnalysis::solve restatement
  (assembled CSR + Eigen_CG-semantics Jacobi-PCG, src/analysis/linear.hpp:54-104,
  src/analysis/solver/solvers.cpp:64-92), whose outputs tests/golden/make_fullsize.py
  stored in tests/golden/c2_fullsize.npz: compliance within 1e-6 relative,
  sensitivities within 1e-5 of max |dc| (L-inf over the stored entries: a fixed
  stride plus the largest), displacements within 1e-5 of max |u|, all at
  ||r||/||f|| <= 1e-8; the FP64 Jacobi-PCG takes the oracle's iteration count.
* The 384x128x128 Hex8 half-MBB beam (19,220,355 DOF, seeded smooth density
  field): the mixed-precision solves against the FP64 GMG solve of the same
  system (an assembled CPU solve of this grid needs ~77 GB), the energy identity
  f.u = u.K u and the sign of every sensitivity.
"""
import os

import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_fullsize.npz")
COMPLIANCE_RTOL, SENS_RTOL, U_RTOL = 1e-6, 1e-5, 1e-5


@pytest.fixture(scope="module")
def c2(ctx):
    F = np.load(GOLD)
    g = cases.build_gpu(ctx, "cantilever3d", *F["grid"])
    rho = cases.uniform_density(g.nel, int(F["seed"]))
    g.set_density(rho)
    yield g, F
    g.close()


@pytest.mark.parametrize("precision,precond", [(icb.FP64, icb.JACOBI), (icb.FP64, icb.GMG),
                                               (icb.MIXED, icb.GMG), (icb.MIXED_REFINE, icb.GMG)])
def test_c2_full_size_matches_oracle(c2, precision, precond):
    g, F = c2
    assert g.numeq == int(F["numeq"])
    info = g.solve(precision=precision, precond=precond, tol=1e-8, maxit=200000)
    assert info["true_relres"] <= 2e-8, info
    c = g.compliance()
    assert abs(c - float(F["compliance"])) <= COMPLIANCE_RTOL * abs(float(F["compliance"]))
    dc = g.sensitivity()
    assert abs(np.abs(dc).max() - float(F["dc_absmax"])) <= SENS_RTOL * float(F["dc_absmax"])
    assert np.abs(dc[F["dc_idx"]] - F["dc"]).max() <= SENS_RTOL * float(F["dc_absmax"])
    u = g.displacement()
    assert np.abs(u[F["u_idx"]] - F["u"]).max() <= U_RTOL * float(F["u_absmax"])
    if precond == icb.JACOBI:
        # the same algorithm at the same tolerance: the oracle's iteration count
        it = int(F["iters_1e8"])
        assert abs(info["iters"] - it) <= max(3, 0.02 * it), (info["iters"], it)


def test_c3_full_size_mixed_matches_fp64(ctx):
    n = (384, 128, 128)
    g = cases.build_gpu(ctx, "halfmbb3d", *n)
    rho = cases.smooth_field(*n, seed=2024)
    g.set_density(rho)
    i64 = g.solve(precision=icb.FP64, precond=icb.GMG, tol=1e-8, maxit=20000)
    assert i64["true_relres"] <= 2e-8, i64
    c64, dc64 = g.compliance(), g.sensitivity()
    u64 = g.displacement()
    assert abs(c64 - u64 @ g.matvec(u64)) <= 1e-7 * c64  # f.u = u.K u at convergence
    assert (dc64 <= 0).all()
    for prec in (icb.MIXED, icb.MIXED_REFINE):
        info = g.solve(precision=prec, precond=icb.GMG, tol=1e-8, maxit=20000)
        assert info["true_relres"] <= 2e-8, (prec, info)
        assert abs(g.compliance() - c64) <= COMPLIANCE_RTOL * c64, prec
        assert np.abs(g.sensitivity() - dc64).max() <= SENS_RTOL * np.abs(dc64).max(), prec
        u = g.displacement()
        assert np.abs(u - u64).max() <= U_RTOL * np.abs(u64).max(), prec
    g.close()
