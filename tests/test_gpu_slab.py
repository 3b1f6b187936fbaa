"""The slab-partitioned solve's device path (icarat_b200.slab with the
library's operator on each slab's icb_problem) on one GPU: the one-rank
partition reproduces the library's FP64 Jacobi-PCG (icb_solve, Eigen_CG
semantics) -- its iteration count to within one and its compliance to 1e-10
-- and the oracle's compliance to 1e-8.  The exchange and the collectives
are covered on CPU ranks by test_slab.py; runs over several GPUs (NCCL) are
not covered here (one GPU per test box).

The multigrid form (slab.SlabMg with the library's operator on the fine
slab and torch element sums on the coarse levels) on one rank reproduces
the library's FP64 GMG-PCG (icb_solve with ICB_GMG): the same hierarchy,
smoother and flexible CG, so the iteration count to within one and the
compliance to 1e-10."""
import numpy as np
import pytest

import cases
import icarat_b200 as icb
from icarat_b200 import slab

pytestmark = pytest.mark.gpu


def test_one_rank_slab_solve_matches_library_solve(ctx):
    import torch
    nx, ny, nz = 40, 12, 10
    L = slab.SlabLayout(nx, ny, nz, 0, 1)
    fixed, f = cases.masks("cantilever3d", nx, ny, nz)
    to4 = lambda a: np.ascontiguousarray(  # noqa: E731
        a.reshape(nz + 1, ny + 1, nx + 1, 3).transpose(3, 0, 1, 2))
    rho = cases.uniform_density(nx * ny * nz, 8)
    prob, op, b, diag, free = slab.gpu_slab(ctx, L, to4(fixed), to4(f),
                                            rho.reshape(nz, ny, nx))
    ex = slab.Exchange(L, None, device=b.device)
    x, info = slab.slab_jacobi_pcg(L, ex, op, b, diag, free, 1e-8, 100000)
    assert info["status"] == 0 and info["relres"] <= 1e-8
    (c,) = ex.allreduce([slab.owned_dot(L, x, b)])
    g = cases.build_gpu(ctx, "cantilever3d", nx, ny, nz)
    g.set_density(rho)
    ref = g.solve(tol=1e-8, maxit=100000)
    assert abs(info["iters"] - ref["iters"]) <= 1, (info, ref["iters"])
    assert abs(c - g.compliance()) <= 1e-10 * abs(g.compliance())
    o = cases.build_oracle("cantilever3d", nx, ny, nz)
    ro = o.solve(rho, tol=1e-10)
    assert abs(c - ro["compliance"]) <= 1e-8 * abs(ro["compliance"])
    torch.cuda.synchronize()
    prob.close()
    g.close()


def test_one_rank_slab_multigrid_matches_library_gmg(ctx):
    import torch
    nx, ny, nz = 40, 12, 10
    L = slab.SlabLayout(nx, ny, nz, 0, 1)
    fixed, f = cases.masks("cantilever3d", nx, ny, nz)
    to4 = lambda a: np.ascontiguousarray(  # noqa: E731
        a.reshape(nz + 1, ny + 1, nx + 1, 3).transpose(3, 0, 1, 2))
    rho = cases.uniform_density(nx * ny * nz, 8)
    prob, op, b, diag, free = slab.gpu_slab(ctx, L, to4(fixed), to4(f),
                                            rho.reshape(nz, ny, nx))
    E = torch.from_numpy(cases.EMIN + rho.reshape(nz, ny, nx) ** cases.PENAL *
                         (cases.E0 - cases.EMIN)).to(b.device)
    units = []

    def kmat(h):
        u = icb.Problem(ctx, 3, 1, 1, 1, lx=h[0], ly=h[1], lz=h[2], nu=cases.NU)
        units.append(u)
        return u.K0()

    ex = slab.Exchange(L, None, device=b.device)
    mg = slab.SlabMg(ex, op, diag, free, E, kmat)
    x, info = slab.slab_gmg_pcg(mg, b, 1e-8, 1000)
    assert info["status"] == 0 and info["relres"] <= 1e-8
    (c,) = ex.allreduce([slab.owned_dot(L, x, b)])
    g = cases.build_gpu(ctx, "cantilever3d", nx, ny, nz)
    g.set_density(rho)
    ref = g.solve(precision=icb.FP64, precond=icb.GMG, tol=1e-8, maxit=1000)
    assert info["levels"] >= 3
    assert abs(info["iters"] - ref["iters"]) <= 1, (info, ref["iters"])
    assert abs(c - g.compliance()) <= 1e-10 * abs(g.compliance())
    torch.cuda.synchronize()
    for u in units:
        u.close()
    prob.close()
    g.close()
