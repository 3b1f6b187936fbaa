"""icb_solve_noalloc: the Jacobi-PCG solve for callers that cannot allocate
device memory (hosts that own all GPU memory through their own pool, serving
loops that must not touch the allocator).

It must give the same displacement as the allocating entry point
(icb_solve, FP64 Jacobi), within the parity bars the other tests use, on
consecutive calls that share its static scratch array.  This file is named
to be collected last so a stop-at-first-failure run has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu

U_RTOL = 1e-5            # displacement, L-inf relative to max |u| (as the parity tests)
COMPLIANCE_RTOL = 1e-6


def _soa(prob, numeq_vec, fill=0.0):
    """numeq vector -> device SoA vector (component c of node n at c*ld + n);
    the constrained slots and the padding past each component's last node
    hold `fill`."""
    import torch
    n = prob.soa_length()
    ld = n // prob.dim
    dof = prob.dof_map()
    h = np.full(n, fill)
    nodes = np.arange(prob.nnode)
    for c in range(prob.dim):
        d = dof[nodes * prob.dim + c]
        free = d < prob.numeq
        h[c * ld + nodes[free]] = numeq_vec[d[free]]
    return torch.from_numpy(h).cuda()


def _numeq(prob, soa_t):
    h = soa_t.cpu().numpy()
    ld = h.size // prob.dim
    dof = prob.dof_map()
    u = np.zeros(prob.numeq)
    nodes = np.arange(prob.nnode)
    for c in range(prob.dim):
        d = dof[nodes * prob.dim + c]
        free = d < prob.numeq
        u[d[free]] = h[c * ld + nodes[free]]
    return u


def _noalloc(prob, b, x, tol=1e-10, maxit=20000):
    info = icb.SolveInfo()
    rc = icb.lib().icb_solve_noalloc(prob.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()),
                                     tol, maxit, C.byref(info))
    return rc, info


@pytest.mark.parametrize("kind,n", [("cantilever2d", (120, 40)), ("cantilever3d", (24, 8, 8))])
def test_noalloc_matches_solve_on_consecutive_calls(ctx, kind, n):
    import torch
    g = cases.build_gpu(ctx, kind, *n)
    assert g.soa_length() <= icb.lib().icb_noalloc_max_soa()
    f = g.load()
    # the second call's b holds NaN in its constrained and padding slots,
    # which the solve must ignore
    for seed, fill in ((11, 0.0), (12, np.nan)):  # two calls in a row on the shared scratch
        b = _soa(g, f, fill)
        rho = cases.uniform_density(g.nel, seed)
        g.set_density(rho)
        ref = g.solve(tol=1e-10, maxit=20000)
        u_ref = g.displacement()
        x = torch.full((g.soa_length(),), 7.0, dtype=torch.float64, device="cuda")
        # b and x were written on torch's stream; the library solves on its own
        torch.cuda.synchronize()
        rc, info = _noalloc(g, b, x)
        torch.cuda.synchronize()
        assert rc == 0, icb.lib().icb_last_error().decode()
        u = _numeq(g, x)
        assert np.abs(u - u_ref).max() <= U_RTOL * np.abs(u_ref).max()
        assert abs(u @ f - u_ref @ f) <= COMPLIANCE_RTOL * abs(u_ref @ f)
        assert info.relres <= 1e-10 and abs(info.iters - ref["iters"]) <= 2


def test_noalloc_rejects_problems_beyond_its_limit(ctx):
    import torch
    lim = icb.lib().icb_noalloc_max_soa()
    g = cases.build_gpu(ctx, "cantilever3d", 128, 64, 64)
    assert g.soa_length() > lim
    g.set_density(np.full(g.nel, 0.5))
    b = torch.zeros(g.soa_length(), dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    rc, _ = _noalloc(g, b, x)
    assert rc == -1  # ICB_ERR_BAD_ARG
    assert "exceeds the static scratch limit" in icb.lib().icb_last_error().decode()
