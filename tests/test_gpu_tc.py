"""The tensor-core (tcgen05, TF32) Hex8 operator against the FP64 operator and
inside the mixed-precision multigrid solve.

Bars: the operator product within 3e-3 of the FP64 product and of the
oracle's assembled matrix (L-inf relative to max |Ku|; TF32 keeps 10
mantissa bits); the mixed solve with the tensor-core V-cycle reaches
||r||/||f|| <= 1e-8 in FP64 with the usual compliance (1e-6) and sensitivity
(1e-5) bars; no tensor-core wait timed out, and a wait that is made to run
out returns ICB_ERR_TIMEOUT without harming the next call.
"""
TF32_RTOL = 3e-3
ICB_ERR_TIMEOUT = -5
import numpy as np
import pytest

import cases
import icarat_b200 as icb
import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n", [("cantilever3d", (9, 5, 4)), ("cantilever3d", (40, 9, 17)),
                                    ("halfmbb3d", (33, 14, 6)), ("cantilever3d", (96, 32, 32))])
def test_tc_operator_matches_fp64(ctx, kind, n):
    import torch
    g = cases.build_gpu(ctx, kind, *n)
    g.set_density(cases.uniform_density(g.nel, 7))
    ns = g.soa_length()
    t0 = icb.get_option("tc_timeouts")
    x64 = torch.randn(ns, dtype=torch.float64, device="cuda")
    y64 = torch.zeros_like(x64)
    x32 = x64.float()
    y32 = torch.full_like(x32, 3.0)  # every live entry must be overwritten
    ysimt = torch.zeros_like(x32)
    torch.cuda.synchronize()  # written on torch's stream; the library uses its own
    g.operator_apply_device(x64.data_ptr(), y64.data_ptr(), icb.FP64)
    g.operator_apply_device(x32.data_ptr(), y32.data_ptr(), icb.TF32)
    g.operator_apply_device(x32.data_ptr(), ysimt.data_ptr(), icb.MIXED)
    g.ctx.synchronize()
    assert icb.get_option("tc_timeouts") == t0
    ld = ns // 3
    live = torch.zeros(ns, dtype=torch.bool, device="cuda")
    for c in range(3):
        live[c * ld:c * ld + g.nnode] = True
    a, b, s = y64[live].cpu().numpy(), y32[live].double().cpu().numpy(), ysimt[live].double().cpu().numpy()
    scale = np.abs(a).max()
    assert np.abs(s - a).max() <= 1e-5 * scale  # FP32 CUDA cores
    assert np.abs(b - a).max() <= TF32_RTOL * scale  # TF32 tensor cores


def _soa_from_numeq(g, v):
    ns = g.soa_length()
    ld = ns // g.dim
    dof = g.dof_map()
    h = np.zeros(ns)
    nodes = np.arange(g.nnode)
    for c in range(g.dim):
        d = dof[nodes * g.dim + c]
        free = d < g.numeq
        h[c * ld + nodes[free]] = v[d[free]]
    return h, dof, ld


@pytest.mark.parametrize("kind,n,seed", [("cantilever3d", (24, 8, 8), 5), ("halfmbb3d", (33, 14, 6), 6)])
def test_tc_operator_matches_oracle_assembled(ctx, kind, n, seed):
    """The tensor-core product against the oracle's assembled stiffness matrix
    (LinearElastic::makeKeFint + assembling, elasticity.cpp:210-254,
    assembling.hpp:17-38) on the free DOFs."""
    import scipy.sparse as sp
    import torch
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, seed)
    g.set_density(rho)
    rp, col, val = o.assemble(rho)
    A = sp.csr_matrix((val, col, rp), shape=(g.numeq,) * 2)
    xq = np.random.default_rng(seed).standard_normal(g.numeq)
    yo = A @ xq
    h, dof, ld = _soa_from_numeq(g, xq)
    x32 = torch.from_numpy(h).float().cuda()
    y32 = torch.full_like(x32, 3.0)
    t0 = icb.get_option("tc_timeouts")
    torch.cuda.synchronize()
    g.operator_apply_device(x32.data_ptr(), y32.data_ptr(), icb.TF32)
    g.ctx.synchronize()
    assert icb.get_option("tc_timeouts") == t0
    yh = y32.double().cpu().numpy()
    y = np.zeros(g.numeq)
    nodes = np.arange(g.nnode)
    for c in range(g.dim):
        d = dof[nodes * g.dim + c]
        free = d < g.numeq
        y[d[free]] = yh[c * ld + nodes[free]]
    assert np.abs(y - yo).max() <= TF32_RTOL * np.abs(yo).max()


@pytest.mark.parametrize("kind,n,seed", [("cantilever3d", (24, 8, 8), 3), ("halfmbb3d", (16, 8, 8), 4),
                                         ("cantilever3d", (19, 7, 9), 5)])
def test_mixed_solve_with_tc_vcycle(ctx, kind, n, seed):
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, seed)
    ro = o.solve(rho, tol=1e-12)
    dco = o.sensitivity(rho, ro["nodeval"])
    g.set_density(rho)
    t0 = icb.get_option("tc_timeouts")
    icb.set_option("tc_operator", 1)
    try:
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8, maxit=20000)
    finally:
        icb.set_option("tc_operator", 0)
    assert info["true_relres"] <= 2e-8, info
    assert abs(g.compliance() - ro["compliance"]) <= 1e-6 * abs(ro["compliance"])
    assert np.abs(g.sensitivity() - dco).max() <= 1e-5 * np.abs(dco).max()
    assert icb.get_option("tc_timeouts") == t0


def test_tc_wait_that_runs_out_reports_timeout_and_recovers(ctx):
    """Every tensor-core MMA wait is bounded.  With the limit set to 0 polls
    each wait gives up at once: the CTA still lets the MMAs it issued finish
    (a second bounded wait), frees its tensor memory and returns; the timeouts
    are counted and the call returns ICB_ERR_TIMEOUT, for the operator and for
    a mixed solve with the tensor-core V-cycle.  With the default limit back,
    the next product and solve are correct."""
    import ctypes as C
    import torch
    kind, n = "cantilever3d", (24, 8, 8)
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, 9)
    g.set_density(rho)
    ns = g.soa_length()
    x32 = torch.randn(ns, dtype=torch.float32, device="cuda")
    y32 = torch.zeros_like(x32)
    torch.cuda.synchronize()
    default = icb.get_option("tc_spin_limit")
    assert default > 0
    t0 = icb.get_option("tc_timeouts")
    icb.set_option("tc_spin_limit", 0)
    try:
        rc = icb.lib().icb_operator_apply_device(g.h, icb.TF32, C.c_void_p(x32.data_ptr()),
                                                 C.c_void_p(y32.data_ptr()))
        t1 = icb.get_option("tc_timeouts")
        icb.set_option("tc_operator", 1)
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8, maxit=20,
                       raise_on_error=False)
    finally:
        icb.set_option("tc_operator", 0)
        icb.set_option("tc_spin_limit", default)
    assert rc == ICB_ERR_TIMEOUT
    assert t1 > t0
    assert info["rc"] == ICB_ERR_TIMEOUT and icb.get_option("tc_timeouts") > t1
    # the context is intact: a normal product and a tensor-core solve are correct
    t2 = icb.get_option("tc_timeouts")
    y64 = torch.zeros(ns, dtype=torch.float64, device="cuda")
    x64 = x32.double()
    torch.cuda.synchronize()
    g.operator_apply_device(x64.data_ptr(), y64.data_ptr(), icb.FP64)
    g.operator_apply_device(x32.data_ptr(), y32.data_ptr(), icb.TF32)
    g.ctx.synchronize()
    a, b = y64.cpu().numpy(), y32.double().cpu().numpy()
    assert np.abs(b - a).max() <= TF32_RTOL * np.abs(a).max()
    ro = o.solve(rho, tol=1e-12)
    icb.set_option("tc_operator", 1)
    try:
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8, maxit=20000)
    finally:
        icb.set_option("tc_operator", 0)
    assert info["true_relres"] <= 2e-8
    assert abs(g.compliance() - ro["compliance"]) <= 1e-6 * abs(ro["compliance"])
    assert icb.get_option("tc_timeouts") == t2
