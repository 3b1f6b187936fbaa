"""The tensor-core (tcgen05, TF32) Hex8 operator against the FP64 operator and
inside the mixed-precision multigrid solve.

Bars: the operator product within 3e-3 of the FP64 product (L-inf relative
to max |Ku|; TF32 keeps 10 mantissa bits); the mixed solve with the
tensor-core V-cycle reaches ||r||/||f|| <= 1e-8 in FP64 with the usual
compliance (1e-6) and sensitivity (1e-5) bars; no tensor-core wait timed out.
"""
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
    x64 = torch.randn(ns, dtype=torch.float64, device="cuda")
    y64 = torch.zeros_like(x64)
    g.operator_apply_device(x64.data_ptr(), y64.data_ptr(), icb.FP64)
    x32 = x64.float()
    y32 = torch.full_like(x32, 3.0)  # every live entry must be overwritten
    ysimt = torch.zeros_like(x32)
    g.operator_apply_device(x32.data_ptr(), y32.data_ptr(), icb.TF32)
    g.operator_apply_device(x32.data_ptr(), ysimt.data_ptr(), icb.MIXED)
    torch.cuda.synchronize()
    assert icb.get_option("tc_timeouts") == 0
    ld = ns // 3
    live = torch.zeros(ns, dtype=torch.bool, device="cuda")
    for c in range(3):
        live[c * ld:c * ld + g.nnode] = True
    a, b, s = y64[live].cpu().numpy(), y32[live].double().cpu().numpy(), ysimt[live].double().cpu().numpy()
    scale = np.abs(a).max()
    assert np.abs(s - a).max() <= 1e-5 * scale  # FP32 CUDA cores
    assert np.abs(b - a).max() <= 3e-3 * scale  # TF32 tensor cores


@pytest.mark.parametrize("kind,n,seed", [("cantilever3d", (24, 8, 8), 3), ("halfmbb3d", (16, 8, 8), 4),
                                         ("cantilever3d", (19, 7, 9), 5)])
def test_mixed_solve_with_tc_vcycle(ctx, kind, n, seed):
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, seed)
    ro = o.solve(rho, tol=1e-12)
    dco = o.sensitivity(rho, ro["nodeval"])
    g.set_density(rho)
    icb.set_option("tc_operator", 1)
    try:
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8, maxit=20000)
    finally:
        icb.set_option("tc_operator", 0)
    assert info["true_relres"] <= 2e-8, info
    assert abs(g.compliance() - ro["compliance"]) <= 1e-6 * abs(ro["compliance"])
    assert np.abs(g.sensitivity() - dco).max() <= 1e-5 * np.abs(dco).max()
    assert icb.get_option("tc_timeouts") == 0
