"""The FP32 Hex8 operator with two element rows per thread (k_matvec_h8p,
switch hex8_pair) against the one-row FP32 kernel (the default) and the FP64
operator, on grids that end inside, at and just past tile boundaries in every
axis.

Bars: 1e-5 of max |Ku| against FP64 (FP32 arithmetic), 1e-5 against the
one-row FP32 kernel (same products, different association), and every SoA
padding entry left as it was (the kernel writes only live nodes).
"""
import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n", [("cantilever3d", (1, 1, 1)), ("cantilever3d", (2, 3, 1)),
                                    ("cantilever3d", (30, 6, 3)), ("halfmbb3d", (31, 7, 4)),
                                    ("cantilever3d", (5, 4, 3)), ("halfmbb3d", (30, 14, 4)),
                                    ("cantilever3d", (31, 15, 2)), ("cantilever3d", (32, 16, 5)),
                                    ("halfmbb3d", (62, 30, 3)), ("cantilever3d", (70, 40, 10)),
                                    ("cantilever3d", (96, 32, 32))])
def test_paired_fp32_operator_matches(ctx, kind, n):
    import torch
    g = cases.build_gpu(ctx, kind, *n)
    g.set_density(cases.uniform_density(g.nel, 17))
    ns = g.soa_length()
    ld = ns // 3
    live = torch.zeros(ns, dtype=torch.bool, device="cuda")
    for c in range(3):
        live[c * ld:c * ld + g.nnode] = True
    x64 = torch.randn(ns, dtype=torch.float64, device="cuda")
    x32 = x64.float()
    y64 = torch.zeros_like(x64)
    ypair = torch.full_like(x32, 3.0)
    yrow = torch.full_like(x32, 3.0)
    torch.cuda.synchronize()
    g.operator_apply_device(x64.data_ptr(), y64.data_ptr(), icb.FP64)
    g.operator_apply_device(x32.data_ptr(), yrow.data_ptr(), icb.MIXED)
    old = icb.get_option("hex8_pair")
    icb.set_option("hex8_pair", 1)
    try:
        g.operator_apply_device(x32.data_ptr(), ypair.data_ptr(), icb.MIXED)
    finally:
        icb.set_option("hex8_pair", old)
    g.ctx.synchronize()
    a = y64[live].cpu().numpy()
    p = ypair[live].double().cpu().numpy()
    r = yrow[live].double().cpu().numpy()
    scale = np.abs(a).max()
    assert np.abs(p - a).max() <= 1e-5 * scale
    assert np.abs(p - r).max() <= 1e-5 * scale
    assert bool((ypair[~live] == 3.0).all())
