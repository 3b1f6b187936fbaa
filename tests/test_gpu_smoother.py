"""icb_smoother_apply_device: one Chebyshev step of the V-cycle with the
operator and its update fused, y <- u + c2 D^-1 (b - K u) + c1 (u - y), in
FP64 and FP32, against a torch FP64 restatement of the same formula built on
the FP64 operator (itself checked against the oracle's assembled matrix in
test_gpu_parity.py).

Bars: FP64 1e-12 of max |y| (the kernel fuses multiplies and adds the
restatement rounds separately); FP32 1e-5 (FP32 arithmetic); SoA padding
left as it was; c1 = 0 does not read y.
"""
import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n", [("cantilever3d", (5, 4, 3)), ("halfmbb3d", (31, 7, 4)),
                                    ("cantilever3d", (33, 17, 9)), ("halfmbb2d", (40, 16)),
                                    ("cantilever2d", (61, 30))])
@pytest.mark.parametrize("c1", [0.0, 0.35])
def test_smoother_step_matches_formula(ctx, kind, n, c1):
    import torch
    g = cases.build_gpu(ctx, kind, *n)
    g.set_density(cases.uniform_density(g.nel, 23))
    ns = g.soa_length()
    dim = 3 if len(n) == 3 else 2
    ld = ns // dim
    live = torch.zeros(ns, dtype=torch.bool, device="cuda")
    for c in range(dim):
        live[c * ld:c * ld + g.nnode] = True
    gen = torch.Generator(device="cuda").manual_seed(5)
    u = torch.randn(ns, dtype=torch.float64, device="cuda", generator=gen)
    b = torch.randn(ns, dtype=torch.float64, device="cuda", generator=gen)
    y0 = torch.randn(ns, dtype=torch.float64, device="cuda", generator=gen)
    dinv = torch.rand(ns, dtype=torch.float64, device="cuda", generator=gen) + 0.5
    # the V-cycle's vectors are 0 on padding and dinv is 0 on constrained DOFs
    Au = torch.zeros_like(u)
    torch.cuda.synchronize()
    g.operator_apply_device(u.data_ptr(), Au.data_ptr(), icb.FP64)
    g.ctx.synchronize()
    fixed = (Au == 0) & live  # constrained rows of K u are exactly 0
    dinv[fixed] = 0.0
    dinv[~live] = 0.0
    c2 = 0.8
    ref = u + c2 * dinv * (b - Au) + (c1 * (u - y0) if c1 != 0.0 else 0.0)
    scale = ref[live].abs().max().item()
    for prec, dt, tol in ((icb.FP64, torch.float64, 1e-12), (icb.MIXED, torch.float32, 1e-5)):
        uu, bb, dd = u.to(dt), b.to(dt), dinv.to(dt)
        y = y0.to(dt).clone()
        y[~live] = 7.0
        if c1 == 0.0:
            y[live] = float("nan")  # not read
        torch.cuda.synchronize()
        g.smoother_apply_device(uu.data_ptr(), y.data_ptr(), bb.data_ptr(), dd.data_ptr(), c1, c2,
                                precision=prec)
        g.ctx.synchronize()
        err = (y[live].double() - ref[live]).abs().max().item()
        assert err <= tol * scale, (prec, err, scale)
        assert bool((y[~live] == 7.0).all())


def test_smoother_rejects_aliasing(ctx):
    import torch
    g = cases.build_gpu(ctx, "cantilever3d", 4, 3, 2)
    g.set_density(cases.uniform_density(g.nel, 1))
    v = torch.zeros(g.soa_length(), dtype=torch.float64, device="cuda")
    with pytest.raises(icb.IcbError):
        g.smoother_apply_device(v.data_ptr(), v.data_ptr(), v.data_ptr(), v.data_ptr(), 0.0, 1.0)
