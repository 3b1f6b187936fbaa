"""Heat conduction (LinearHeat with SIMP conductivity, the opt-heat app) on
the device against the oracle's assembled restatement.

Bars: temperatures within 1e-8 of the largest, objective u^T K u within 1e-8,
sensitivities within 1e-6 (L-inf relative), loop objective histories within
1e-4 per step; solves at ||r||/||f|| <= 1e-12.
"""
import numpy as np
import pytest

import icarat_b200 as icb
import pyoracle as po

pytestmark = pytest.mark.gpu

C2_1 = [100.0, 60.0, 0.0, 15.0, 0.0, 0.0]   # anisotropic, xy coupling
C2_2 = [0.1, 0.1, 0.0, 0.0, 0.0, 0.0]
C3_1 = [10.0, 8.0, 6.0, 1.0, 0.5, 0.3]
C3_2 = [0.01, 0.01, 0.01, 0.0, 0.0, 0.0]


def _pair(ctx, dim, n, L, c1, c2, bcs, fluxes):
    o = po.Problem(dim, *n, lx=L[0], ly=L[1], lz=L[2] if dim == 3 else None, state=3)
    g = icb.Heat(ctx, dim, *n, lx=L[0], ly=L[1], lz=L[2] if dim == 3 else None, cond1=c1,
                 cond2=c2)
    for flag, val, rng in bcs:
        o.dirichlet_box([flag, 0, 0, 0, 0, 0], [val, 0, 0, 0, 0, 0], rng)
        g.dirichlet_box(flag, val, rng)
    for q, rng in fluxes:
        o.traction_box([q, 0, 0], rng)
        g.flux_box(q, rng)
    g.finalize()
    return o, g


CASES = [
    # 2D: the opt-heat layout (T = 0 on part of the top, flux box over the plate)
    (2, (20, 20), (1.0, 1.0, 1.0), C2_1, C2_2,
     [(1, 0.0, [0.4, 0.6, 1.0, 1.0, 0, 0])], [(0.1, [0, 1, 0, 1, 0, 0])]),
    # 2D with a non-zero prescribed temperature on a side
    (2, (16, 9), (2.0, 1.0, 1.0), C2_1, C2_2,
     [(1, 1.5, [0, 0, 0, 1, 0, 0])], [(0.3, [2, 2, 0, 1, 0, 0])]),
    # 3D, general conductivity tensor
    (3, (8, 6, 5), (1.0, 0.75, 0.625), C3_1, C3_2,
     [(1, 0.0, [0, 1, 0.75, 0.75, 0, 0.625])], [(0.2, [0, 0, 0, 0.75, 0, 0.625])]),
]


@pytest.mark.parametrize("dim,n,L,c1,c2,bcs,fluxes", CASES)
def test_heat_solve_matches_oracle(ctx, dim, n, L, c1, c2, bcs, fluxes):
    o, g = _pair(ctx, dim, n, L, c1, c2, bcs, fluxes)
    rho = np.random.default_rng(5).uniform(0.05, 1.0, g.nel)
    r = o.heat_solve(c1, c2, rho, tol=1e-13)
    g.set_density(rho)
    info = g.solve(tol=1e-13, maxit=100000)
    assert info["status"] == 0
    T = g.temperature()
    assert np.abs(T - r["nodeval"]).max() <= 1e-8 * np.abs(r["nodeval"]).max()
    assert abs(g.objective() - r["objective"]) <= 1e-8 * abs(r["objective"])
    dc = g.sensitivity(rho)
    dco = o.heat_sensitivity(c1, c2, rho, r["nodeval"])
    assert np.abs(dc - dco).max() <= 1e-6 * np.abs(dco).max()


def test_heat_loop_matches_oracle(ctx):
    dim, n, L = 2, (24, 24), (1.0, 1.0, 1.0)
    o, g = _pair(ctx, dim, n, L, C2_1, C2_2, [(1, 0.0, [0.4, 0.6, 1.0, 1.0, 0, 0])],
                 [(0.1, [0, 1, 0, 1, 0, 0])])
    rho0 = np.full(g.nel, 0.35)
    steps, R = 8, 0.06
    ho, xo = o.heat_loop(C2_1, C2_2, rho0, steps, R, tol=1e-12)
    h, x = g.run(rho0, steps, R, tol=1e-12)
    assert np.abs(h - ho).max() / np.abs(ho).max() <= 1e-4
    assert h[-1] < h[0]  # the design improves


def test_heat_rejects_weaker_material_one(ctx):
    with pytest.raises(icb.IcbError):
        icb.Heat(ctx, 2, 4, 4, cond1=[0.1, 0.1, 0, 0, 0, 0], cond2=[1, 1, 0, 0, 0, 0])
