"""Parity of the CUDA path (through the C ABI) with the oracle.

Bars: integer set-up (DOF map) bit-exact; K0 and loads to 1e-14; operator
products to 1e-12 relative; solves at ||r||/||f|| <= 1e-8 give compliance
within 1e-6 relative and sensitivities within 1e-5 (L-inf relative to
max |dc|) of the oracle solved to 1e-12.
"""
import numpy as np
import pytest

import cases
import icarat_b200 as icb
import pyoracle as po

pytestmark = pytest.mark.gpu

COMPLIANCE_RTOL = 1e-6
SENS_RTOL = 1e-5


@pytest.mark.parametrize("dims,kw", [
    ((2, 3, 3), {}), ((2, 3, 3), {"state": 1}), ((3, 2, 2, 2), {}),
    ((3, 2, 2, 2), {"lx": 3.0, "ly": 1.0, "lz": 1.5}), ((2, 4, 2), {"lx": 2.0, "ly": 3.0, "nu": 0.25}),
])
def test_K0_matches_oracle(ctx, dims, kw):
    a = po.Problem(*dims, **kw).K0()
    b = icb.Problem(ctx, *dims, **kw).K0()
    assert np.abs(a - b).max() < 1e-14 * np.abs(a).max()


def test_dof_numbering_and_traction_loads_match_oracle(ctx):
    # ICARAT fdm.toml (20x10 quad4, plane strain) and 3d.toml-style boxes
    for dims, kw, dirich, tract in [
        ((2, 20, 10), {"state": 1, "young": (0.001, 200.0)},
         [([1, 1, 0, 0, 0, 0], [0] * 6, [0, 0, 0, 10, 0, 10])],
         [([0.0, -0.01, 0.0], [20, 20, 0, 10, 0, 0])]),
        ((2, 12, 6), {}, [([1, 1], [0, 0], [0, 0, 0, 6, 0, 0]), ([0, 1], [0, 0], [11, 12, 0, 0, 0, 0])],
         [([0.5, -1.0, 0], [3, 9, 6, 6, 0, 0]), ([1.0, 0.0, 0], [0, 12, 0, 6, 0, 0])]),
        ((3, 10, 4, 4), {"lx": 20.0, "ly": 8.0, "lz": 8.0, "young": (0.001, 100.0)},
         [([1, 1, 1], [0, 0, 0], [0, 0, 0, 200, 0, 200])],
         [([0, 0, -0.001], [15, 20, 0, 8, 0, 3]), ([0, 0.3, 0], [0, 20, 8, 8, 0, 8]),
          ([0.2, 0, 0], [0, 20, 0, 8, 8, 8])]),
    ]:
        o = po.Problem(*dims, **kw)
        g = icb.Problem(ctx, *dims, **kw)
        for fl, v, r in dirich:
            o.dirichlet_box(fl, v, r)
            g.dirichlet_box(fl, v, r)
        for v, r in tract:
            o.traction_box(v, r)
            g.traction_box(v, r)
        dof_o, numeq_o = o.dofs()
        numeq = g.finalize()
        assert numeq == numeq_o
        assert np.array_equal(g.dof_map(), dof_o)
        fo, fg = o.fext(), g.load()
        assert np.abs(fo - fg).max() <= 1e-14 * max(1.0, np.abs(fo).max())


@pytest.mark.parametrize("kind,n", [("cantilever2d", (37, 13)), ("cantilever2d", (120, 40)),
                                    ("halfmbb2d", (33, 9)),
                                    ("cantilever3d", (9, 5, 4)), ("cantilever3d", (40, 9, 17)),
                                    ("halfmbb3d", (12, 8, 6))])
def test_matvec_and_diagonal_match_assembled(ctx, kind, n):
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, 5)
    g.set_density(rho)
    rp, col, val = o.assemble(rho)
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, rp), shape=(g.numeq,) * 2)
    x = np.random.default_rng(1).standard_normal(g.numeq)
    y = g.matvec(x)
    yo = A @ x
    assert np.abs(y - yo).max() <= 1e-12 * np.abs(yo).max()
    assert np.allclose(g.diagonal(), A.diagonal(), rtol=1e-13, atol=0)


@pytest.mark.parametrize("kind,n,seed", [("cantilever2d", (120, 40), 1), ("cantilever2d", (31, 33), 2),
                                         ("halfmbb2d", (60, 20), 6),
                                         ("cantilever3d", (24, 8, 8), 3), ("halfmbb3d", (16, 8, 8), 4)])
def test_fp64_jacobi_solve_parity(ctx, kind, n, seed):
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, seed)
    ro = o.solve(rho, tol=1e-12)
    dco = o.sensitivity(rho, ro["nodeval"])
    g.set_density(rho)
    info = g.solve(tol=1e-8, maxit=100000)
    assert info["relres"] <= 1e-8 and info["true_relres"] <= 2e-8
    c = g.compliance()
    assert abs(c - ro["compliance"]) <= COMPLIANCE_RTOL * abs(ro["compliance"])
    dc = g.sensitivity()
    assert np.abs(dc - dco).max() <= SENS_RTOL * np.abs(dco).max()
    u = g.displacement()
    assert np.abs(u - ro["u"]).max() <= 1e-5 * np.abs(ro["u"]).max()
    # same algorithm as the oracle at the same tolerance: iteration counts agree closely
    ro8 = o.solve(rho, tol=1e-8)
    assert abs(info["iters"] - ro8["iters"]) <= max(3, 0.02 * ro8["iters"])


def test_nonzero_dirichlet_values(ctx):
    o = po.Problem(2, 16, 8)
    g = icb.Problem(ctx, 2, 16, 8)
    for p in (o, g):
        p.dirichlet_box([1, 1], [0, 0], [0, 0, 0, 8, 0, 0])
        p.dirichlet_box([1, 0], [0.01, 0], [16, 16, 0, 8, 0, 0])
    g.finalize()
    rho = cases.uniform_density(o.nel, 9, 0.3, 1.0)
    ro = o.solve(rho, tol=1e-13)
    g.set_density(rho)
    g.solve(tol=1e-11)
    assert np.abs(g.node_values() - ro["nodeval"]).max() <= 1e-8 * np.abs(ro["nodeval"]).max()
    assert abs(g.compliance() - ro["compliance"]) <= 1e-6 * abs(ro["compliance"]) + 1e-14


def test_zero_load_and_errors(ctx):
    g = icb.Problem(ctx, 2, 8, 4)
    g.dirichlet_box([1, 1], [0, 0], [0, 0, 0, 4, 0, 0])
    g.finalize()
    with pytest.raises(icb.IcbError):
        g.solve()  # no density yet: STATE
    g.set_density(np.full(g.nel, 0.5))
    info = g.solve()
    assert info["iters"] == 0 and g.compliance() == 0.0
    with pytest.raises(icb.IcbError):
        g.solve(tol=-1.0)
    with pytest.raises(icb.IcbError):
        icb.Problem(ctx, 4, 2, 2)


@pytest.mark.parametrize("dim,n", [(2, (8, 4)), (3, (6, 3, 4))])
def test_zero_load_and_fully_constrained_with_every_solver(ctx, dim, n):
    """A problem with no load and one with every DOF constrained (numeq = 0)
    solve at iteration 0 with every solver and give zero compliance and
    sensitivities."""
    box = [0, n[0], 0, n[1], 0, n[2] if dim == 3 else 0]
    free = icb.Problem(ctx, dim, *n)
    free.dirichlet_box([1] * dim, [0.0] * dim, [0, 0] + box[2:])
    free.finalize()
    fixed = icb.Problem(ctx, dim, *n)
    fixed.dirichlet_box([1] * dim, [0.0] * dim, box)
    fixed.finalize()
    assert fixed.numeq == 0
    for g in (free, fixed):
        g.set_density(np.full(g.nel, 0.5))
        for precision, precond in ((icb.FP64, icb.JACOBI), (icb.FP64, icb.GMG),
                                   (icb.MIXED, icb.GMG), (icb.MIXED_REFINE, icb.GMG)):
            info = g.solve(precision=precision, precond=precond)
            assert info["iters"] == 0, (precision, precond, info)
            assert g.compliance() == 0.0
            assert not g.sensitivity().any()
            assert not g.displacement().any()


def test_maxit_status(ctx):
    g = cases.build_gpu(ctx, "cantilever2d", 40, 20)
    g.set_density(cases.uniform_density(g.nel, 3))
    info = g.solve(tol=1e-12, maxit=5, raise_on_error=False)
    assert info["rc"] == -4 and info["iters"] == 5


def test_full_size_cantilever3d_properties(ctx):
    """192x64x64 Hex8 (2.4M DOF): residual, symmetry and energy identities."""
    g = cases.build_gpu(ctx, "cantilever3d", 192, 64, 64)
    rho = cases.uniform_density(g.nel, 2024)
    g.set_density(rho)
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal(g.numeq), rng.standard_normal(g.numeq)
    Kx, Ky = g.matvec(x), g.matvec(y)
    assert abs(x @ Ky - y @ Kx) <= 1e-12 * abs(x @ Ky)
    assert x @ Kx > 0
    info = g.solve(tol=1e-8, maxit=200000)
    assert info["true_relres"] <= 2e-8
    u = g.displacement()
    c = g.compliance()
    assert abs(c - u @ g.matvec(u)) <= 1e-7 * c  # f.u = u.K u at convergence
    dc = g.sensitivity()
    # sum_e rho_e dc_e = -p sum_e rho_e^p (E0 - Emin) u_e^T K0 u_e >= -p c
    assert (dc <= 0).all() and -(rho * dc).sum() <= cases.PENAL * c * (1 + 1e-8)


# ----------------------------------------------------------- multigrid ----
@pytest.mark.parametrize("precision", [icb.FP64, icb.MIXED, icb.MIXED_REFINE])
@pytest.mark.parametrize("kind,n,seed", [("cantilever2d", (120, 40), 1), ("cantilever2d", (37, 23), 2),
                                         ("halfmbb2d", (61, 20), 6),
                                         ("cantilever3d", (24, 8, 8), 3), ("cantilever3d", (19, 7, 9), 5),
                                         ("halfmbb3d", (16, 8, 8), 4)])
def test_gmg_solve_parity(ctx, precision, kind, n, seed):
    """GMG-preconditioned CG -- FP64, FP64 Krylov with an FP32 V-cycle, or FP64
    defect correction around an all-FP32 GMG-PCG -- reaches the FP64
    tolerance and matches the oracle; odd element counts exercise the
    ceil-coarsening."""
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, seed)
    ro = o.solve(rho, tol=1e-12)
    dco = o.sensitivity(rho, ro["nodeval"])
    g.set_density(rho)
    info = g.solve(precision=precision, precond=icb.GMG, tol=1e-8, maxit=20000)
    assert info["true_relres"] <= 2e-8, info
    c = g.compliance()
    assert abs(c - ro["compliance"]) <= COMPLIANCE_RTOL * abs(ro["compliance"])
    dc = g.sensitivity()
    assert np.abs(dc - dco).max() <= SENS_RTOL * np.abs(dco).max()
    ro8 = o.solve(rho, tol=1e-8)
    assert info["matvecs"] < ro8["matvecs"], (info, ro8["matvecs"])


def test_gmg_repeated_solves_reuse_hierarchy(ctx):
    g = cases.build_gpu(ctx, "cantilever3d", 16, 8, 8)
    o = cases.build_oracle("cantilever3d", 16, 8, 8)
    for seed in (1, 2, 3):
        rho = cases.uniform_density(g.nel, seed)
        g.set_density(rho)
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8)
        ro = o.solve(rho, tol=1e-12)
        assert abs(g.compliance() - ro["compliance"]) <= COMPLIANCE_RTOL * ro["compliance"]
        assert info["iters"] > 0


def test_mixed_full_size_cantilever3d(ctx):
    """192x64x64 (2.4M DOF) mixed-precision GMG solve: FP64 residual <= 1e-8 and
    agreement with the FP64 GMG solve of the same system."""
    g = cases.build_gpu(ctx, "cantilever3d", 192, 64, 64)
    rho = cases.uniform_density(g.nel, 2024)
    g.set_density(rho)
    i64 = g.solve(precision=icb.FP64, precond=icb.GMG, tol=1e-8, maxit=20000)
    c64, dc64 = g.compliance(), g.sensitivity()
    for prec in (icb.MIXED, icb.MIXED_REFINE):
        imx = g.solve(precision=prec, precond=icb.GMG, tol=1e-8, maxit=20000)
        assert imx["true_relres"] <= 2e-8 and i64["true_relres"] <= 2e-8
        assert abs(g.compliance() - c64) <= COMPLIANCE_RTOL * c64
        assert np.abs(g.sensitivity() - dc64).max() <= SENS_RTOL * np.abs(dc64).max()


@pytest.mark.parametrize("kind,n", [("cantilever2d", (61, 20)), ("halfmbb3d", (16, 8, 8))])
def test_device_and_host_loop_forms_agree(ctx, kind, n):
    """The multigrid PCG and the OC bisection give bitwise-identical results
    whether their iterations run in a conditional WHILE graph on the device
    or in host-polled batches (the kernels after the stop are gated)."""
    rho = cases.uniform_density(int(np.prod(n)), 11)
    out = {}
    for dev in (1, 0):
        icb.set_option("device_loops", dev)
        try:
            g = cases.build_gpu(ctx, kind, *n)
            g.set_density(rho)
            info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8)
            u = g.displacement()
            hist, x = icb.run_loop(g, "oc", np.full(g.nel, 0.4), 3, 1.5, move=0.2)
            out[dev] = (info["iters"], u, hist, x)
            g.close()
        finally:
            icb.set_option("device_loops", 1)
    assert icb.get_option("device_loops") == 1
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("modal", [1, 0])
def test_non_cubic_hex8_operator_and_solve(ctx, modal):
    """Box elements with three different edge lengths and nu = 0.42: the
    corner-mode operator (its 45 coefficients depend on the box) and the dense
    one both match the assembled oracle, and the mixed GMG solve (which uses
    them on every level) matches the oracle's solution."""
    n, L, nu = (13, 7, 5), (19.5, 5.6, 9.0), 0.42   # h = 1.5, 0.8, 1.8
    import pyoracle as po
    o = po.Problem(3, *n, lx=L[0], ly=L[1], lz=L[2], young=(cases.EMIN, cases.E0), nu=nu,
                   penal=cases.PENAL)
    g = icb.Problem(ctx, 3, *n, lx=L[0], ly=L[1], lz=L[2], young=(cases.EMIN, cases.E0), nu=nu,
                    penal=cases.PENAL)
    fixed, f = cases.masks("cantilever3d", *n)
    o.fixed[:] = fixed
    o.fext_full[:] = f
    g.dirichlet_mask(fixed)
    for nd in np.nonzero(np.abs(f.reshape(-1, 3)).sum(1))[0]:
        g.nodal_load(nd, f.reshape(-1, 3)[nd])
    g.finalize()
    rho = cases.uniform_density(o.nel, 9)
    icb.set_option("hex8_modal", modal)
    try:
        g.set_density(rho)
        rp, col, val = o.assemble(rho)
        import scipy.sparse as sp
        A = sp.csr_matrix((val, col, rp), shape=(g.numeq,) * 2)
        x = np.random.default_rng(2).standard_normal(g.numeq)
        yo = A @ x
        assert np.abs(g.matvec(x) - yo).max() <= 1e-12 * np.abs(yo).max()
        info = g.solve(precision=icb.MIXED, precond=icb.GMG, tol=1e-8, maxit=20000)
        assert info["true_relres"] <= 2e-8, info
        ro = o.solve(rho, tol=1e-12)
        assert abs(g.compliance() - ro["compliance"]) <= COMPLIANCE_RTOL * abs(ro["compliance"])
        dc = g.sensitivity()
        dco = o.sensitivity(rho, ro["nodeval"])
        assert np.abs(dc - dco).max() <= SENS_RTOL * np.abs(dco).max()
    finally:
        icb.set_option("hex8_modal", 1)


@pytest.mark.parametrize("kind,n", [("strip2d", (1024, 4)), ("strip2d", (300, 1)),
                                    ("cantilever3d", (40, 1, 12)), ("cantilever3d", (48, 16, 1)),
                                    ("halfmbb3d", (1, 6, 5))])
def test_thin_and_high_aspect_grids(ctx, kind, n):
    """Grids one element thick along an axis, or so flat that 2:1 coarsening
    of every axis reaches a one-element axis before a small coarsest system
    (1024x4 stopped at 256x1 with 1028 DOFs, past the dense limit; the 3D
    plates stopped at the fine grid): the operator and its diagonal match the
    assembled oracle (corner-mode and dense Hex8), and the FP64 and mixed GMG
    solves, which keep a one-element axis while the others halve, match the
    oracle's solution."""
    import scipy.sparse as sp
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho = cases.uniform_density(o.nel, 11, 0.3, 1.0)
    g.set_density(rho)
    rp, col, val = o.assemble(rho)
    A = sp.csr_matrix((val, col, rp), shape=(g.numeq,) * 2)
    x = np.random.default_rng(4).standard_normal(g.numeq)
    yo = A @ x
    for modal in ([1, 0] if len(n) == 3 else [1]):
        icb.set_option("hex8_modal", modal)
        try:
            assert np.abs(g.matvec(x) - yo).max() <= 1e-12 * np.abs(yo).max()
        finally:
            icb.set_option("hex8_modal", 1)
    assert np.allclose(g.diagonal(), A.diagonal(), rtol=1e-13, atol=0)
    ro = o.solve(rho, tol=1e-12)
    assert ro["relres"] <= 1e-12
    dco = o.sensitivity(rho, ro["nodeval"])
    for precision in (icb.FP64, icb.MIXED, icb.MIXED_REFINE):
        info = g.solve(precision=precision, precond=icb.GMG, tol=1e-8, maxit=20000)
        assert info["true_relres"] <= 2e-8, info
        assert abs(g.compliance() - ro["compliance"]) <= COMPLIANCE_RTOL * abs(ro["compliance"])
        dc = g.sensitivity()
        assert np.abs(dc - dco).max() <= SENS_RTOL * np.abs(dco).max()
