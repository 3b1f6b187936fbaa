"""Generate the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py [--small-fem]

ref_opt.npz -- outputs of ICARAT's own OC and MMA updates (OCSolver.hpp,
    MMASolver.cpp compiled from the ICARAT sources into oracle/_ref by
    oracle/Makefile) on seeded inputs: one OC update with a plain-volume
    callback, one OC update whose callback filters and thresholds (as
    opt_macro_oc.cpp:155-164 does), and a 6-step MMA trajectory with m = 1.
ref_gcmma.npz -- ICARAT's own GCMMASolver (GCMMASolver.cpp from the ICARAT
    sources, same build) driven through 8 outer updates with inner
    iterations on the analytic problem min sum c / x^3 s.t. sum v x^2 / V
    <= 1 (steep enough that several approximations are not conservative):
    every update's output design and every ConCheck verdict.
small_fem.npz -- oracle outputs on small structured problems (K0 matrices,
    loads of ICARAT's fdm.toml boundary conditions, a solve and its
    sensitivities), kept as regression vectors for the oracle itself.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402


def ref_opt():
    rng = np.random.default_rng(20240611)
    n = 300
    out = {}
    x = rng.uniform(0.1, 0.9, n)
    df = -rng.uniform(0.01, 3.0, n)
    dg = rng.uniform(0.5, 1.5, n)
    xmin, xmax = np.full(n, 1e-4), np.ones(n)
    g = 0.45 * dg.sum()
    out["oc_x"], out["oc_df"], out["oc_dg"], out["oc_g"] = x, df, dg, g
    out["oc_out"] = po.oc_update(x, df, g, dg, xmin, xmax, 0.2, lambda xx: float(xx @ dg),
                                 use_ref=True)
    # OC with the filtered + thresholded volume callback on a 15x10 grid
    p = po.Problem(2, 15, 10)
    cone = po.Cone(p, 1.5)
    x2 = rng.uniform(0.2, 0.8, p.nel)
    df2 = -rng.uniform(0.01, 1.0, p.nel)
    dv2 = np.ones(p.nel)
    beta = 2.0

    def vol(xx):
        return float(po.threshold(cone.apply(xx), beta).sum())

    g2 = 0.5 * p.nel
    out["ocf_x"], out["ocf_df"], out["ocf_g"], out["ocf_beta"] = x2, df2, g2, beta
    out["ocf_out"] = po.oc_update(x2, df2, g2, dv2, np.full(p.nel, 1e-4), np.ones(p.nel), 0.2,
                                  vol, use_ref=True)
    # MMA trajectory (m = 1), objective and constraint gradients from seeded draws
    m = po.MMA(n, 1, use_ref=True)
    xm = rng.uniform(0.2, 0.6, n)
    traj, dfs, gs, dgs = [xm.copy()], [], [], []
    for _ in range(6):
        dfm = -rng.uniform(0.1, 2.0, n) * (1.0 + xm)
        dgm = np.full(n, 1.0 / (0.4 * n))
        gm = np.array([xm.sum() / (0.4 * n) - 1.0])
        xm = m.update(xm, dfm, gm, dgm, np.full(n, 1e-4), np.ones(n))
        traj.append(xm.copy())
        dfs.append(dfm)
        gs.append(gm)
        dgs.append(dgm)
    out["mma_traj"], out["mma_df"], out["mma_g"], out["mma_dg"] = (
        np.array(traj), np.array(dfs), np.array(gs), np.array(dgs))
    return out


def gcmma_problem(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 2.0, n)
    v = rng.uniform(0.5, 1.5, n)
    V = 0.35 * 0.25 * v.sum()
    return c, v, V


def gcmma_run(gc, n, c, v, V, x0, outers=8):
    """Outer / inner GCMMA sequence of the GCMMA app (opt_macro_gcmma.cpp:
    153-212) on f0 = sum c / x^3, f = sum v x^2 / V - 1; returns the designs
    after every update and the ConCheck verdicts, in order."""
    f0 = lambda x: float((c / x ** 3).sum())  # noqa: E731
    f = lambda x: float(v @ x ** 2 / V - 1.0)  # noqa: E731
    xmin, xmax = np.full(n, 1e-4), np.ones(n)
    x = x0.copy()
    outs, checks = [], []
    for _ in range(outers):
        df0, df = -3.0 * c / x ** 4, 2.0 * v * x / V
        xm = gc.outer(x, f0(x), df0, f(x), df, xmin, xmax)
        outs.append(xm.copy())
        ok = gc.concheck(f0(xm), f(xm))
        checks.append(ok)
        k = 0
        while not ok and k < 15:
            xm = gc.inner(xm, f0(xm), f(xm), x, f0(x), df0, f(x), df, xmin, xmax)
            outs.append(xm.copy())
            ok = gc.concheck(f0(xm), f(xm))
            checks.append(ok)
            k += 1
        x = xm
    return np.array(outs), np.array(checks)


def ref_gcmma():
    n = 96
    c, v, V = gcmma_problem(n, 7)
    x0 = np.full(n, 0.5)
    outs, checks = gcmma_run(po.GCMMA(n, 1, use_ref=True), n, c, v, V, x0)
    return {"c": c, "v": v, "V": V, "x0": x0, "outs": outs, "checks": checks}


def small_fem():
    out = {}
    out["K0_q4_stress"] = po.Problem(2, 2, 2).K0()
    out["K0_q4_strain"] = po.Problem(2, 2, 2, state=1).K0()
    out["K0_h8"] = po.Problem(3, 2, 2, 2).K0()
    out["K0_h8_rect"] = po.Problem(3, 2, 2, 2, lx=3.0, ly=1.0, lz=1.5).K0()
    # ICARAT's opt-mma-HelmholtzFilter/fdm.toml: 20x10 quad4, plane_strain,
    # x = 0 clamped, traction (0,-0.01) on the edge x = 20
    p = po.Problem(2, 20, 10, state=1, young=(0.001, 200.0), nu=0.3)
    p.dirichlet_box([1, 1, 0, 0, 0, 0], [0] * 6, [0, 0, 0, 10, 0, 10])
    p.traction_box([0.0, -0.01, 0.0], [20, 20, 0, 10, 0, 0])
    dof, numeq = p.dofs()
    out["fdm_dof"], out["fdm_numeq"], out["fdm_fext"] = dof, numeq, p.fext()
    rho = np.full(p.nel, 0.4)
    r = p.solve(rho, tol=1e-12)
    out["fdm_u"], out["fdm_comp"] = r["u"], r["compliance"]
    out["fdm_dc"] = p.sensitivity(rho, r["nodeval"])
    # ICARAT's opt-mma-HelmholtzFilter/3d.toml boundary conditions on a 10x4x4 box
    p3 = po.Problem(3, 10, 4, 4, lx=20.0, ly=8.0, lz=8.0, young=(0.001, 100.0))
    p3.dirichlet_box([1, 1, 1], [0, 0, 0], [0, 0, 0, 200, 0, 200])
    p3.traction_box([0, 0, -0.001], [15, 20, 0, 8, 0, 3])
    d3, n3 = p3.dofs()
    out["h8_dof"], out["h8_numeq"], out["h8_fext"] = d3, n3, p3.fext()
    return out


if __name__ == "__main__":
    if po.ref_available():
        np.savez_compressed(os.path.join(HERE, "ref_opt.npz"), **ref_opt())
        print("wrote ref_opt.npz (ICARAT OC/MMA from oracle/_ref)")
        np.savez_compressed(os.path.join(HERE, "ref_gcmma.npz"), **ref_gcmma())
        print("wrote ref_gcmma.npz (ICARAT GCMMA from oracle/_ref)")
    else:
        print("oracle/_ref not built: ref_opt.npz left as it is")
    if "--small-fem" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "small_fem.npz"), **small_fem())
        print("wrote small_fem.npz")
