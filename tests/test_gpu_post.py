"""Post-processing and the wider app loops against the oracle: element
stresses / von Mises (Elastic::makeMisesStress), nodal reactions
(LinearAnalysis reaction), the per-step report of the device loops, and the
non-design MMA loop with the cone filter (opt-macro-mma-nondesign) through
the C ABI and through the C++ app on the class shim.

Bars: stresses and von Mises within 1e-9 of the oracle (relative to the
largest value), reactions within 1e-9 of the largest load-scale entry, loop
compliance histories within 1e-4 per step (the app-history bar), all at
||r||/||f|| <= 1e-10.
"""
import os
import subprocess
import tomllib

import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _solved_pair(ctx, kind, n, seed, state=None):
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    if state is not None:  # plane strain variants: rebuild both with the state
        import pyoracle as po
        o2 = po.Problem(2, *n, state=state, young=(cases.EMIN, cases.E0), nu=cases.NU,
                        penal=cases.PENAL)
        o2.fixed[:], o2.fext_full[:] = o.fixed, o.fext_full
        o = o2
        g = icb.Problem(ctx, 2, *n, state=state, young=(cases.EMIN, cases.E0), nu=cases.NU,
                        penal=cases.PENAL)
        fixed, f = cases.masks(kind, *n)
        g.dirichlet_mask(fixed)
        for nn in np.nonzero(np.abs(f.reshape(-1, 2)).sum(1))[0]:
            g.nodal_load(nn, f.reshape(-1, 2)[nn])
        g.finalize()
    rho = cases.uniform_density(g.nel, seed)
    g.set_density(rho)
    g.solve(tol=1e-12, maxit=100000)
    return o, g, rho


@pytest.mark.parametrize("kind,n,state", [("cantilever2d", (40, 16), None),
                                          ("cantilever2d", (31, 9), 1),
                                          ("halfmbb3d", (12, 6, 5), None),
                                          ("cantilever3d", (10, 4, 7), None)])
def test_von_mises_and_reactions_match_oracle(ctx, kind, n, state):
    o, g, rho = _solved_pair(ctx, kind, n, 3, state)
    nv = g.node_values()
    m, st = g.von_mises(with_stress=True)
    mo, sto = o.von_mises(rho, nv, with_stress=True)
    assert np.abs(st - sto).max() <= 1e-9 * np.abs(sto).max()
    assert np.abs(m - mo).max() <= 1e-9 * mo.max()
    r = g.reactions()
    ro = o.reactions(rho, nv)
    assert np.abs(r - ro).max() <= 1e-9 * np.abs(ro).max()
    # equilibrium: at free DOFs the internal force is the load
    free = o.fixed == 0
    assert np.abs(r[free] - o.fext_full[free]).max() <= 1e-8 * np.abs(ro).max()


def test_step_report_matches_final_state(ctx):
    g = cases.build_gpu(ctx, "cantilever2d", 30, 10)
    seen = []
    hist, x = icb.run_loop(g, "oc", np.full(g.nel, 0.5), 5, 1.5, move=0.2,
                           on_step=lambda *a: seen.append(a))
    assert [s[0] for s in seen] == [1, 2, 3, 4, 5]
    assert np.allclose([s[1] for s in seen], hist, rtol=0, atol=0)
    step, comp, rho, nv, mises = seen[-1]
    assert np.array_equal(nv, g.node_values())
    assert np.array_equal(mises, g.von_mises())
    assert rho.min() > 0.0 and rho.max() <= 1.0


def _nondesign_masks(nx, ny, rows):
    """The app's element lists (opt_macro_mma_nondesign.cpp:254-301) on a unit grid."""
    cx = (np.arange(nx) + 0.5)[None, :].repeat(ny, 0).ravel()
    cy = (np.arange(ny) + 0.5)[:, None].repeat(nx, 1).ravel()
    nd = np.zeros(nx * ny, bool)
    ds = np.zeros(nx * ny, bool)
    rho0 = np.full(nx * ny, np.nan)
    for val, (xr, yr) in rows:
        inside = (xr[0] < cx) & (cx < xr[1]) & (yr[0] < cy) & (cy < yr[1])
        nd |= inside
        ds |= ~inside
        rho0[inside] = val
    return nd, ds, rho0


def test_mma_cone_nondesign_loop_matches_oracle(ctx):
    nx, ny = 40, 16
    rows = [(1.0, ((14.0, 26.0), (10.0, 16.0))), (1e-4, ((6.0, 12.0), (4.0, 9.0)))]
    nd, ds, r0 = _nondesign_masks(nx, ny, rows)
    rho0 = np.where(np.isnan(r0), 0.4, r0)
    o = cases.build_oracle("cantilever2d", nx, ny)
    g = cases.build_gpu(ctx, "cantilever2d", nx, ny)
    steps = 10
    ho, xo = o.mma_cone_loop(rho0, steps, 2.0, nondesign=nd, volset=ds, tol=1e-10)
    h, x = icb.run_loop(g, "mma", rho0, steps, 2.0, filter_type=icb.FILTER_CONE, nondesign=nd,
                        volume_set=ds, precond=icb.JACOBI, tol=1e-10, maxit=100000)
    assert np.abs(h - ho).max() / np.abs(ho).max() <= 1e-4
    assert np.abs(x - xo).max() <= 1e-2
    # non-design variables keep their value: zero gradients leave MMA at x
    assert np.abs(x[nd] - rho0[nd]).max() <= 1e-6


def test_nondesign_app_on_shim_matches_oracle():
    path = os.path.join(REPO, "tests", "golden", "toml", "nondesign2d.toml")
    with open(path, "rb") as fh:
        cfg = tomllib.load(fh)
    tp = cfg["this_problem"]
    r = subprocess.run([os.path.join(REPO, "icarat-contact_b200", "lib", "opt_macro_mma_nondesign_gpu"),
                        path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = np.array([[float(v) for v in ln.split(",")] for ln in r.stdout.split()])
    assert out.shape == (tp["steps"], 4)
    from test_shim import _oracle_from_toml
    p, rho_init = _oracle_from_toml(cfg)
    nx, ny = cfg["mesh"]["division"][:2]
    rows = [(v[0], (rng[0], rng[1])) for v, rng in tp["non_design"]]
    nd, ds, r0 = _nondesign_masks(nx, ny, rows)
    rho0 = np.where(np.isnan(r0), rho_init, r0)
    ho, _ = p.mma_cone_loop(rho0, tp["steps"], tp["filterR"], nondesign=nd, volset=ds, tol=1e-10)
    assert np.abs(out[:, 1] - ho).max() / np.abs(ho).max() <= 1e-4
    assert out[0, 2] == 0.0 and np.all(out[:, 3] > 0)
