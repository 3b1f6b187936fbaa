"""Filters, threshold, OC, MMA and the ICARAT app loops on the GPU, through
the C ABI, against the oracle and against ICARAT's own OC/MMA (golden
vectors from oracle/_ref).

Bars: filters and threshold 1e-13 relative (same sums, same order);
Helmholtz filter 1e-7 (both sides solve to 1e-10); OC 1e-4 on x (the
bisection stops at a relative lambda width of 1e-5); MMA 1e-9; loop
histories 1e-4 per step (relative compliance).
"""
import os

import numpy as np
import pytest

import cases
import icarat_b200 as icb
import pyoracle as po

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("dims,kw,r", [((2, 23, 11), {}, 1.5), ((2, 30, 12), {}, 3.0),
                                       ((2, 16, 9), {"lx": 8.0, "ly": 9.0}, 1.2),
                                       ((3, 9, 7, 5), {}, 1.5), ((3, 8, 6, 6), {}, 2.0)])
def test_cone_filter_matches_oracle(ctx, dims, kw, r):
    o = po.Problem(*dims, **kw)
    g = icb.Problem(ctx, *dims, **kw)
    g.finalize()
    x = np.random.default_rng(1).uniform(0.01, 1.0, o.nel)
    oc, gc = po.Cone(o, r), icb.Cone(g, r)
    a, b = oc.apply(x), gc.apply(x)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    s = np.random.default_rng(2).standard_normal(o.nel)
    a, b = oc.apply(s, sens=True), gc.apply(s, sens=True)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_threshold_matches_oracle(ctx):
    x = np.random.default_rng(3).uniform(0, 1, 1000)
    for beta in (1.0, 2.0, 16.0):
        a, b = icb.threshold(ctx, x, beta)
        assert np.abs(a - po.threshold(x, beta)).max() <= 1e-14
        assert np.abs(b - po.threshold_deriv(x, beta)).max() <= 1e-12 * beta


@pytest.mark.parametrize("dims,R", [((2, 40, 20), 2.0), ((2, 25, 10), 3.0), ((3, 12, 8, 6), 3.0),
                                    ((3, 70, 17, 9), 2.5), ((3, 33, 40, 3), 4.0)])
def test_helmholtz_filter_matches_oracle(ctx, dims, R):
    o = po.Problem(*dims)
    g = icb.Problem(ctx, *dims)
    g.finalize()
    x = np.random.default_rng(4).uniform(0.01, 1.0, o.nel)
    h = icb.Helmholtz(g, R)
    for sens in (False, True):
        a, b = o.helmholtz(R, x, sens=sens), h.apply(x, sens=sens)
        assert np.abs(a - b).max() <= 1e-7 * np.abs(a).max()


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "ref_opt.npz")), reason="no fixture")
def test_oc_update_matches_icarat(ctx):
    G = np.load(os.path.join(GOLD, "ref_opt.npz"))
    # filtered + thresholded volume callback on a 15x10 grid (golden from ICARAT's OC)
    g = icb.Problem(ctx, 2, 15, 10)
    g.finalize()
    cone = icb.Cone(g, 1.5)
    n = g.nel
    x, steps = icb.oc_update(g, cone, G["ocf_x"], G["ocf_df"], float(G["ocf_g"]), np.ones(n),
                             np.full(n, 1e-4), np.ones(n), 0.2, beta=float(G["ocf_beta"]))
    assert np.abs(x - G["ocf_out"]).max() <= 1e-4
    assert 10 <= steps <= 100


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "ref_opt.npz")), reason="no fixture")
def test_mma_matches_icarat(ctx):
    G = np.load(os.path.join(GOLD, "ref_opt.npz"))
    traj = G["mma_traj"]
    n = traj.shape[1]
    m = icb.MMA(ctx, n)
    for k in range(G["mma_df"].shape[0]):
        # ICARAT's own iterate in, so both sides see the same history
        x = m.update(traj[k], G["mma_df"][k], G["mma_g"][k], G["mma_dg"][k], np.full(n, 1e-4),
                     np.ones(n))
        assert np.abs(x - traj[k + 1]).max() <= 1e-9, k


def test_oc_loop_c1_history(ctx):
    """The opt-macro-oc loop on the 120x40 cantilever (cone r = 1.5, move 0.2,
    threshold schedule, 50 steps): per-step compliance within 1e-4 of the
    oracle's loop."""
    kind, n = "cantilever2d", (120, 40)
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho0 = np.full(o.nel, 0.5)
    ho, xo, _ = o.oc_loop(rho0, 50, 1.5, 0.2, use_beta=True, tol=1e-10)
    hg, xg = icb.run_loop(g, "oc", rho0, 50, 1.5, move=0.2, use_threshold=True, tol=1e-10)
    rel = np.abs(hg - ho) / np.abs(ho)
    assert rel.max() <= 1e-4, rel
    assert hg[-1] < 0.5 * hg[0]  # the design improves


def test_mma_helmholtz_loop_history(ctx):
    kind, n = "halfmbb2d", (40, 16)
    o = cases.build_oracle(kind, *n)
    g = cases.build_gpu(ctx, kind, *n)
    rho0 = np.full(o.nel, 0.4)
    ho, xo = o.mma_loop(rho0, 15, 2.0, tol=1e-10)
    hg, xg = icb.run_loop(g, "mma", rho0, 15, 2.0, tol=1e-10)
    rel = np.abs(hg - ho) / np.abs(ho)
    assert rel.max() <= 1e-4, rel
    assert np.abs(xg - xo).max() <= 1e-3


def test_oc_update_across_filter_rebuilds_matches_oracle(ctx):
    """OC updates through the C ABI with a cone filter of radius 2, then one of
    radius 3, then a new one of radius 2 (each created after the previous one
    was destroyed, so the allocators may hand out the same addresses): every
    update matches the oracle's OC with the same filtered and thresholded
    volume callback (OCSolver.hpp:20-68, opt_macro_oc.cpp:153-164)."""
    nx, ny = 30, 12
    o = po.Problem(2, nx, ny)
    g = icb.Problem(ctx, 2, nx, ny)
    g.finalize()
    n = o.nel
    rng = np.random.default_rng(7)
    x0 = rng.uniform(0.2, 0.8, n)
    df = -rng.uniform(0.1, 2.0, n)
    dg = np.ones(n)
    lo, hi = np.full(n, 1e-4), np.ones(n)
    beta, target = 2.0, 0.45 * n
    outs = []
    for r in (2.0, 3.0, 2.0):
        cone = icb.Cone(g, r)
        xg, steps = icb.oc_update(g, cone, x0, df, target, dg, lo, hi, 0.2, beta=beta)
        cone.close()
        oc = po.Cone(o, r)
        xo = po.oc_update(x0, df, target, dg, lo, hi, 0.2,
                          lambda xk: float(po.threshold(oc.apply(xk), beta).sum()))
        assert np.abs(xg - xo).max() <= 1e-4, r
        assert 10 <= steps <= 100
        outs.append(xg)
    assert np.array_equal(outs[0], outs[2])
    assert not np.array_equal(outs[0], outs[1])


def test_repeated_loops_on_one_problem_agree(ctx):
    """The app loops keep their filters, updaters and work vectors with the
    problem: a second run (and one with another filter radius in between)
    starts from a fresh solver state and repeats the first bitwise."""
    g = cases.build_gpu(ctx, "halfmbb2d", 40, 16)
    rho0 = np.full(g.nel, 0.4)
    for kind in ("mma", "oc"):
        h1, x1 = icb.run_loop(g, kind, rho0, 6, 2.0, tol=1e-10)
        icb.run_loop(g, kind, rho0, 2, 3.0, tol=1e-10)
        h2, x2 = icb.run_loop(g, kind, rho0, 6, 2.0, tol=1e-10)
        assert np.array_equal(h1, h2) and np.array_equal(x1, x2), kind
    a = icb.run_gcmma(g, rho0, 4, 1.5)
    b = icb.run_gcmma(g, rho0, 4, 1.5)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("kind", ["oc", "mma"])
def test_loop_checkpoint_resume_repeats_the_run(ctx, kind):
    """A loop stopped after step 4 with a checkpoint and resumed on another
    problem of the same grid repeats the uninterrupted 8-step run bitwise:
    the design, V0, the stop rule's state and (MMA) the iteration count,
    asymptotes and previous designs are everything carried between steps."""
    g = cases.build_gpu(ctx, "halfmbb2d", 40, 16)
    rho0 = np.full(g.nel, 0.4)
    full_h, full_x = icb.run_loop(g, kind, rho0, 8, 2.0, tol=1e-10)
    ck = np.zeros(icb.checkpoint_bytes(g, kind), np.uint8)
    h1, _ = icb.run_loop(g, kind, rho0, 4, 2.0, tol=1e-10, checkpoint=ck)
    g2 = cases.build_gpu(ctx, "halfmbb2d", 40, 16)
    h2, x2 = icb.run_loop(g2, kind, None, 8, 2.0, tol=1e-10, resume=ck)
    assert np.array_equal(h1, full_h[:4])
    assert np.array_equal(h2[4:], full_h[4:]) and not h2[:4].any()
    assert np.array_equal(x2, full_x)
    g2.close()


@pytest.mark.parametrize("kind", ["oc", "mma"])
def test_loop_stop_rule(ctx, kind):
    """conv_eps applies Optimize::isConvergence(eps, minstep): the step whose
    objective changed by less than eps (relative) after minstep ends the loop
    (its update still runs); the history up to there equals the full run's."""
    g = cases.build_gpu(ctx, "halfmbb2d", 40, 16)
    rho0 = np.full(g.nel, 0.4)
    full, _ = icb.run_loop(g, kind, rho0, 8, 2.0, tol=1e-10)
    done = np.zeros(1, np.int32)
    h, _ = icb.run_loop(g, kind, rho0, 8, 2.0, tol=1e-10, conv_eps=0.9, conv_min_steps=3,
                        steps_done=done)
    rel = np.abs(np.diff(full)) / np.abs(full[1:])
    expect = next(s for s in range(4, 9) if rel[s - 2] < 0.9)
    assert done[0] == expect
    assert np.array_equal(h[:expect], full[:expect]) and not h[expect:].any()
