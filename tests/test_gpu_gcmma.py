"""GCMMA on the device (GCMMASolver's outer / inner updates and ConCheck, and
the opt-macro-gcmma loop) against ICARAT's own GCMMASolver outputs (golden
vectors) and the oracle's loop; the GCMMA app on the C++ shim against the
same loop.

Bars: the update sequence reproduces every ConCheck verdict of ICARAT's
GCMMASolver and its designs within 1e-9; loop compliance histories within
1e-4 per step with the same inner-iteration counts.
"""
import os
import subprocess
import sys
import tomllib

import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(REPO, "tests", "golden")


def test_gcmma_updates_match_icarat_golden(ctx):
    sys.path.insert(0, GOLD)
    import make_golden as mg
    G = np.load(os.path.join(GOLD, "ref_gcmma.npz"))
    n = len(G["x0"])
    gc = icb.GCMMA(ctx, n)
    outs, checks = mg.gcmma_run(gc, n, G["c"], G["v"], float(G["V"]), G["x0"])
    gc.close()
    assert np.array_equal(checks, G["checks"])
    assert np.abs(outs - G["outs"]).max() < 1e-9


def test_run_gcmma_matches_oracle(ctx):
    nx, ny, steps = 30, 10, 26  # inner iterations start near step 20
    o = cases.build_oracle("cantilever2d", nx, ny)
    g = cases.build_gpu(ctx, "cantilever2d", nx, ny)
    rho0 = np.full(g.nel, 0.5)
    ho, io, xo = o.gcmma_loop(rho0, steps, 2.0, tol=1e-10)
    h, inner, x = icb.run_gcmma(g, rho0, steps, 2.0, precond=icb.JACOBI, tol=1e-10, maxit=100000)
    assert np.abs(h - ho).max() / np.abs(ho).max() <= 1e-4
    assert np.array_equal(inner, io)
    assert inner.sum() > 0  # the inner loop ran


def test_gcmma_app_on_shim_matches_oracle():
    path = os.path.join(GOLD, "toml", "gcmma2d.toml")
    with open(path, "rb") as fh:
        cfg = tomllib.load(fh)
    r = subprocess.run([os.path.join(REPO, "icarat-contact_b200", "lib", "opt_macro_gcmma_gpu"),
                        path], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = np.array([[float(v) for v in ln.split(",")] for ln in r.stdout.split()])
    steps = cfg["this_problem"]["steps"]
    assert out.shape == (steps, 4)
    assert out[:, 3].sum() > 0  # the inner loop ran
    from test_shim import _oracle_from_toml
    p, rho_init = _oracle_from_toml(cfg)
    ho, io, _ = p.gcmma_loop(np.full(p.nel, rho_init), steps, 2.0, tol=1e-10)
    assert np.abs(out[:, 1] - ho).max() / np.abs(ho).max() <= 1e-4
    assert np.array_equal(out[:, 3].astype(int), io)
