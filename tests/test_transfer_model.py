"""The multigrid transfers' index arithmetic, restated on the CPU.

k_restrict and k_prolong_add (mg.cu) take a per-axis coarsening shift s
(1: the axis halves, ceil for odd counts; 0: a one-element axis is kept).
Their index formulas are transcribed here literally, applied to unit vectors
on small grids, and checked for two things the kernels rely on: every index
they form stays inside its grid, and the restriction is the transpose of the
prolongation (R = P^T) for every shift pattern the hierarchy builder can
produce.  No GPU.
"""
import itertools

import numpy as np


def _coarse(nel, s):
    return (nel + 1) // 2 if s else nel


def _prolong(fine_nodes, coarse_nodes, sh, xc):
    """x_f = P x_c: per fine node, I0 = i >> s, I1 = (i + s) >> s along each
    axis and nested midpoints, as k_prolong_add forms them."""
    dim = len(fine_nodes)
    xf = np.zeros(fine_nodes)
    for idx in itertools.product(*[range(n) for n in fine_nodes]):
        lo_hi = []
        for a in range(dim):
            i, s = idx[a], sh[a]
            I0, I1 = i >> s, (i + s) >> s
            assert 0 <= I0 < coarse_nodes[a] and 0 <= I1 < coarse_nodes[a]
            lo_hi.append((I0, I1))
        v = 0.0
        for pick in itertools.product((0, 1), repeat=dim):
            v += xc[tuple(lo_hi[a][pick[a]] for a in range(dim))]
        xf[idx] = v * 0.5 ** dim
    return xf


def _restrict(fine_nodes, coarse_nodes, sh, rf):
    """b_c = R r_f: per coarse node, fine I << s and neighbours -s..s with
    weight 1/2 off the centre, those inside the fine grid, as k_restrict
    forms them."""
    dim = len(fine_nodes)
    bc = np.zeros(coarse_nodes)
    for idx in itertools.product(*[range(n) for n in coarse_nodes]):
        v = 0.0
        for off in itertools.product(*[range(-sh[a], sh[a] + 1) for a in range(dim)]):
            f = tuple((idx[a] << sh[a]) + off[a] for a in range(dim))
            if all(0 <= f[a] < fine_nodes[a] for a in range(dim)):
                v += rf[f] * 0.5 ** sum(1 for o in off if o)
        bc[idx] = v
    return bc


def _matrices(fine_el, sh):
    fine_nodes = tuple(n + 1 for n in fine_el)
    coarse_nodes = tuple(_coarse(n, s) + 1 for n, s in zip(fine_el, sh))
    nf, nc = int(np.prod(fine_nodes)), int(np.prod(coarse_nodes))
    P = np.zeros((nf, nc))
    R = np.zeros((nc, nf))
    for j in range(nc):
        e = np.zeros(nc)
        e[j] = 1.0
        P[:, j] = _prolong(fine_nodes, coarse_nodes, sh, e.reshape(coarse_nodes)).ravel()
    for j in range(nf):
        e = np.zeros(nf)
        e[j] = 1.0
        R[:, j] = _restrict(fine_nodes, coarse_nodes, sh, e.reshape(fine_nodes)).ravel()
    return P, R


def test_restriction_is_the_transpose_of_prolongation():
    for fine_el in [(1,), (2,), (5,), (6,), (3, 1), (4, 5), (1, 3), (2, 1, 3), (3, 2, 1), (1, 1, 4)]:
        # the builder halves every axis with at least two elements and keeps the others
        sh = tuple(1 if n >= 2 else 0 for n in fine_el)
        P, R = _matrices(fine_el, sh)
        assert np.array_equal(R, P.T), (fine_el, sh)
        # interpolation reproduces constants on every fine node
        assert np.allclose(P.sum(1), 1.0), (fine_el, sh)


def test_every_shift_pattern_on_a_small_box():
    # shifts of 0 on axes longer than one element are never built, but the
    # formulas stay consistent for them too
    for sh in itertools.product((0, 1), repeat=3):
        P, R = _matrices((3, 2, 2), sh)
        assert np.array_equal(R, P.T), sh
