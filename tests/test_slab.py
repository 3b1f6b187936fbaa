"""The x-slab partition of one solve (icarat_b200.slab) on CPU ranks (gloo):
world sizes 2 and 3 reproduce the one-rank solve's compliance to 1e-12 and
its iteration count to within one, and both match the oracle's
LinearAnalysis::solve restatement.  The slab operator here is a torch element-by-element sum of
E_e K0 u_e with the oracle's K0 (on a GPU rank the library's operator on the
slab's icb_problem takes its place); the partition, the node-plane halo
exchange and the two all-reduces per iteration are the product code.

The multigrid-preconditioned form (slab.SlabMg, slab.slab_gmg_pcg): levels
split over the slabs down to a gather level, the rest on rank 0; world
sizes 2 and 3 and every allowed gather level reproduce the one-rank solve,
which matches the oracle's compliance; the collectives per iteration are
counted."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GRID = (23, 5, 4)
SEED = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _lnode(a, b):
    return (a ^ b) + 2 * b


def _corners():
    out = [None] * 8
    for c in range(2):
        for b in range(2):
            for a in range(2):
                out[_lnode(a, b) + 4 * c] = (a, b, c)
    return out


def _ebe(L, K0, E, fixed):
    """y = sum over the slab's elements of E_e K0 u_e (constrained rows 0)"""
    import torch
    nz, ny, nx = L.nz, L.ny, L.nxl
    cs = _corners()

    def op(u):
        g = L.grid(u)
        ue = torch.stack([g[:, c:c + nz, b:b + ny, a:a + nx] for (a, b, c) in cs]).reshape(24, -1)
        ye = (K0 @ ue) * E.reshape(1, -1)
        y = torch.zeros_like(u)
        yg = L.grid(y)
        for q, (a, b, c) in enumerate(cs):
            yg[:, c:c + nz, b:b + ny, a:a + nx] += ye[3 * q:3 * q + 3].reshape(3, nz, ny, nx)
        y[fixed] = 0.0
        return y

    def diag():
        d = torch.zeros(3 * L.ld, dtype=torch.float64)
        dg = L.grid(d)
        kd = torch.diagonal(K0)
        for q, (a, b, c) in enumerate(cs):
            dg[:, c:c + nz, b:b + ny, a:a + nx] += (kd[3 * q:3 * q + 3].reshape(3, 1) *
                                                    E.reshape(1, -1)).reshape(3, nz, ny, nx)
        d[fixed] = 0.0
        return d

    return op, diag


def _solve(rank, world, dist):
    import torch
    sys.path.insert(0, os.path.join(REPO, "icarat-contact_b200", "python"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cases
    import pyoracle as po
    from icarat_b200 import slab
    nx, ny, nz = GRID
    L = slab.SlabLayout(nx, ny, nz, rank, world)
    K0 = torch.from_numpy(po.Problem(3, 1, 1, 1).K0())
    rho = cases.uniform_density(nx * ny * nz, SEED).reshape(nz, ny, nx)[:, :, L.e0:L.e1]
    E = torch.from_numpy(cases.EMIN + rho ** cases.PENAL * (cases.E0 - cases.EMIN)).contiguous()
    fixed, f = cases.masks("cantilever3d", nx, ny, nz)
    to4 = lambda a: torch.from_numpy(np.ascontiguousarray(  # noqa: E731
        a.reshape(nz + 1, ny + 1, nx + 1, 3).transpose(3, 0, 1, 2)))
    fx = L.to_slab(to4(fixed.astype(np.float64))) != 0
    pad = torch.ones(3 * L.ld, dtype=torch.bool)
    L.grid(pad).fill_(False)
    free = ~(fx | pad)
    b = torch.where(free, L.to_slab(to4(f)), torch.zeros(3 * L.ld, dtype=torch.float64))
    op, diag = _ebe(L, K0, E, ~free)
    ex = slab.Exchange(L, dist)
    x, info = slab.slab_jacobi_pcg(L, ex, op, b, diag(), free, 1e-8, 100000)
    (c,) = ex.allreduce([slab.owned_dot(L, x, b)])
    return info, c


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    info, c = _solve(rank, world, dist)
    dist.destroy_process_group()
    q.put((rank, info, c))


def _run(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=150) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    return res


@pytest.mark.timeout(300)
def test_slab_partition_reproduces_one_rank_solve():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    sys.path.insert(0, os.path.join(REPO, "icarat-contact_b200", "python"))
    import cases
    from icarat_b200 import slab
    info1, c1 = _solve(0, 1, None)
    assert info1["status"] == 0 and info1["relres"] <= 1e-8
    o = cases.build_oracle("cantilever3d", *GRID)
    ro = o.solve(cases.uniform_density(o.nel, SEED), tol=1e-8)
    assert abs(c1 - ro["compliance"]) <= 1e-8 * abs(ro["compliance"])
    assert abs(info1["iters"] - ro["iters"]) <= 1
    for world in (2, 3):
        res = _run(world)
        for rank, info, c in res:
            # the shared planes' sums and the dot products are associated
            # differently from the one-rank solve, so the last iteration's
            # residual differs in its last bits: the count may differ by one
            assert abs(info["iters"] - info1["iters"]) <= 1, (world, rank, info, info1)
            assert info["status"] == 0 and info["relres"] <= 1e-8
            assert abs(c - c1) <= 1e-12 * abs(c1), (world, rank, c, c1)
        assert len({r[2] for r in res}) == 1  # every rank holds the same compliance
    assert [r[1] - r[0] for r in slab.slab_ranges(GRID[0], 3)] == [7, 8, 8]


MG_GRID = (23, 6, 5)


def _mg_solve(rank, world, dist, align, gather, grid=MG_GRID, mixed=False):
    """the multigrid-preconditioned slab solve of `grid` on this rank (FP64, or
    the FP32 V-cycle under FP64 CG); the coarse levels' element matrices from
    the oracle's K0 of a one-element problem with the level's edges"""
    import torch
    sys.path.insert(0, os.path.join(REPO, "icarat-contact_b200", "python"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cases
    import pyoracle as po
    from icarat_b200 import slab
    nx, ny, nz = grid
    L = slab.SlabLayout(nx, ny, nz, rank, world, ranges=slab.slab_ranges(nx, world, align))

    def kmat(h):
        return po.Problem(3, 1, 1, 1, lx=h[0], ly=h[1], lz=h[2], nu=cases.NU).K0()

    rho = cases.uniform_density(nx * ny * nz, SEED).reshape(nz, ny, nx)[:, :, L.e0:L.e1]
    E = torch.from_numpy(cases.EMIN + rho ** cases.PENAL * (cases.E0 - cases.EMIN)).contiguous()
    fixed, f = cases.masks("cantilever3d", nx, ny, nz)
    to4 = lambda a: torch.from_numpy(np.ascontiguousarray(  # noqa: E731
        a.reshape(nz + 1, ny + 1, nx + 1, 3).transpose(3, 0, 1, 2)))
    fx = L.to_slab(to4(fixed.astype(np.float64))) != 0
    pad = torch.ones(3 * L.ld, dtype=torch.bool)
    L.grid(pad).fill_(False)
    free = ~(fx | pad)
    b = torch.where(free, L.to_slab(to4(f)), torch.zeros(3 * L.ld, dtype=torch.float64))
    op, diag = slab.element_sum(L, torch.from_numpy(kmat((1.0, 1.0, 1.0))), E, ~free)
    ex = slab.Exchange(L, dist)
    mg = slab.SlabMg(ex, op, diag(), free, E, kmat, gather_level=gather,
                     dtype=torch.float32 if mixed else torch.float64)
    x, info = slab.slab_gmg_pcg(mg, b, 1e-8, 1000)
    counts = dict(ex.counts)
    (c,) = ex.allreduce([slab.owned_dot(L, x, b)])
    return info, c, counts


def _mg_rank_main(rank, world, port, q, align, gather, grid, mixed):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    out = _mg_solve(rank, world, dist, align, gather, grid, mixed)
    dist.destroy_process_group()
    q.put((rank,) + out)


def _mg_run(world, align, gather, grid=MG_GRID, mixed=False):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_mg_rank_main,
                         args=(r, world, port, q, align, gather, grid, mixed))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=150) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    return res


@pytest.mark.timeout(300)
def test_slab_multigrid_partition_reproduces_one_rank_solve():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cases
    info1, c1, _ = _mg_solve(0, 1, None, 1, None)
    assert info1["status"] == 0 and info1["relres"] <= 1e-8
    assert info1["levels"] == 4 and info1["gather_level"] == 3
    o = cases.build_oracle("cantilever3d", *MG_GRID)
    ro = o.solve(cases.uniform_density(o.nel, SEED), tol=1e-12)
    assert abs(c1 - ro["compliance"]) <= 1e-10 * abs(ro["compliance"])
    # the V-cycle cuts Jacobi-PCG's iteration count by an order of magnitude
    assert 10 * info1["iters"] < ro["iters"]
    # (world, slab alignment, gather level): boundaries 12 (two coarsenings)
    # and 8, 16 (three); the gather level from the first coarse level to the
    # coarsest one
    for world, align, gather, g in ((2, 4, None, 2), (2, 4, 1, 1), (3, 8, None, 3),
                                    (3, 2, 1, 1)):
        res = _mg_run(world, align, gather)
        for rank, info, c, counts in res:
            assert info["gather_level"] == g, (world, gather, info)
            assert info["status"] == 0 and info["relres"] <= 1e-8
            assert abs(info["iters"] - info1["iters"]) <= 1, (world, rank, info, info1)
            assert abs(c - c1) <= 1e-12 * abs(c1), (world, rank, c, c1)
            # two FP64 all-reduces per pass of the loop (the converging one
            # included) after the two of the start; one reduce to rank 0 and
            # one broadcast per V-cycle (plus the set-up's two reduces)
            passes, vcycles = info["matvecs"], info["matvecs"] + 1
            assert counts["allreduce"] == 2 + 2 * passes
            assert counts["reduce"] == vcycles + 2 and counts["broadcast"] == vcycles
        assert len({r[2] for r in res}) == 1


@pytest.mark.timeout(300)
def test_slab_multigrid_thin_grid_and_bad_partitions():
    """a grid one element thick (the z axis kept while x and y halve) on two
    ranks; slab boundaries a coarsening cannot keep, and a gather level
    the boundaries do not allow, are refused"""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import cases
    grid = (24, 6, 1)
    info1, c1, _ = _mg_solve(0, 1, None, 1, None, grid)
    assert info1["status"] == 0 and info1["levels"] == 3
    o = cases.build_oracle("cantilever3d", *grid)
    ro = o.solve(cases.uniform_density(o.nel, SEED), tol=1e-12)
    # a plate one element thick bends: compliance 1.6e6 against 1.8e4 for the
    # block above, and the rounding of the ranks' sums shows at ~1e-11
    assert abs(c1 - ro["compliance"]) <= 1e-10 * abs(ro["compliance"])
    for rank, info, c, counts in _mg_run(2, 4, None, grid):
        assert abs(info["iters"] - info1["iters"]) <= 1 and abs(c - c1) <= 1e-10 * abs(c1)
    # the gather level by size: the first level of at most gather_dofs DOFs
    # (23 x 6 x 5 -> 12 x 3 x 3: 624 DOFs -> 6 x 2 x 2: 189 -> 3 x 1 x 1: 48),
    # else the deepest the boundaries allow (one rank: the coarsest)
    import torch
    from icarat_b200 import slab
    L = slab.SlabLayout(23, 6, 5, 0, 1)
    E = torch.ones(5, 6, L.nxl, dtype=torch.float64)
    free = torch.zeros(3 * L.ld, dtype=torch.bool)
    L.grid(free).fill_(True)
    K = torch.eye(24, dtype=torch.float64)
    op, diag = slab.element_sum(L, K, E, ~free)
    for gd, g in ((100000, 1), (624, 1), (623, 2), (189, 2), (188, 3), (10, 3), (None, 3)):
        mg = slab.SlabMg(slab.Exchange(L, None), op, diag(), free, E, lambda h: K.numpy(),
                         gather_dofs=gd)
        assert mg.g == g, (gd, mg.g)
    with pytest.raises(ValueError, match="even"):
        _mg_solve(1, 3, None, 1, None)  # boundaries 7 and 15
    with pytest.raises(ValueError, match="gather level"):
        _mg_solve(0, 1, None, 1, 0)
    with pytest.raises(ValueError, match="gather level"):
        _mg_solve(0, 2, None, 4, 3)  # 12 keeps two coarsenings, not three


@pytest.mark.timeout(300)
def test_slab_multigrid_fp32_vcycle_partitions_like_one_rank():
    """the library's mixed form (FP32 levels, FP64 coarsest solve and CG) on
    the slabs: the iteration count of the FP64 V-cycle, and worlds 2 and 3
    reproduce the one-rank compliance (the FP32 V-cycles of the partitions
    round differently, so to 1e-10 rather than 1e-12)"""
    info64, c64, _ = _mg_solve(0, 1, None, 1, None)
    info1, c1, _ = _mg_solve(0, 1, None, 1, None, mixed=True)
    assert info1["status"] == 0 and info1["relres"] <= 1e-8
    assert abs(info1["iters"] - info64["iters"]) <= 1 and abs(c1 - c64) <= 1e-10 * abs(c64)
    for world, align, gather in ((2, 4, None), (3, 2, 1)):
        res = _mg_run(world, align, gather, mixed=True)
        for rank, info, c, counts in res:
            assert info["status"] == 0 and abs(info["iters"] - info1["iters"]) <= 1
            assert abs(c - c1) <= 1e-10 * abs(c1), (world, rank, c, c1)
            assert counts["allreduce"] == 2 + 2 * info["matvecs"]
        assert len({r[2] for r in res}) == 1
