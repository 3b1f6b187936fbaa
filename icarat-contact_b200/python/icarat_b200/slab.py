"""One structured Hex8 solve partitioned over ranks in x-slabs: the multi-GPU
form of LinearAnalysis::solve with Eigen_CG semantics
(src/analysis/linear.hpp:54-104, src/analysis/solver/solvers.cpp:64-92).

ICARAT carries the fields of such a decomposition without using them
(procno, procid, begdof, gnumeq in src/problem/base.hpp:25-33; the
countDOFMPI / generateLoadMainMPI hooks of
src/io/boundary_condition_icarat.hpp:55,194).  Here, with W ranks:

* rank r owns the elements with x in [e0_r, e1_r) (contiguous slabs, as even
  as the element count allows) and the node planes x in [e0_r, e1_r), the
  last rank also the plane x = nx.  It stores the node planes [e0_r, e1_r] of
  its slab: the plane x = e1_r is a copy of the next rank's first plane.
* An operator application sums the slab's elements (on a GPU: the library's
  matrix-free operator on the slab's own icb_problem), then adds the
  neighbours' partial sums on the two shared planes: one exchange of a node
  plane (3 (ny+1)(nz+1) values) with each neighbour, by send / recv into local
  buffers; every rank then holds the full sums on its copy of each plane.
* Jacobi-PCG as the single-GPU JacobiPcg runs it (x0 = 0, stop when
  ||r||^2 < max(tol^2 ||b||^2, DBL_MIN), inverse diagonal 1 where the
  diagonal is 0 and 0 on constrained DOFs, Eigen's iteration count).  Per
  iteration the dot products sum over the owned planes only and are
  all-reduced in FP64 twice: p.Ap, then r.r and r.z together.  Every other
  vector operation is local, so the copies of a shared plane stay identical.

Vectors are the library's SoA field vectors (component c of node n at
c * ld + n, n = i + j sx + k sx sy over the slab's nodes) as torch tensors on
the rank's device; `op(u) -> y` computes the slab's element sum for every
node (constrained rows 0).  The collectives go through torch.distributed:
NCCL between GPUs, gloo between CPU ranks.
"""
import math

import torch

DBL_MIN = 2.2250738585072014e-308


def slab_ranges(nx, world):
    """[(e0, e1)] element ranges of the ranks: contiguous, sizes differing by
    at most one element, every rank at least one element"""
    if world > nx:
        raise ValueError("more ranks than element columns")
    return [(r * nx // world, (r + 1) * nx // world) for r in range(world)]


class SlabLayout:
    """The slab of rank `rank`: its element range, node planes, SoA stride and
    the views the exchange and the reductions use."""

    def __init__(self, nx, ny, nz, rank, world, ld=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.rank, self.world = rank, world
        self.e0, self.e1 = slab_ranges(nx, world)[rank]
        self.nxl = self.e1 - self.e0
        self.sx, self.sy, self.sz = self.nxl + 1, ny + 1, nz + 1
        self.nnode = self.sx * self.sy * self.sz
        self.ld = ld if ld is not None else ((self.nnode + 63) // 64) * 64
        # owned node planes of the slab: all but the copy of the next rank's first
        self.nown = self.sx if rank == world - 1 else self.sx - 1

    def grid(self, v):
        """(3, sz, sy, sx) view of a SoA vector"""
        return v.view(3, self.ld)[:, :self.nnode].view(3, self.sz, self.sy, self.sx)

    def owned(self, v):
        return self.grid(v)[:, :, :, :self.nown]

    def to_slab(self, full):
        """the slab's part of a (3, nz+1, ny+1, nx+1) node array, as a SoA vector"""
        v = full.new_zeros(3 * self.ld)
        self.grid(v).copy_(full[:, :, :, self.e0:self.e1 + 1])
        return v


class Exchange:
    """Halo exchange of the shared planes and the FP64 all-reduce, over a
    torch.distributed process group (`dist` is torch.distributed, or None for
    one rank); `device` is where the rank's vectors live."""

    def __init__(self, layout, dist=None, group=None, device="cpu"):
        self.L, self.dist, self.group, self.device = layout, dist, group, device

    def add_shared_planes(self, y):
        """y <- y + the neighbours' partial sums on the two shared planes"""
        L, dist = self.L, self.dist
        if dist is None or L.world == 1:
            return y
        g = L.grid(y)
        ops, recv = [], []
        if L.rank > 0:  # first plane, shared with rank - 1
            send = g[:, :, :, 0].contiguous()
            buf = torch.empty_like(send)
            ops += [dist.P2POp(dist.isend, send, L.rank - 1, self.group),
                    dist.P2POp(dist.irecv, buf, L.rank - 1, self.group)]
            recv.append((0, buf))
        if L.rank < L.world - 1:  # last plane, shared with rank + 1
            send = g[:, :, :, L.sx - 1].contiguous()
            buf = torch.empty_like(send)
            ops += [dist.P2POp(dist.isend, send, L.rank + 1, self.group),
                    dist.P2POp(dist.irecv, buf, L.rank + 1, self.group)]
            recv.append((L.sx - 1, buf))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        for i, buf in recv:
            g[:, :, :, i] += buf
        return y

    def allreduce(self, vals):
        """sums over the ranks of FP64 scalars (0-dim tensors on the rank's
        device): one collective, one host synchronisation"""
        t = torch.stack([v.to(torch.float64) for v in vals])
        if self.dist is not None and self.L.world > 1:
            self.dist.all_reduce(t, group=self.group)
        return t.tolist()


def owned_dot(L, a, b):
    """the rank's part of a.b: its owned node planes only"""
    return (L.owned(a) * L.owned(b)).sum()


def slab_jacobi_pcg(L, ex, op, b, diag, free, tol, maxit):
    """Jacobi-PCG on the partitioned system.  b: the slab's right-hand side
    (0 on constrained DOFs, identical on both copies of a shared plane); diag:
    the slab's element sum of the diagonal (partial on the shared planes);
    free: bool SoA mask of the unknowns (False on constrained DOFs and the
    padding).  Returns (x, info): info holds Eigen's iteration count (the
    converging iteration excluded), the operator applications, ||r||/||b||
    and a status (0, -3 breakdown, -4 iteration limit, -6 non-finite)."""
    d = ex.add_shared_planes(diag.clone())
    one = torch.ones_like(d)
    dinv = torch.where(free, torch.where(d != 0, 1.0 / torch.where(d != 0, d, one), one),
                       torch.zeros_like(d))
    x = torch.zeros_like(b)
    r = torch.where(free, b, torch.zeros_like(b))
    z = dinv * r
    p = z.clone()
    bb, rz = ex.allreduce([owned_dot(L, r, r), owned_dot(L, r, z)])
    thr = max(tol * tol * bb, DBL_MIN)
    it, mv, rr = 0, 0, bb
    if bb == 0.0 or bb < thr:
        return x, {"iters": 0, "matvecs": 0, "relres": 0.0, "status": 0}
    status = -4
    while it < maxit:
        q = ex.add_shared_planes(op(p))
        mv += 1
        (pq,) = ex.allreduce([owned_dot(L, p, q)])
        if not pq > 0.0:
            status = -3
            break
        alpha = rz / pq
        x.add_(p, alpha=alpha)
        r.add_(q, alpha=-alpha)
        z = dinv * r
        rr, rzn = ex.allreduce([owned_dot(L, r, r), owned_dot(L, r, z)])
        if not (math.isfinite(rr) and math.isfinite(rzn)):
            status = -6
            break
        if rr < thr:
            status = 0
            break
        it += 1
        p.mul_(rzn / rz).add_(z)
        rz = rzn
    return x, {"iters": it, "matvecs": mv, "relres": math.sqrt(rr / bb), "status": status}


def gpu_slab(ctx, L, fixed4, load4, rho_slab, young=(1e-9, 1.0), nu=0.3, penal=3.0):
    """The slab of rank L.rank as an icb_problem on the rank's GPU: its grid,
    the Dirichlet flags and loads of its node planes ((3, nz+1, ny+1, nx+1)
    arrays of the whole grid, component-major) and its element densities
    (nz, ny, nxl).  Returns (prob, op, b, diag, free) with b, diag and free
    as SoA tensors on the device; the library's loads are not used: every
    rank takes the full load of its planes, copies included."""
    import numpy as np

    from . import Problem
    dev = torch.device("cuda", ctx.device)
    prob = Problem(ctx, 3, L.nxl, L.ny, L.nz, young=young, nu=nu, penal=penal)
    fx = np.ascontiguousarray(fixed4[:, :, :, L.e0:L.e1 + 1].transpose(1, 2, 3, 0)).reshape(-1)
    prob.dirichlet_mask(fx.astype(np.uint8))
    prob.finalize()
    assert prob.soa_length() == 3 * L.ld
    prob.set_density(np.ascontiguousarray(rho_slab).reshape(-1))
    fixed_soa = L.to_slab(torch.from_numpy(np.ascontiguousarray(fixed4, np.float64))) != 0
    pad = torch.ones(3 * L.ld, dtype=torch.bool)
    L.grid(pad).fill_(False)
    free = ~(fixed_soa | pad)
    b = torch.where(free, L.to_slab(torch.from_numpy(np.ascontiguousarray(load4, np.float64))),
                    torch.zeros(3 * L.ld, dtype=torch.float64))
    # the slab's diagonal (numeq order) scattered to the SoA layout
    dq = prob.diagonal()
    dof = prob.dof_map()
    diag = np.zeros(3 * L.ld)
    nodes = np.arange(L.nnode)
    for c in range(3):
        d = dof[nodes * 3 + c]
        ok = d < prob.numeq
        diag[c * L.ld + nodes[ok]] = dq[d[ok]]
    return (prob, device_operator(prob), b.to(dev), torch.from_numpy(diag).to(dev),
            free.to(dev))


def device_operator(prob, stream=None):
    """op(u) for a GPU rank: the library's FP64 matrix-free operator on the
    slab's icb_problem (density already set), on SoA tensors of the device"""
    from . import FP64

    def op(u):
        y = torch.empty_like(u)
        torch.cuda.current_stream().synchronize()
        prob.operator_apply_device(u.data_ptr(), y.data_ptr(), FP64)
        prob.ctx.synchronize()
        return y

    return op
