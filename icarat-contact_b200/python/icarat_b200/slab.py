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


def slab_ranges(nx, world, align=1):
    """[(e0, e1)] element ranges of the ranks: contiguous, every rank at least
    one element.  The inner boundaries are multiples of `align` (the columns
    are dealt out in blocks of `align`, the last block possibly shorter, the
    block counts differing by at most one); align = 1 gives sizes that differ
    by at most one element.  A multigrid partition aligns the boundaries to
    2^m so that m coarsenings keep every boundary on a coarse node plane."""
    if align < 1:
        raise ValueError("align must be positive")
    q = (nx + align - 1) // align
    if world > q:
        raise ValueError("more ranks than element columns (in blocks of %d)" % align)
    cut = [min(nx, align * (r * q // world)) for r in range(world)] + [nx]
    return [(cut[r], cut[r + 1]) for r in range(world)]


class SlabLayout:
    """The slab of rank `rank`: its element range, node planes, SoA stride and
    the views the exchange and the reductions use."""

    def __init__(self, nx, ny, nz, rank, world, ld=None, ranges=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.rank, self.world = rank, world
        self.ranges = list(ranges) if ranges is not None else slab_ranges(nx, world)
        self.e0, self.e1 = self.ranges[rank]
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
        self.counts = {"exchange": 0, "allreduce": 0, "reduce": 0, "broadcast": 0}

    def on(self, layout):
        """an exchange of the same ranks for another level's layout"""
        return Exchange(layout, self.dist, self.group, self.device)

    def add_shared_planes(self, y):
        """y <- y + the neighbours' partial sums on the two shared planes"""
        L, dist = self.L, self.dist
        if dist is None or L.world == 1:
            return y
        self.counts["exchange"] += 1
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
            self.counts["allreduce"] += 1
            self.dist.all_reduce(t, group=self.group)
        return t.tolist()

    def reduce_to_root(self, t):
        """t <- the sum of every rank's t on rank 0 (the others' t undefined)"""
        if self.dist is not None and self.L.world > 1:
            self.counts["reduce"] += 1
            self.dist.reduce(t, dst=self._root(), group=self.group)
        return t

    def broadcast_from_root(self, t):
        """every rank's t <- rank 0's t"""
        if self.dist is not None and self.L.world > 1:
            self.counts["broadcast"] += 1
            self.dist.broadcast(t, src=self._root(), group=self.group)
        return t

    def _root(self):
        # global rank of the group's rank 0
        if self.group is None:
            return 0
        return self.dist.get_global_rank(self.group, 0)


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


# ------------------------------------------------------------- multigrid ---
# The partitioned form of the library's geometric multigrid preconditioner
# (mg_impl.cuh, MgPcg): the same level hierarchy, masks, moduli, Chebyshev
# smoother, transfers and flexible CG, with the levels split over the ranks'
# x-slabs down to a gather level and the levels from there on held by rank 0
# alone.  ICARAT has no multigrid (its iterative solve is Eigen's Jacobi CG,
# src/analysis/solver/solvers.cpp:64-92).

COARSE_DOFS = 160  # the library's default coarsest size (dense solve)


def _corners():
    """(a, b, c) offsets of the Hex8 corners in element-matrix order: corner
    lnode(a, b) + 4 c with lnode(a, b) = (a ^ b) + 2 b (meshBox order)"""
    out = [None] * 8
    for c in range(2):
        for b in range(2):
            for a in range(2):
                out[(a ^ b) + 2 * b + 4 * c] = (a, b, c)
    return out


def element_sum(L, K, E, fixed):
    """(op, diag) of the slab's element sum: op(u) = sum_e E_e K u_e and
    diag() = its diagonal, both 0 on constrained rows; K is the (24, 24) unit
    element matrix (DOF 3 q + c: component c of corner q), E the slab's
    moduli (nz, ny, nxl), fixed a bool SoA mask of the constrained DOFs.  The
    torch form of the library's matrix-free Hex8 operator, used on the coarse
    levels of the partitioned multigrid; the partial sums on the shared
    planes are completed by Exchange.add_shared_planes."""
    nz, ny, nx = L.nz, L.ny, L.nxl
    cs = _corners()
    Ev = E.reshape(1, -1)

    def op(u):
        g = L.grid(u)
        ue = torch.stack([g[:, c:c + nz, b:b + ny, a:a + nx] for (a, b, c) in cs])
        ye = (K @ ue.reshape(24, -1)) * Ev
        y = torch.zeros_like(u)
        yg = L.grid(y)
        for q, (a, b, c) in enumerate(cs):
            yg[:, c:c + nz, b:b + ny, a:a + nx] += ye[3 * q:3 * q + 3].reshape(3, nz, ny, nx)
        return y.masked_fill_(fixed, 0.0)

    def diag():
        d = torch.zeros(3 * L.ld, dtype=E.dtype, device=E.device)
        dg = L.grid(d)
        kd = torch.diagonal(K)
        for q, (a, b, c) in enumerate(cs):
            dg[:, c:c + nz, b:b + ny, a:a + nx] += (kd[3 * q:3 * q + 3].reshape(3, 1) *
                                                    Ev).reshape(3, nz, ny, nx)
        return d.masked_fill_(fixed, 0.0)

    return op, diag


def mg_levels(nx, ny, nz, coarse_dofs=COARSE_DOFS):
    """[(nx, ny, nz, sh)] of the multigrid levels, finest first, by the
    library's rule (MgPcg::build): 2:1 coarsening of the element grid with
    ceil for odd counts, an axis one element thick kept (sh 0) while the
    others halve (sh 1), until the grid has <= coarse_dofs DOFs (constrained
    ones counted) or no axis halves"""
    lv = [(nx, ny, nz, (1, 1, 1))]
    while True:
        fx, fy, fz, _ = lv[-1]
        sh = (int(fx >= 2), int(fy >= 2), int(fz >= 2))
        if 3 * (fx + 1) * (fy + 1) * (fz + 1) <= coarse_dofs or not any(sh):
            return lv
        lv.append(((fx + 1) // 2 if sh[0] else fx, (fy + 1) // 2 if sh[1] else fy,
                   (fz + 1) // 2 if sh[2] else fz, sh))


def element_lmax(K):
    """lambda_max(diag(K)^-1 K) of an element matrix with the library's 2 %
    margin: the Chebyshev bound for every modulus field (x^T K x / x^T D x
    is a weighted mean of the element quotients)"""
    import numpy as np
    K = np.asarray(K, dtype=np.float64)
    s = 1.0 / np.sqrt(np.diag(K))
    return float(np.linalg.eigvalsh(K * s[:, None] * s[None, :])[-1]) * 1.02


def chebyshev_coefficients(lmax, nu):
    """(c1, c2) of the three-term Chebyshev smoother in D^-1 K on
    [lmax/10, lmax], steps 0..nu-1 (Saad, Iterative Methods for Sparse Linear
    Systems, 2nd ed., Alg. 12.1): x_{k+1} = x_k + c1_k (x_k - x_{k-1}) +
    c2_k D^-1 (b - K x_k)"""
    a, b = lmax / 10.0, lmax
    theta, delta = 0.5 * (b + a), 0.5 * (b - a)
    sigma = theta / delta
    rho0 = 1.0 / sigma
    c1, c2 = [0.0] * nu, [0.0] * nu
    c2[0] = 1.0 / theta
    for k in range(1, nu):
        rho1 = 1.0 / (2.0 * sigma - rho0)
        c1[k] = rho1 * rho0
        c2[k] = 2.0 * rho1 / delta
        rho0 = rho1
    return c1, c2


def _restrict_axis(v, axis, nc, m):
    """R = P^T along one axis: coarse node I takes the fine node 2I with
    weight 1 and 2I - 1, 2I + 1 with weight 1/2, of the fine nodes [0, m)"""
    v = v.movedim(axis, -1)
    vp = v.new_zeros(v.shape[:-1] + (2 * nc + 2,))
    vp[..., 1:m + 1] = v[..., :m]
    out = vp[..., 1:2 * nc + 1:2] + 0.5 * (vp[..., 0:2 * nc:2] + vp[..., 2:2 * nc + 2:2])
    return out.movedim(-1, axis)


def _prolong_axis(c, axis, nf):
    """P along one axis: fine node i is the midpoint of the coarse nodes
    i >> 1 and (i + 1) >> 1 (the node itself, exactly, for even i)"""
    i = torch.arange(nf, device=c.device)
    return 0.5 * (c.index_select(axis, i >> 1) + c.index_select(axis, (i + 1) >> 1))


def restrict_slab(Lf, Lc, sh, r):
    """the partial coarse vector R r on the coarse layout Lc from the fine
    node planes rank Lf.rank owns (a shared plane is summed by one rank
    only); complete it with the coarse level's shared-plane exchange"""
    v = Lf.grid(r)[:, :, :, :Lf.nown]
    if sh[0]:
        v = _restrict_axis(v, 3, Lc.sx, Lf.nown)
    if sh[1]:
        v = _restrict_axis(v, 2, Lc.sy, Lf.sy)
    if sh[2]:
        v = _restrict_axis(v, 1, Lc.sz, Lf.sz)
    out = r.new_zeros(3 * Lc.ld)
    Lc.grid(out).copy_(v)
    return out


def prolong_slab(Lc, Lf, sh, xc):
    """P xc on every fine node plane the rank stores (x first, then y, then
    z: the library's nested midpoints), as a SoA vector of the layout Lf"""
    v = Lc.grid(xc)
    if sh[0]:
        v = _prolong_axis(v, 3, Lf.sx)
    if sh[1]:
        v = _prolong_axis(v, 2, Lf.sy)
    if sh[2]:
        v = _prolong_axis(v, 1, Lf.sz)
    out = xc.new_zeros(3 * Lf.ld)
    Lf.grid(out).copy_(v)
    return out


def coarsen_moduli(E, sh, shape):
    """coarse moduli (nz, ny, nx) = shape: the mean of each coarse element's
    children, an element sticking out of the domain summing the children
    that exist over all its child slots (the library's k_coarsen_E)"""
    nzc, nyc, nxc = shape
    p = E.new_zeros((nzc << sh[2], nyc << sh[1], nxc << sh[0]))
    p[:E.shape[0], :E.shape[1], :E.shape[2]] = E
    s = p.reshape(nzc, 1 << sh[2], nyc, 1 << sh[1], nxc, 1 << sh[0]).sum(dim=(1, 3, 5))
    return s / float(1 << (sh[0] + sh[1] + sh[2]))


def _inv_diag(d, free):
    """the smoother's D^-1: 0 on constrained DOFs and padding, 1 where the
    diagonal is 0 (the library's k_diag rule)"""
    one = torch.ones_like(d)
    return torch.where(free, torch.where(d != 0, 1.0 / torch.where(d != 0, d, one), one),
                       torch.zeros_like(d))


def _trailing_zeros(v):
    return (v & -v).bit_length() - 1


class _Level:
    """one multigrid level as this rank holds it"""

    def __init__(self, L, ex, sh, K, E, free, op, dinv):
        self.L, self.ex, self.sh, self.K, self.E = L, ex, sh, K, E
        self.free, self.fixed = free, ~free
        self.op, self.dinv = op, dinv

    def apply(self, u):
        """K u, complete on the shared planes"""
        return self.ex.add_shared_planes(self.op(u))


class SlabMg:
    """The library's V-cycle (MgPcg::level in mg_impl.cuh) on an x-slab
    partition.  Levels 0 .. g-1 are split over the ranks: level l
    keeps the fine slabs' boundaries divided by 2^(x halvings so far), which
    slab_ranges(..., align=2^m) keeps integral, so every rank coarsens its
    own moduli and restricts and prolongates its own node planes; a
    smoothing step, a residual and a restriction each exchange the shared
    planes once.  The restriction to level g (the gather level) is reduced
    to rank 0, which runs the V-cycle of levels g .. coarsest on the whole
    level-g grid (the coarsest by a dense Cholesky solve; the library
    inverts it) and broadcasts the level-g correction; every rank then
    prolongates its part.  Nothing but the level-g vectors crosses to rank 0.

    ex, op, diag, free: the fine level as slab_jacobi_pcg takes it (the
    exchange of the fine layout, the slab's element sum, its partial
    diagonal, the unknowns' mask); E: the slab's moduli (nz, ny, nxl);
    kmat(h): the unit element matrix (24, 24) of an element with edges h
    (the library's K0 of a one-element problem); h: the fine element's
    edges.  gather_level: g; by default the first level of at most
    gather_dofs DOFs (constrained ones counted), or the coarsest level the
    slab boundaries allow if that comes first or gather_dofs is None.

    dtype: the V-cycle's precision.  float32 is the library's mixed form
    (MgPcg<double, float>): the levels' vectors, moduli, diagonals and
    element sums in FP32, the coarsest system assembled and solved in FP64,
    the flexible CG (operator `op`, residual, reductions) in FP64.  vop: the
    V-cycle's fine-level operator in dtype (on a GPU rank the library's FP32
    operator on the slab problem); by default `op` for float64 and a torch
    element sum otherwise."""

    def __init__(self, ex, op, diag, free, E, kmat, h=(1.0, 1.0, 1.0), smooth=2,
                 coarse_dofs=COARSE_DOFS, gather_level=None, gather_dofs=None,
                 dtype=torch.float64, vop=None):
        L0 = ex.L
        W, rank = L0.world, L0.rank
        dev, dt = E.device, dtype
        self.op, self.dtype = op, dtype
        E = E.to(torch.float64)
        self.rank, self.ex, self.nu = rank, ex, int(smooth) if smooth > 0 else 2
        self.dims = dims = mg_levels(L0.nx, L0.ny, L0.nz, coarse_dofs)
        nl = self.nl = len(dims)
        if nl < 2:
            raise ValueError("grid too small for a multigrid hierarchy")
        sx = [0]
        for d in dims[1:]:
            sx.append(sx[-1] + d[3][0])
        a = min((_trailing_zeros(e0) for e0, _ in L0.ranges[1:]), default=64)
        allowed = [l for l in range(1, nl) if sx[l] <= a]
        if not allowed:
            raise ValueError("slab boundaries must be even for a multigrid partition "
                             "(slab_ranges(..., align=2**m))")
        if gather_level is not None:
            g = int(gather_level)
        else:
            small = [l for l in allowed if gather_dofs is not None and
                     3 * (dims[l][0] + 1) * (dims[l][1] + 1) * (dims[l][2] + 1) <= gather_dofs]
            g = min(small) if small else max(allowed)
        if g not in allowed:
            raise ValueError("gather level %d not in %s for these slab boundaries" % (g, allowed))
        self.g = g
        # element edges, matrices and the Chebyshev bound of every level
        hs = [tuple(h)]
        K64 = [torch.as_tensor(kmat(hs[0]), dtype=torch.float64)]
        lmax, changed = element_lmax(K64[0].numpy()), False
        for l in range(1, nl):
            sh = dims[l][3]
            hs.append(tuple(2.0 * hs[-1][k] if sh[k] else hs[-1][k] for k in range(3)))
            K64.append(torch.as_tensor(kmat(hs[-1]), dtype=torch.float64))
            changed = changed or sh[0] != sh[1] or sh[1] != sh[2]
            if changed:
                lmax = max(lmax, element_lmax(K64[-1].numpy()))
        Ks = [k.to(device=dev, dtype=dt) for k in K64]
        self.lmax = lmax
        self.c1, self.c2 = chebyshev_coefficients(lmax, self.nu)

        d0 = ex.add_shared_planes(diag.to(torch.float64).clone()).to(dt)
        if vop is None:
            vop = op if dt == torch.float64 else element_sum(L0, Ks[0], E.to(dt), ~free)[0]
        self.lv = [_Level(L0, ex, (1, 1, 1), Ks[0], E, free, vop, _inv_diag(d0, free))]

        def fixed_float(lv):
            m = torch.zeros(3 * lv.L.ld, dtype=dt, device=dev)
            lv.L.grid(m).copy_((~lv.L.grid(lv.free)).to(dt))
            return m

        def make(L, lex, l, E_l, mask):
            free = torch.zeros(3 * L.ld, dtype=torch.bool, device=dev)
            L.grid(free).copy_(L.grid(mask) == 0)
            o, dg = element_sum(L, Ks[l], E_l.to(dt), ~free)
            return _Level(L, lex, dims[l][3], Ks[l], E_l, free, o,
                          _inv_diag(lex.add_shared_planes(dg()), free))

        # levels 1 .. g-1 on the slabs; the slab layout of level g (where the
        # restriction lands and the correction is taken from)
        for l in range(1, g + 1):
            nx, ny, nz, sh = dims[l]
            ranges = [(e0 >> sx[l], (e1 >> sx[l]) if r < W - 1 else nx)
                      for r, (e0, e1) in enumerate(L0.ranges)]
            L = SlabLayout(nx, ny, nz, rank, W, ranges=ranges)
            f = self.lv[-1]
            E_l = coarsen_moduli(f.E, sh, (nz, ny, L.nxl))
            mask = restrict_slab(f.L, L, sh, fixed_float(f))
            if l < g:
                lex = ex.on(L)
                self.lv.append(make(L, lex, l, E_l, lex.add_shared_planes(mask)))
                continue
            # level g: the whole grid on rank 0
            self.land = L
            self.Lg = Lg = SlabLayout(nx, ny, nz, 0, 1)
            Ef = E_l.new_zeros((nz, ny, nx))
            Ef[:, :, L.e0:L.e1] = E_l
            ex.reduce_to_root(Ef)
            mf = ex.reduce_to_root(self._to_full(mask))
            if rank == 0:
                self.lv.append(make(Lg, Exchange(Lg, None, device=dev), l, Ef, mf))
        if rank == 0:
            for l in range(g + 1, nl):
                nx, ny, nz, sh = dims[l]
                L = SlabLayout(nx, ny, nz, 0, 1)
                f = self.lv[-1]
                self.lv.append(make(L, Exchange(L, None, device=dev), l,
                                    coarsen_moduli(f.E, sh, (nz, ny, nx)),
                                    restrict_slab(f.L, L, sh, fixed_float(f))))
            self._factor(self.lv[-1])

    # coarsest level: dense Cholesky of the free DOFs in FP64 (rank 0)
    def _factor(self, C):
        idx = torch.nonzero(C.free).reshape(-1)
        self.cidx, self.chol = idx, None
        n = idx.numel()
        if n == 0:
            return
        op64, _ = element_sum(C.L, C.K.to(torch.float64), C.E, C.fixed)
        A = C.E.new_zeros((n, n))
        for j in range(n):
            e = C.E.new_zeros(3 * C.L.ld)
            e[idx[j]] = 1.0
            A[:, j] = op64(e)[idx]
        self.chol = torch.linalg.cholesky(0.5 * (A + A.T))

    def _coarse(self, b):
        x = torch.zeros_like(b)
        if self.chol is not None:
            bd = b[self.cidx].to(torch.float64).unsqueeze(1)
            x[self.cidx] = torch.cholesky_solve(bd, self.chol).squeeze(1).to(b.dtype)
        return x

    def _to_full(self, part):
        full = part.new_zeros(3 * self.Lg.ld)
        self.Lg.grid(full)[:, :, :, self.land.e0:self.land.e1 + 1] = self.land.grid(part)
        return full

    def _from_full(self, full):
        out = full.new_zeros(3 * self.land.ld)
        self.land.grid(out).copy_(self.Lg.grid(full)[:, :, :, self.land.e0:self.land.e1 + 1])
        return out

    def _cheb(self, lv, b, cur, prev, c1, c2):
        dn = c2 * lv.dinv * (b - lv.apply(cur))
        if c1 != 0.0:
            dn = dn + c1 * (cur - prev)
        return cur + dn

    def _level(self, l, b):
        if l == self.nl - 1:
            return self._coarse(b)
        lv, c1, c2 = self.lv[l], self.c1, self.c2
        cur, oth = c2[0] * lv.dinv * b, torch.zeros_like(b)
        for k in range(1, self.nu):
            cur, oth = self._cheb(lv, b, cur, oth, c1[k], c2[k]), cur
        res = b - lv.apply(cur)
        if l + 1 != self.g:
            C = self.lv[l + 1]
            bc = C.ex.add_shared_planes(restrict_slab(lv.L, C.L, C.sh, res))
            Lc, sh, xc = C.L, C.sh, self._level(l + 1, bc.masked_fill_(C.fixed, 0.0))
        else:
            sh = self.dims[self.g][3]
            full = self.ex.reduce_to_root(self._to_full(restrict_slab(lv.L, self.land, sh, res)))
            if self.rank == 0:
                xg = self._level(self.g, full.masked_fill_(self.lv[self.g].fixed, 0.0))
            else:
                xg = torch.empty_like(full)
            Lc, xc = self.land, self._from_full(self.ex.broadcast_from_root(xg.contiguous()))
        cur = torch.where(lv.free, cur + prolong_slab(Lc, lv.L, sh, xc), cur)
        for k in range(self.nu):
            cur, oth = self._cheb(lv, b, cur, oth, c1[k], c2[k]), cur
        return cur

    def vcycle(self, r):
        """z = V-cycle(r) on the fine slabs in the V-cycle's precision, returned
        in r's (every rank calls it together)"""
        return self._level(0, r.to(self.dtype)).to(r.dtype)


def slab_gmg_pcg(mg, b, tol, maxit):
    """The library's multigrid-preconditioned flexible CG (MgPcg::solve: FP64
    iterate, operator and reductions, the V-cycle in mg.dtype) on the
    partitioned system: x0 = 0, stop when
    ||r||^2 < max(tol^2 ||b||^2, DBL_MIN), Polak-Ribiere beta
    (r.z_new - r.z_old) / r.z_old, the converging iteration not counted.
    Per iteration one operator application with its plane exchange, one
    V-cycle and two FP64 all-reduces: p.Ap, then r.r, r.z_old and r.z_new
    together (the V-cycle of the last iteration is the price of the second
    fusion).  Returns (x, info) as slab_jacobi_pcg, info also holding the
    level count and the gather level."""
    lv = mg.lv[0]
    L, ex, free = lv.L, lv.ex, lv.free
    x = torch.zeros_like(b)
    r = torch.where(free, b, torch.zeros_like(b))
    (bb,) = ex.allreduce([owned_dot(L, r, r)])

    def done(it, mv, rr, status):
        return x, {"iters": it, "matvecs": mv, "status": status, "levels": mg.nl,
                   "gather_level": mg.g, "relres": math.sqrt(rr / bb) if bb > 0 else 0.0}

    if not math.isfinite(bb):
        return done(0, 0, bb, -6)
    thr = max(tol * tol * bb, DBL_MIN)
    if bb == 0.0 or bb < thr:
        return done(0, 0, bb, 0)
    z = mg.vcycle(r)
    (rz,) = ex.allreduce([owned_dot(L, r, z)])
    if not (math.isfinite(rz) and rz > 0.0):
        return done(0, 0, bb, -3 if math.isfinite(rz) else -6)
    p = z.clone()
    it, mv, rr, status = 0, 0, bb, -4
    while it < maxit:
        q = ex.add_shared_planes(mg.op(p))
        mv += 1
        (pq,) = ex.allreduce([owned_dot(L, p, q)])
        alpha = rz / pq if pq > 0.0 else math.nan
        if not math.isfinite(alpha):
            status = -3
            break
        r.add_(q, alpha=-alpha)
        zn = mg.vcycle(r)
        rr, rzo, rzn = ex.allreduce([owned_dot(L, r, r), owned_dot(L, r, z),
                                     owned_dot(L, r, zn)])
        if not math.isfinite(rr):
            status = -6
            break
        x.add_(p, alpha=alpha)
        if rr < thr:
            status = 0
            break
        if not math.isfinite(rzn):
            status = -6
            break
        beta = (rzn - rzo) / rz
        rz, z = rzn, zn
        p.mul_(beta).add_(zn)
        it += 1
    return done(it, mv, rr, status)


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


def device_operator(prob, stream=None, precision=None):
    """op(u) for a GPU rank: the library's matrix-free operator on the slab's
    icb_problem (density already set), on SoA tensors of the device: FP64
    (float64 tensors) by default, the FP32 CUDA-core operator (float32
    tensors) with precision=MIXED"""
    from . import FP64, MIXED
    precision = FP64 if precision is None else precision
    dt = torch.float64 if precision == FP64 else torch.float32
    if precision not in (FP64, MIXED):
        raise ValueError("precision must be FP64 or MIXED")

    def op(u):
        if u.dtype != dt or not u.is_contiguous():
            raise ValueError("operator input must be a contiguous %s tensor" % dt)
        y = torch.empty_like(u)
        torch.cuda.current_stream().synchronize()
        prob.operator_apply_device(u.data_ptr(), y.data_ptr(), precision)
        prob.ctx.synchronize()
        return y

    return op
