"""Problem builders shared by the tests and bench.py: the same boundary
conditions, loads and seeded densities on the oracle and on the library.

Workloads (sizes as stated; all inputs synthetic and seeded):
  cantilever2d  120x40 unit Q4 plane stress, E0 = 1, Emin = 1e-9, nu = 0.3,
                p = 3, x = 0 edge clamped, unit downward point load at the
                right-edge mid node.
  cantilever3d  192x64x64 unit Hex8, x = 0 face clamped, unit line load per
                length in -z along the bottom edge (z = 0) of the x = L face:
                0.5 on the two end nodes, 1.0 on the interior nodes.
  halfmbb2d     2D half-MBB beam: ux = 0 on x = 0, uy = 0 at the bottom-right
                node, unit downward load at the top-left node.
  halfmbb3d     384x128x128 Hex8 half-MBB beam (ux = 0 on x = 0, uz = 0 on
                the line x = L, z = 0, uy = 0 on y = 0; line load in -z along
                x = 0, z = H).
  strip2d       a long Q4 strip clamped along its bottom edge (y = 0), unit
                downward load at the top-edge middle node, 0.5 along x at the
                top node at x = L/4 (thin grids that stay well conditioned).
"""
import numpy as np

E0, EMIN, NU, PENAL = 1.0, 1e-9, 0.3, 3.0


def _mask_cantilever2d(nx, ny):
    fixed = np.zeros((ny + 1, nx + 1, 2), np.uint8)
    fixed[:, 0, :] = 1
    f = np.zeros((ny + 1, nx + 1, 2))
    f[ny // 2, nx, 1] = -1.0
    return fixed.reshape(-1), f.reshape(-1)


def _mask_cantilever3d(nx, ny, nz):
    fixed = np.zeros((nz + 1, ny + 1, nx + 1, 3), np.uint8)
    fixed[:, :, 0, :] = 1
    f = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    f[0, :, nx, 2] = -1.0
    f[0, 0, nx, 2] = f[0, ny, nx, 2] = -0.5
    return fixed.reshape(-1), f.reshape(-1)


def _mask_halfmbb3d(nx, ny, nz):
    fixed = np.zeros((nz + 1, ny + 1, nx + 1, 3), np.uint8)
    fixed[:, :, 0, 0] = 1          # symmetry plane x = 0
    fixed[0, :, nx, 2] = 1         # roller line x = L, z = 0
    fixed[:, 0, :, 1] = 1          # y = 0 face
    f = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    f[nz, :, 0, 2] = -1.0
    f[nz, 0, 0, 2] = f[nz, ny, 0, 2] = -0.5
    return fixed.reshape(-1), f.reshape(-1)


def _mask_halfmbb2d(nx, ny):
    fixed = np.zeros((ny + 1, nx + 1, 2), np.uint8)
    fixed[:, 0, 0] = 1          # symmetry edge x = 0
    fixed[0, nx, 1] = 1         # roller at the bottom-right corner
    f = np.zeros((ny + 1, nx + 1, 2))
    f[ny, 0, 1] = -1.0
    return fixed.reshape(-1), f.reshape(-1)


def _mask_strip2d(nx, ny):
    fixed = np.zeros((ny + 1, nx + 1, 2), np.uint8)
    fixed[0, :, :] = 1
    f = np.zeros((ny + 1, nx + 1, 2))
    f[ny, nx // 2, 1] = -1.0
    f[ny, nx // 4, 0] = 0.5
    return fixed.reshape(-1), f.reshape(-1)


def masks(kind, nx, ny, nz=1):
    if kind == "strip2d":
        return _mask_strip2d(nx, ny)
    if kind == "halfmbb2d":
        return _mask_halfmbb2d(nx, ny)
    if kind == "cantilever2d":
        return _mask_cantilever2d(nx, ny)
    if kind == "cantilever3d":
        return _mask_cantilever3d(nx, ny, nz)
    if kind == "halfmbb3d":
        return _mask_halfmbb3d(nx, ny, nz)
    raise ValueError(kind)


def smooth_field(nx, ny, nz, seed, lo=0.001, hi=1.0, modes=16):
    """Seeded smooth random density: affine map to [lo, hi] of
    sum_k a_k cos(2 pi (k . x_c / L) + phi_k), k integer triples in [0,4]^3,
    a_k ~ N(0,1), phi_k ~ U[0, 2 pi), at element centres."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    f = np.zeros((nz, ny, nx))
    for _ in range(modes):
        k = rng.integers(0, 5, 3)
        a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
        # separable evaluation of cos(2 pi (kx x + ky y + kz z) + ph)
        cx, sx = np.cos(2 * np.pi * k[0] * x), np.sin(2 * np.pi * k[0] * x)
        cy, sy = np.cos(2 * np.pi * k[1] * y), np.sin(2 * np.pi * k[1] * y)
        cz, sz = np.cos(2 * np.pi * k[2] * z + ph), np.sin(2 * np.pi * k[2] * z + ph)
        cxy = np.outer(cy, cx) - np.outer(sy, sx)
        sxy = np.outer(sy, cx) + np.outer(cy, sx)
        f += a * (cz[:, None, None] * cxy[None] - sz[:, None, None] * sxy[None])
    f = (f - f.min()) / max(f.max() - f.min(), 1e-300)
    return (lo + (hi - lo) * f).reshape(-1)


def uniform_density(nel, seed, lo=0.01, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, nel)


def build_oracle(kind, nx, ny, nz=1):
    import pyoracle as po
    dim = 2 if kind.endswith("2d") else 3
    p = po.Problem(dim, nx, ny, nz, young=(EMIN, E0), nu=NU, penal=PENAL)
    fixed, f = masks(kind, nx, ny, nz)
    p.fixed[:] = fixed
    p.fext_full[:] = f
    return p


def build_gpu(ctx, kind, nx, ny, nz=1):
    import icarat_b200 as icb
    dim = 2 if kind.endswith("2d") else 3
    p = icb.Problem(ctx, dim, nx, ny, nz, young=(EMIN, E0), nu=NU, penal=PENAL)
    fixed, f = masks(kind, nx, ny, nz)
    p.dirichlet_mask(fixed)
    nodes = np.nonzero(np.abs(f.reshape(-1, dim)).sum(1))[0]
    for n in nodes:
        p.nodal_load(n, f.reshape(-1, dim)[n])
    p.finalize()
    return p


# ------------------------------------------------------- batched / served --
def _edge_mask2d(nx, ny, edge):
    fixed = np.zeros((ny + 1, nx + 1, 2), np.uint8)
    if edge == 0:
        fixed[:, 0, :] = 1
    elif edge == 1:
        fixed[:, nx, :] = 1
    elif edge == 2:
        fixed[0, :, :] = 1
    else:
        fixed[ny, :, :] = 1
    return fixed


def random_instance2d(rng, nelx_range=(64, 1024), aspect_range=(1.0, 4.0), vf_range=(0.2, 0.6),
                      r_range=(1.2, 4.0), aspect_fixed=None):
    """One batched/served 2D instance: nelx log-uniform, aspect uniform (or
    fixed), a random clamped edge, 1-4 unit point loads (direction uniform on
    the circle) at random boundary nodes off the clamped edge."""
    lo, hi = nelx_range
    nx = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
    a = aspect_fixed if aspect_fixed else rng.uniform(*aspect_range)
    ny = max(1, int(round(nx / a)))
    vf, r = rng.uniform(*vf_range), rng.uniform(*r_range)
    edge = int(rng.integers(4))
    fixed = _edge_mask2d(nx, ny, edge)
    boundary = [(j, i) for j in range(ny + 1) for i in range(nx + 1)
                if (i in (0, nx) or j in (0, ny)) and not fixed[j, i].any()]
    load = np.zeros((ny + 1, nx + 1, 2))
    for k in rng.choice(len(boundary), size=int(rng.integers(1, 5)), replace=False):
        j, i = boundary[k]
        th = rng.uniform(0, 2 * np.pi)
        load[j, i] += (np.cos(th), np.sin(th))
    return dict(dim=2, nx=nx, ny=ny, nz=1, vf=vf, r=r, fixed=fixed.reshape(-1),
                load=load.reshape(-1))


def random_instance3d(rng, nelx_range=(32, 128), vf_range=(0.2, 0.5), r_range=(1.5, 3.0)):
    """A served 3D job: nelx uniform, nely = nelz = nelx/2, x = 0 clamped,
    1-4 unit loads in random directions at random nodes of the x = L face."""
    nx = int(rng.integers(nelx_range[0], nelx_range[1] + 1))
    ny = nz = max(1, nx // 2)
    fixed = np.zeros((nz + 1, ny + 1, nx + 1, 3), np.uint8)
    fixed[:, :, 0, :] = 1
    load = np.zeros((nz + 1, ny + 1, nx + 1, 3))
    for _ in range(int(rng.integers(1, 5))):
        v = rng.standard_normal(3)
        load[rng.integers(nz + 1), rng.integers(ny + 1), nx] += v / np.linalg.norm(v)
    return dict(dim=3, nx=nx, ny=ny, nz=nz, vf=rng.uniform(*vf_range), r=rng.uniform(*r_range),
                fixed=fixed.reshape(-1), load=load.reshape(-1))


def grid_desc(inst):
    import icarat_b200 as icb
    d = inst["dim"]
    return icb.GridDesc(d, inst["nx"], inst["ny"], inst["nz"] if d == 3 else 1,
                        float(inst["nx"]), float(inst["ny"]), float(inst["nz"] if d == 3 else 1),
                        icb.THREE_D if d == 3 else icb.PLANE_STRESS, EMIN, E0, NU, PENAL)


def build_instance(ctx, inst):
    import icarat_b200 as icb
    d = inst["dim"]
    p = icb.Problem(ctx, d, inst["nx"], inst["ny"], inst["nz"], young=(EMIN, E0), nu=NU, penal=PENAL)
    p.dirichlet_mask(inst["fixed"])
    L = inst["load"].reshape(-1, d)
    for n in np.nonzero(np.abs(L).sum(1))[0]:
        p.nodal_load(n, L[n])
    p.finalize()
    return p
