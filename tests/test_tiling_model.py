"""The operators' tilings, restated on the CPU.

k_matvec_h8 / k_matvec_h8m (Hex8) and k_matvec_q4 (Q4) give each thread one
element column (plus a one-element halo on the low side of its tile) and let
the thread whose column ends at a node write that node; k_matvec_h8p (the FP32
Hex8 default) gives each thread two element rows of a column and writes the
node row between them and the one above; k_helm_apply3 (the
3D Helmholtz operator) gives each thread one node column and stages each plane
with a one-node halo in shared memory.  No atomics: the result is only right
if every node of the grid is written by exactly one thread-layer.  The
launchers' grid arithmetic and the kernels' ownership tests are transcribed
here and checked for exact coverage over awkward sizes (one-element axes,
sizes just past a tile boundary) and every z or y split.  No GPU.
"""
import numpy as np

TX, TY3, TY2 = 32, 8, 4  # operator.cu: threads along x, rows per 3D tile, warps per 2D CTA
HTX, HTY = 32, 8         # helm.cu: the Helmholtz operator's node tile


def _h8_owners(nx, ny, nz, zchunk):
    """count of owning thread-layers per node (sz, sy, sx) for one Hex8 launch"""
    sx, sy, sz = nx + 1, ny + 1, nz + 1
    bx, by = (sx + TX - 2) // (TX - 1), (sy + TY3 - 2) // (TY3 - 1)
    bz = (sz + zchunk - 1) // zchunk
    cnt = np.zeros((sz, sy, sx), np.int32)
    lx = np.arange(TX)[None, :]
    ly = np.arange(TY3)[:, None]
    for byi in range(by):
        for bxi in range(bx):
            ei = bxi * (TX - 1) - 1 + lx
            ej = byi * (TY3 - 1) - 1 + ly
            ni, nj = ei + 1, ej + 1
            own_xy = (lx < TX - 1) & (ly < TY3 - 1) & (ni < sx) & (nj < sy)
            own_xy = np.broadcast_to(own_xy, (TY3, TX))
            ii = np.broadcast_to(ni, (TY3, TX))[own_xy]
            jj = np.broadcast_to(nj, (TY3, TX))[own_xy]
            assert (ii >= 0).all() and (jj >= 0).all()
            for bzi in range(bz):
                z0 = bzi * zchunk
                z1 = min(z0 + zchunk, sz) - 1
                for ek in range(z0 - 1, z1 + 1):
                    if ek >= z0:  # the layer's bottom plane is complete: output it
                        cnt[ek, jj, ii] += 1
    return cnt


TW = 4  # operator.cu kPairWarps: warps of the paired-row FP32 Hex8 kernel


def _h8p_owners(nx, ny, nz, zchunk):
    """k_matvec_h8p: two element rows per thread, a 31 x (2 TW - 1) node tile;
    count of writes per node (sz, sy, sx), and a check that every node a
    thread loads (unguarded by its validity flags) and every shared-memory
    exchange slot it reads are inside their ranges"""
    sx, sy, sz = nx + 1, ny + 1, nz + 1
    bx, by = (sx + TX - 2) // (TX - 1), (sy + 2 * TW - 2) // (2 * TW - 1)
    bz = (sz + zchunk - 1) // zchunk
    cnt = np.zeros((sz, sy, sx), np.int32)
    lx = np.arange(TX)[None, :]
    ly = np.arange(TW)[:, None]
    for byi in range(by):
        for bxi in range(bx):
            X0, Y0 = bxi * (TX - 1), byi * (2 * TW - 1)
            ei = np.broadcast_to(X0 - 1 + lx, (TW, TX))
            ej = np.broadcast_to(Y0 - 1 + 2 * ly, (TW, TX))
            lyb = np.broadcast_to(ly, (TW, TX))
            ni = ei + 1
            ocol = (np.broadcast_to(lx, (TW, TX)) < TX - 1) & (ni < sx)
            own1 = ocol & (ej + 1 >= 0) & (ej + 1 < sy)
            own2 = ocol & (lyb < TW - 1) & (ej + 2 < sy)
            # the row-(j+2) partner read from shared memory: warp ly + 1, same lane
            assert (lyb[own2] + 1 < TW).all()
            for bzi in range(bz):
                z0 = bzi * zchunk
                z1 = min(z0 + zchunk, sz) - 1
                for ek in range(z0 - 1, z1 + 1):
                    if ek >= z0:
                        cnt[ek, (ej + 1)[own1], ni[own1]] += 1
                        cnt[ek, (ej + 2)[own2], ni[own2]] += 1
    return cnt


def test_hex8_paired_tiling_writes_every_node_once():
    sizes = [(1, 1, 1), (1, 6, 5), (30, 14, 1), (31, 15, 2), (32, 16, 3), (62, 30, 4),
             (5, 13, 9), (40, 1, 12), (48, 17, 1), (13, 29, 5), (70, 40, 3)]
    for nx, ny, nz in sizes:
        for zchunk in sorted({1, 2, 3, nz, nz + 1, (nz + 2) // 2}):
            cnt = _h8p_owners(nx, ny, nz, zchunk)
            assert (cnt == 1).all(), (nx, ny, nz, zchunk, cnt.min(), cnt.max())


def _q4_owners(nx, ny, target):
    """count of owning thread-layers per node (sy, sx) for one Q4 launch"""
    sx, sy = nx + 1, ny + 1
    strips = (sx + TX - 2) // (TX - 1)
    bx = (strips + TY2 - 1) // TY2
    by = max(1, min(sy, (target + bx - 1) // bx))
    ychunk = (sy + by - 1) // by
    by = (sy + ychunk - 1) // ychunk
    cnt = np.zeros((sy, sx), np.int32)
    for bxi in range(bx):
        for w in range(TY2):
            x0 = (bxi * TY2 + w) * (TX - 1)
            lx = np.arange(TX)
            ni = x0 - 1 + lx + 1
            own = (lx < TX - 1) & (ni < sx) & (x0 < sx)
            for byi in range(by):
                y0 = byi * ychunk
                y1 = min(y0 + ychunk, sy) - 1
                for ej in range(y0 - 1, y1 + 1):
                    if ej >= y0:
                        cnt[ej, ni[own]] += 1
    return cnt


def test_hex8_tiling_writes_every_node_once():
    sizes = [(1, 1, 1), (1, 6, 5), (30, 6, 1), (31, 7, 2), (32, 8, 3), (62, 14, 4), (5, 13, 9),
             (40, 1, 12), (48, 16, 1), (13, 7, 5)]
    for nx, ny, nz in sizes:
        for zchunk in sorted({1, 2, 3, nz, nz + 1, (nz + 2) // 2}):
            cnt = _h8_owners(nx, ny, nz, zchunk)
            assert (cnt == 1).all(), (nx, ny, nz, zchunk, cnt.min(), cnt.max())


def test_q4_tiling_writes_every_node_once():
    for nx, ny in [(1, 1), (30, 1), (31, 2), (123, 5), (124, 7), (300, 1), (37, 13), (250, 40)]:
        for target in (1, 3, 148 * 4):
            cnt = _q4_owners(nx, ny, target)
            assert (cnt == 1).all(), (nx, ny, target, cnt.min(), cnt.max())


def _helm_owners(sx, sy, sz, zc):
    """count of writes per node (sz, sy, sx) for one k_helm_apply3 launch, and
    a check that the staged plane (tile + one-node halo) is filled completely
    and read inside its bounds"""
    NX, NY, NT = HTX + 2, HTY + 2, HTX * HTY
    tx, ty, bz = (sx + HTX - 1) // HTX, (sy + HTY - 1) // HTY, (sz + zc - 1) // zc
    staged = np.zeros(NX * NY, np.int32)
    for tid in range(NT):
        for t in range(2):
            q = tid + t * NT
            if q < NX * NY:
                staged[q] += 1
    assert (staged == 1).all()  # every halo cell has exactly one loader
    # reads sP[ly + r][lx + c], r, c in 0..2
    assert HTY - 1 + 2 < NY and HTX - 1 + 2 < NX
    cnt = np.zeros((sz, sy, sx), np.int32)
    lx, ly = np.arange(HTX)[None, :], np.arange(HTY)[:, None]
    for byi in range(ty):
        for bxi in range(tx):
            i = np.broadcast_to(bxi * HTX + lx, (HTY, HTX))
            j = np.broadcast_to(byi * HTY + ly, (HTY, HTX))
            own = (i < sx) & (j < sy)
            for bzi in range(bz):
                z0 = bzi * zc
                z1 = min(z0 + zc, sz) - 1
                for k in range(z0 - 1, z1 + 2):
                    ko = k - 1
                    if z0 <= ko <= z1:
                        cnt[ko, j[own], i[own]] += 1
    return cnt


def test_helmholtz_tiling_writes_every_node_once():
    for sx, sy, sz in [(2, 2, 2), (33, 9, 2), (32, 8, 5), (65, 17, 13), (7, 40, 3)]:
        for zc in sorted({1, 2, sz, (sz + 1) // 2}):
            cnt = _helm_owners(sx, sy, sz, zc)
            assert (cnt == 1).all(), (sx, sy, sz, zc)
