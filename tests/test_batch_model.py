"""The index arithmetic behind the batched launches, restated on the CPU.

Three things the fused batch relies on for bitwise-equal results and for
race-free writes, checked over awkward sizes with the launchers' formulas
transcribed from the sources:

* the Q4 operator's fused dot (operator.cu, q4_body): one slot per (node row,
  warp strip); for every cut of the rows into blocks (the per-design grid of
  q4_grid and any rows-per-item a batched launch picks) each slot is written
  exactly once, so the slot-order sum is the same;
* the prolongation (mg_impl.cuh, prolong_rows_b): groups of kProlongRows node
  rows per thread, in the per-design grid and in the batched work items
  (ProlongL, rows per item a multiple of the group): every fine node row is
  processed exactly once and no coarse row index leaves the coarse grid;
* the tiled OC step (opt.cu, oc_step_tile_b): 32 x 32-element tiles, four rows
  per thread; every element belongs to exactly one (tile, thread, row) and
  every stencil read of the staged tile stays inside it.
No GPU.
"""
import numpy as np
import pytest

TX, TY2 = 32, 4          # operator.cu: threads along x (one warp), warps per 2D CTA
SMS = 148
PROLONG_ROWS = 4         # mg_impl.cuh: kProlongRows
OC_TW, OC_TH, OC_HALO, VB = 32, 32, 8, 256   # opt.cu


def _q4_grid(sx, sy, sms=SMS):
    """operator.cu q4_grid: (bx, by, ychunk) of a design's own launch"""
    target = sms * 4
    strips = (sx + TX - 2) // (TX - 1)
    bx = (strips + TY2 - 1) // TY2
    by = max(1, min(sy, (target + bx - 1) // bx))
    ychunk = (sy + by - 1) // by
    by = (sy + ychunk - 1) // ychunk
    return bx, by, ychunk


def _dot_slot_writes(sx, sy, ychunk):
    bx, _, _ = _q4_grid(sx, sy)
    by = (sy + ychunk - 1) // ychunk
    strips = bx * TY2
    cnt = np.zeros(sy * strips, np.int32)
    for byi in range(by):
        y0, y1 = byi * ychunk, min(byi * ychunk + ychunk, sy) - 1
        for bxi in range(bx):
            for w in range(TY2):
                strip = bxi * TY2 + w
                for ej in range(y0, y1 + 1):  # rows with ej >= Y0 write their slot
                    cnt[ej * strips + strip] += 1
    return cnt


@pytest.mark.parametrize("nx,ny", [(1, 1), (12, 5), (31, 8), (32, 64), (62, 17), (150, 40),
                                   (513, 257), (1024, 300)])
def test_q4_dot_slots_written_once_for_every_row_cut(nx, ny):
    sx, sy = nx + 1, ny + 1
    _, _, natural = _q4_grid(sx, sy)
    for ychunk in sorted({natural, 1, 2, 3, 7, 16, sy}):
        cnt = _dot_slot_writes(sx, sy, ychunk)
        assert (cnt == 1).all(), (nx, ny, ychunk)


def _prolong_rows(fine_sy, sh_y, row_groups):
    """fine rows processed (with their coarse rows J0, J1) by groups starting
    at the given rows"""
    coarse_sy = (fine_sy // 2 + 1) if sh_y else fine_sy  # ceil(ny / 2) + 1 coarse node rows
    seen = np.zeros(fine_sy, np.int32)
    for j0 in row_groups:
        for r in range(PROLONG_ROWS):
            j = j0 + r
            if j >= fine_sy:  # fx = 7: nothing to do
                continue
            seen[j] += 1
            J0, J1 = j >> sh_y, (j + sh_y) >> sh_y
            assert 0 <= J0 < coarse_sy and 0 <= J1 < coarse_sy
    return seen


@pytest.mark.parametrize("ny,sh_y", [(ny, 1) for ny in (1, 2, 3, 4, 7, 8, 16, 31, 64, 129, 256)]
                         + [(1, 0)])  # an axis is kept only when it is one element thick
def test_prolongation_row_groups_cover_every_row_once(ny, sh_y):
    fine_sy = ny + 1
    # the design's own launch: gridDim.y = ceil(sy / kProlongRows), group = blockIdx.y
    own = [b * PROLONG_ROWS for b in range((fine_sy + PROLONG_ROWS - 1) // PROLONG_ROWS)]
    assert (_prolong_rows(fine_sy, sh_y, own) == 1).all()
    # batched items: ry = kP * kProlongRows rows each, groups of kProlongRows inside
    for kp in (1, 2, 3, 4):
        ry = kp * PROLONG_ROWS
        groups = []
        for item in range((fine_sy + ry - 1) // ry):
            j1 = min(fine_sy, (item + 1) * ry)
            groups += list(range(item * ry, j1, PROLONG_ROWS))
        assert (_prolong_rows(fine_sy, sh_y, groups) == 1).all(), (ny, kp)


def _cone_offsets(radius):
    R = int(np.floor(radius)) + 1
    return [(di, dj) for dj in range(-R, R + 1) for di in range(-R, R + 1)
            if np.hypot(di, dj) <= radius]


@pytest.mark.parametrize("nx,ny,radius", [(1, 1, 1.2), (5, 3, 1.5), (32, 32, 4.0), (33, 31, 2.5),
                                          (100, 45, 3.0), (64, 1, 1.2), (1, 70, 2.0),
                                          (130, 97, 6.9)])
def test_oc_tiles_cover_every_element_once_and_stay_in_the_tile(nx, ny, radius):
    offs = _cone_offsets(radius)
    hx = max(abs(o[0]) for o in offs)
    hy = max(abs(o[1]) for o in offs)
    assert hx <= OC_HALO and hy <= OC_HALO  # the tiled form's limit (oc_tiling)
    twp, thp = OC_TW + 2 * hx, OC_TH + 2 * hy
    # the staged tile fits the loads a thread issues (kPer) and the table (kTab)
    assert twp * thp <= ((OC_TW + 2 * OC_HALO) * (OC_TH + 2 * OC_HALO) + VB - 1) // VB * VB
    assert len(offs) <= ((2 * OC_HALO + 1) ** 2 + VB - 1) // VB * VB
    ntx, nty = (nx + OC_TW - 1) // OC_TW, (ny + OC_TH - 1) // OC_TH
    cnt = np.zeros((ny, nx), np.int32)
    t = np.arange(VB)
    tx, ty = t & 31, t >> 5
    for b in range(ntx * nty):
        x0, y0 = (b % ntx) * OC_TW, (b // ntx) * OC_TH
        for k in range(OC_TH // 8):
            i, j = x0 + tx, y0 + ty + 8 * k
            inside = (i < nx) & (j < ny)
            np.add.at(cnt, (j[inside], i[inside]), 1)
            c0 = (ty + hy + 8 * k) * twp + tx + hx
            for di, dj in offs:
                q = c0 + dj * twp + di
                # every neighbour read of the staged tile lies inside it and holds
                # element (i + di, j + dj) (the staged value is 0 outside the grid)
                assert ((q >= 0) & (q < twp * thp)).all()
                qy, qx = np.divmod(q, twp)
                assert (x0 - hx + qx == i + di).all() and (y0 - hy + qy == j + dj).all()
    assert (cnt == 1).all()
