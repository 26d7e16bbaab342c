"""The reference's binary grid dump (outputGridData -> outputGridDataBinary,
file_access.cpp:1193-1325 and 1530-1677, after toNaturalData,
conversions.cpp:37-57), driven through oracle/_ref/libmhdrefio.so, against a
numpy restatement of its record layout and div B rules.  This pins the
checker that tests/test_gpu_grid_pack.py holds the device pack to."""
import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from pyoracle import grid_writer_available, ref_grid_records

pytestmark = pytest.mark.skipif(not grid_writer_available(),
                                reason="oracle/_ref/libmhdrefio.so not built")

BCS = [
    (M.PERIODIC,) * 4,
    (M.NEUMANN, M.OPEN, M.DIRICHLET, M.PERIODIC),
    (M.OPEN, M.NEUMANN, M.PERIODIC, M.DIRICHLET),
    (M.DIRICHLET,) * 4,
]


def restated_records(U, dx, dy, gamma, bc, start_x, start_y, natural, conservation):
    """numpy restatement: [nx*ny, fields] float64 in the writer's order."""
    _, NX, NY = U.shape
    nx, ny = NX - 4, NY - 4
    B = U[4:6].copy()
    left, right, bottom, top = bc
    # outputGridData's B ghosts on periodic and open sides, then its ranges
    if left == M.PERIODIC:
        B[:, 0:2, 2:ny + 2] = B[:, nx:nx + 2, 2:ny + 2]
    if left == M.OPEN:
        B[:, 0:2, 2:ny + 2] = B[:, 2:3, 2:ny + 2]
    if right == M.PERIODIC:
        B[:, nx + 2:nx + 4, 2:ny + 2] = B[:, 2:4, 2:ny + 2]
    if right == M.OPEN:
        B[:, nx + 2:nx + 4, 2:ny + 2] = B[:, nx + 1:nx + 2, 2:ny + 2]
    if bottom == M.PERIODIC:
        B[:, 2:nx + 2, 0:2] = B[:, 2:nx + 2, ny:ny + 2]
    if bottom == M.OPEN:
        B[:, 2:nx + 2, 0:2] = B[:, 2:nx + 2, 2:3]
    if top == M.PERIODIC:
        B[:, 2:nx + 2, ny + 2:ny + 4] = B[:, 2:nx + 2, 2:4]
    if top == M.OPEN:
        B[:, 2:nx + 2, ny + 2:ny + 4] = B[:, 2:nx + 2, ny + 1:ny + 2]
    cut = (M.NEUMANN, M.OPEN)
    x0, x1 = (3 if left in cut else 2), (nx + 1 if right in cut else nx + 2)
    y0, y1 = (3 if bottom in cut else 2), (ny + 1 if top in cut else ny + 2)
    divb = np.zeros((NX, NY))
    i, j = np.meshgrid(np.arange(x0, x1), np.arange(y0, y1), indexing="ij")
    divb[x0:x1, y0:y1] = np.abs((B[0][i + 1, j] - B[0][i - 1, j]) / (2.0 * dx)
                                + (B[1][i, j + 1] - B[1][i, j - 1]) / (2.0 * dy))
    s = (slice(2, nx + 2), slice(2, ny + 2))
    r, mx, my, mz = U[0][s], U[1][s], U[2][s], U[3][s]
    bx, by, bz, en = U[4][s], U[5][s], U[6][s], U[7][s]
    ii, jj = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64),
                         indexing="ij")
    cols = [start_x + ii * dx, start_y + jj * dy, r]
    if natural:
        mm = mx * mx + my * my + mz * mz
        bb = bx * bx + by * by + bz * bz
        cols += [mx / r, my / r, mz / r, (gamma - 1.0) * (en - 0.5 * mm / r - 0.5 * bb)]
    cols += [bx, by, bz, divb[s]]
    if conservation:
        cols += [mx, my, mz, en]
    return np.stack([c.reshape(-1) for c in cols], axis=1)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("natural,conservation", [(1, 1), (1, 0), (0, 1), (0, 0)])
def test_reference_writer_matches_restatement(bc, natural, conservation):
    p = P.random_smooth(9, 7, seed=4, bc=bc)
    U = p.U.copy()
    U[4:6] += np.random.default_rng(5).normal(0, 0.1, U[4:6].shape)  # ghosts too
    want = restated_records(U, p.dx, p.dy, p.gamma, bc, -2.0, 0.5, natural, conservation)
    got = ref_grid_records(U, p.dx, p.dy, p.gamma, bc, -2.0, 0.5, natural, conservation, True)
    assert got == want.tobytes()
    got32 = ref_grid_records(U, p.dx, p.dy, p.gamma, bc, -2.0, 0.5, natural, conservation,
                             False)
    assert got32 == want.astype(np.float32).tobytes()
