"""mhd_divb_calc_noalloc: the div B diagnostic for callers that cannot
allocate device memory (plug-ins inside applications that own all device
memory through their own pool, runtimes that forbid allocation once running,
because cudaMalloc can synchronise the device and stall other streams).

The caller owns the state and the 2-double result on the device; the entry
point's own scratch is a fixed device array inside the library.  Checked
through the C ABI against the allocating entry point (mhd_divb_calc) on the
same state, twice in a row, so the second call reuses the scratch the first
one left behind; in the reference's dense layout and in a pitched layout
with a row offset; at the largest accepted row count and with no interior
row at all.  The device's free memory must not move across calls.  Kept in a
file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P

pytestmark = pytest.mark.gpu

MAX_ROWS = 16384


def _reference_result(p, bc):
    """max, integral and the state with the periodic B ghosts written, from
    the allocating entry point."""
    ctx = M.Context(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, flags=0)
    try:
        ctx.upload(p.U)
        if 2 in bc:
            ctx.init_dirichlet()
        m_ref, t_ref = ctx.divb_calc()
        return m_ref, t_ref, ctx.download()
    finally:
        ctx.close()


def _pitched(U, row_offset, pad):
    """U copied into a device block whose rows hold `row_offset` unused
    doubles before and `pad` after the reference's row of ny + 4."""
    import torch

    K, NX, NY = U.shape
    pitch = NY + row_offset + pad
    host = np.full((K, NX, pitch), 7.0)  # filler outside the rows
    host[:, :, row_offset:row_offset + NY] = U
    return torch.from_numpy(host).cuda(), pitch


def _call(lib, U_dev, p, pitch, row_offset, bc, result):
    bcs = (C.c_int * 4)(*bc)
    return lib.mhd_divb_calc_noalloc(C.c_void_p(U_dev.data_ptr()), p.nx, p.ny, pitch, row_offset,
                                     p.dx, p.dy, bcs, C.c_void_p(result.data_ptr()), None)


def _check_twice(p, bc, row_offset=0, pad=0, tol=1e-12):
    import torch

    torch.cuda.init()
    m_ref, t_ref, U_ref = _reference_result(p, bc)
    lib = M.library()
    U_dev, pitch = _pitched(p.U.copy(), row_offset, pad)
    result = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the second call runs on the scratch the first one left behind
        assert _call(lib, U_dev, p, pitch, row_offset, bc, result) == M.OK
        torch.cuda.synchronize()
        m, t = result.cpu().tolist()
        assert m == m_ref
        assert abs(t - t_ref) <= tol * abs(t_ref)
        back = U_dev.cpu().numpy()
        assert np.array_equal(back[:, :, row_offset:row_offset + p.ny + 4], U_ref)
        if row_offset or pad:  # nothing outside the caller's rows is touched
            assert np.all(back[:, :, :row_offset] == 7.0)
            assert np.all(back[:, :, row_offset + p.ny + 4:] == 7.0)
        result.fill_(-1.0)


@pytest.mark.parametrize("bc", [(1, 1, 1, 1), (3, 4, 1, 2), (1, 3, 4, 1)])
def test_divb_noalloc_matches_allocating_entry_point(bc):
    p = P.random_blocky(130, 97, seed=11 + bc[1], bc=bc)
    _check_twice(p, bc)


def test_divb_noalloc_pitched_rows_with_offset():
    bc = (1, 3, 1, 4)
    p = P.random_blocky(67, 45, seed=5, bc=bc)
    _check_twice(p, bc, row_offset=14, pad=9)


def test_divb_noalloc_largest_accepted_grid():
    bc = (1, 1, 3, 3)
    p = P.random_blocky(MAX_ROWS, 6, seed=3, bc=bc)
    _check_twice(p, bc)


def test_divb_noalloc_no_interior_row():
    """nx = 2 with both x sides non-periodic: divBCalculation's loops are
    empty and it reports 0 and 0; so must the entry point, with no error."""
    import torch

    bc = (3, 4, 1, 1)
    p = P.random_blocky(2, 9, seed=4, bc=bc)
    m_ref, t_ref, _ = _reference_result(p, bc)
    assert m_ref == 0.0 and t_ref == 0.0
    lib = M.library()
    U_dev, pitch = _pitched(p.U.copy(), 0, 0)
    result = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):
        assert _call(lib, U_dev, p, pitch, 0, bc, result) == M.OK
        torch.cuda.synchronize()
        assert result.cpu().tolist() == [0.0, 0.0]
        result.fill_(-1.0)


def test_divb_noalloc_allocates_nothing():
    """After a first call (which may load the library's device code and its
    scratch array), further calls leave the device's free memory as it was."""
    import torch

    bc = (1, 1, 1, 1)
    p = P.random_blocky(256, 128, seed=9, bc=bc)
    lib = M.library()
    U_dev, pitch = _pitched(p.U.copy(), 0, 0)
    result = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _call(lib, U_dev, p, pitch, 0, bc, result) == M.OK
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for _ in range(20):
        assert _call(lib, U_dev, p, pitch, 0, bc, result) == M.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before


def test_divb_noalloc_rejects_oversized_grid():
    lib = M.library()
    bcs = (C.c_int * 4)(1, 1, 1, 1)
    st = lib.mhd_divb_calc_noalloc(C.c_void_p(1), MAX_ROWS + 1, 8, 12, 0, 1.0, 1.0, bcs,
                                   C.c_void_p(1), None)
    assert st == M.ERR_WRONG_PARAMETER
