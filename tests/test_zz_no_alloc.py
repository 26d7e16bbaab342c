"""mhd_divb_calc_noalloc: the div B diagnostic for callers that cannot
allocate device memory (plug-ins inside applications that own all device
memory through their own pool, runtimes that forbid allocation once running,
because cudaMalloc can synchronise the device and stall other streams).

The caller owns the state and the 2-double result on the device; the entry
point's own scratch is a fixed device array inside the library.  Checked
through the C ABI against the allocating entry point (mhd_divb_calc) on the
same state, twice in a row, so the second call reuses the scratch the first
one left behind.  Kept in a file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bc", [(1, 1, 1, 1), (3, 4, 1, 2), (1, 3, 4, 1)])
def test_divb_noalloc_matches_allocating_entry_point(bc):
    import torch

    torch.cuda.init()
    p = P.random_blocky(130, 97, seed=11 + bc[1], bc=bc)
    ctx = M.Context(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, flags=0)
    ctx.upload(p.U)
    if 2 in bc:
        ctx.init_dirichlet()
    m_ref, t_ref = ctx.divb_calc()
    U_ref = ctx.download()  # with the periodic B ghosts the call wrote

    lib = M.library()
    NY = p.ny + 4
    U_dev = torch.from_numpy(p.U.copy()).cuda()  # the reference's dense layout
    result = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    bcs = (C.c_int * 4)(*bc)
    for _ in range(2):  # the second call runs on the scratch the first one left behind
        st = lib.mhd_divb_calc_noalloc(C.c_void_p(U_dev.data_ptr()), p.nx, p.ny, NY, 0, p.dx,
                                       p.dy, bcs, C.c_void_p(result.data_ptr()), None)
        assert st == M.OK
        torch.cuda.synchronize()
        m, t = result.cpu().tolist()
        assert m == m_ref
        assert abs(t - t_ref) <= 1e-12 * abs(t_ref)
        assert np.array_equal(U_dev.cpu().numpy(), U_ref)
        result.fill_(-1.0)
    ctx.close()


def test_divb_noalloc_rejects_oversized_grid():
    lib = M.library()
    bcs = (C.c_int * 4)(1, 1, 1, 1)
    st = lib.mhd_divb_calc_noalloc(C.c_void_p(1), 16385, 8, 12, 0, 1.0, 1.0, bcs, C.c_void_p(1),
                                   None)
    assert st == M.ERR_WRONG_PARAMETER
