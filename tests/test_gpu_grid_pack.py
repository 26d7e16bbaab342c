"""The device grid-dump pack (mhd_grid_pack) against the reference's own
writer (outputGridData -> outputGridDataBinary through
oracle/_ref/libmhdrefio.so) on the same device state: the bytes the reference
fwrites, for doubles and floats, every output category mix and boundary mix,
after steps of the ENO-Roe and ENO-LF schemes."""
import ctypes as C

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from gpu_helpers import make_ctx, same
from pyoracle import grid_writer_available, ref_grid_records

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not grid_writer_available(),
                                 reason="oracle/_ref/libmhdrefio.so not built")]

BCS = [
    (M.PERIODIC,) * 4,
    (M.NEUMANN, M.OPEN, M.DIRICHLET, M.PERIODIC),
    (M.OPEN, M.NEUMANN, M.PERIODIC, M.DIRICHLET),
    (M.DIRICHLET,) * 4,
]


def _stepped(p, scheme, nsteps):
    ctx = make_ctx(p, scheme=scheme, dt_max=0.01)
    dt = 1e-3
    for _ in range(nsteps):
        st, dt = ctx.step(dt)
        assert not st.isError
    return ctx


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("scheme", [M.ENO_ROE, M.ENO_LF])
def test_grid_pack_matches_reference_writer(bc, scheme):
    p = P.random_smooth(37, 29, seed=6, bc=bc)
    ctx = _stepped(p, scheme, 3)
    U = ctx.download()
    for natural, conservation in [(1, 1), (1, 0), (0, 1), (0, 0)]:
        for single in (0, 1):
            got = ctx.grid_records(natural, conservation, single, -2.0, 0.25)
            want = ref_grid_records(U, p.dx, p.dy, p.gamma, bc, -2.0, 0.25, natural,
                                    conservation, not single)
            assert got == want, (natural, conservation, single)
    assert same(ctx.download(), U)  # the pack leaves the state as it was
    ctx.close()


def test_grid_pack_blocky_state_and_sizes():
    """A shocked state at a larger, non-square size; the size query and the
    too-small-buffer status."""
    bc = (M.OPEN, M.OPEN, M.NEUMANN, M.NEUMANN)
    p = P.random_blocky(300, 170, seed=8, bc=bc)
    ctx = _stepped(p, M.ENO_ROE, 2)
    U = ctx.download()
    got = ctx.grid_records(1, 1, 0, 0.0, 0.0)
    assert len(got) == 15 * 300 * 170 * 8
    assert got == ref_grid_records(U, p.dx, p.dy, p.gamma, bc, 0.0, 0.0, 1, 1, True)
    gp = M.GridPackParams(1, 0, 1, 0.0, 0.0)
    n = C.c_size_t(0)
    assert ctx.lib.mhd_grid_pack(ctx.h, C.byref(gp), None, 0, C.byref(n)) == M.OK
    assert n.value == 11 * 300 * 170 * 4
    small = (C.c_char * (n.value - 1))()
    assert ctx.lib.mhd_grid_pack(ctx.h, C.byref(gp), small, n.value - 1, None) == \
        M.ERR_WRONG_PARAMETER
    ctx.close()
