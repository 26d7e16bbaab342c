"""mhd_step_host, the step through host memory (the end-to-end call of the
bench): with the banded copies (the first spatial operator follows the
copied row bands; with RK3 the copy back follows the last operator's row
bands) and with one copy each way, against device-resident steps, bit for
bit, including the characteristics of an Euler step, the step's dt and RK3
retries (the copy back is discarded and repeated)."""
import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from gpu_helpers import make_ctx, same

pytestmark = pytest.mark.gpu

BCS = [
    (M.PERIODIC,) * 4,
    (M.NEUMANN, M.OPEN, M.DIRICHLET, M.PERIODIC),
    (M.OPEN, M.NEUMANN, M.NEUMANN, M.OPEN),
    (M.DIRICHLET,) * 4,
]


def _host_steps(p, banded, nsteps, **kw):
    ctx = make_ctx(p, **kw)
    ctx.set_step_host_banded(banded)
    U = np.ascontiguousarray(p.U.copy())
    dt, dts = 1e-3, []
    for _ in range(nsteps):
        st, dt = ctx.step_host(U, dt)
        assert not st.isError
        dts.append(dt)
    chars = ctx.characteristics() if kw.get("flags", 0) & M.FLAG_CHARACTERISTICS else None
    ctx.close()
    return U, dts, chars


def _device_steps(p, nsteps, **kw):
    ctx = make_ctx(p, **kw)
    dt, dts = 1e-3, []
    for _ in range(nsteps):
        st, dt = ctx.step(dt)
        assert not st.isError
        dts.append(dt)
    U = ctx.download()
    chars = ctx.characteristics() if kw.get("flags", 0) & M.FLAG_CHARACTERISTICS else None
    ctx.close()
    return U, dts, chars


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", [(320, 96), (231, 130)])
def test_step_host_banded_matches_device_steps(bc, shape):
    """ENO-Roe RK3 on grids of 33 to 46 tile rows: the banded copy, one copy
    and device-resident steps give the same states and dts."""
    p = P.random_smooth(*shape, seed=sum(bc) + shape[0], bc=bc)
    kw = dict(scheme=M.ENO_ROE, dt_max=0.01, flags=0)
    Ub, db, _ = _host_steps(p, True, 4, **kw)
    Uo, do, _ = _host_steps(p, False, 4, **kw)
    Ud, dd, _ = _device_steps(p, 4, **kw)
    assert db == do == dd
    assert same(Ub, Uo)  # ghost cells included
    assert same(Ub[:, 2:-2, 2:-2], Ud[:, 2:-2, 2:-2])
    assert same(Uo[:, 2:-2, 2:-2], Ud[:, 2:-2, 2:-2])


def test_step_host_lf_copy_back_bands():
    """ENO-LF (its dissipation coefficients come from the whole grid before
    the first flux) copies the state in with one copy; the copy back follows
    the last operator's bands: the same states and dts as one copy each way
    and as device-resident steps."""
    bc = (M.PERIODIC, M.PERIODIC, M.NEUMANN, M.OPEN)
    p = P.random_smooth(300, 64, seed=11, bc=bc)
    kw = dict(scheme=M.ENO_LF, dt_max=0.01, flags=0)
    Ub, db, _ = _host_steps(p, True, 3, **kw)
    Uo, do, _ = _host_steps(p, False, 3, **kw)
    Ud, dd, _ = _device_steps(p, 3, **kw)
    assert db == do == dd
    assert same(Ub, Uo)
    assert same(Ub[:, 2:-2, 2:-2], Ud[:, 2:-2, 2:-2])


@pytest.mark.parametrize("scheme", [M.ENO_ROE, M.ENO_LF])
def test_step_host_copy_back_with_rk3_retries(scheme):
    """An explosion on 256 x 240 cells (open sides) from dt = dt_max: its
    wave speeds grow within the first steps, so RK3 stages ask for retries
    (seen as steps with more launches).  After a retry the banded copy back
    is discarded and the state copied again: states and dts equal one copy
    each way and device-resident steps; the characteristics of the last
    stage too."""
    p = P.explosion(256, 240)
    dtm = 0.02 / 16
    kw = dict(scheme=scheme, dt_min=1e-9, dt_max=dtm, cfl=0.4, flags=M.FLAG_CHARACTERISTICS)
    res = []
    for banded in (True, False):
        ctx = make_ctx(p, **kw)
        ctx.set_step_host_banded(banded)
        U = np.ascontiguousarray(p.U.copy())
        dt, dts = dtm, []
        for _ in range(4):
            st, dt = ctx.step_host(U, dt)
            assert not st.isError
            dts.append(dt)
        res.append((U, dts, ctx.characteristics()))
        ctx.close()
    ctx = make_ctx(p, **kw)
    dt, dts, per_step = dtm, [], []
    for _ in range(4):
        l0 = ctx.counters()["launches"]
        st, dt = ctx.step(dt)
        assert not st.isError
        per_step.append(ctx.counters()["launches"] - l0)
        dts.append(dt)
    Ud, cd = ctx.download(), ctx.characteristics()
    ctx.close()
    assert max(per_step) > min(per_step), "no RK3 retry in these steps"
    (Ub, db, cb), (Uo, do, co) = res
    assert db == do == dts
    assert same(Ub, Uo)
    assert same(Ub[:, 2:-2, 2:-2], Ud[:, 2:-2, 2:-2])
    for a, b, d in zip(cb, co, cd):
        assert same(a, b) and same(a, d)


def test_step_host_banded_euler_characteristics_and_blocky_state():
    """Euler with the characteristics flag (the first operator keeps them) on a
    shocked state; the banded copy keeps them bit for bit."""
    bc = (M.NEUMANN, M.NEUMANN, M.PERIODIC, M.PERIODIC)
    p = P.random_blocky(300, 128, seed=3, bc=bc)
    kw = dict(scheme=M.ENO_ROE, time_method=M.EULER, dt_max=0.002,
              flags=M.FLAG_CHARACTERISTICS)
    Ub, db, cb = _host_steps(p, True, 3, **kw)
    Ud, dd, cd = _device_steps(p, 3, **kw)
    assert db == dd
    assert same(Ub[:, 2:-2, 2:-2], Ud[:, 2:-2, 2:-2])
    for a, b in zip(cb, cd):
        assert same(a, b)
