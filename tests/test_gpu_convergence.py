"""Linear MHD waves on the periodic box: the measured L1 convergence order of
the device runs, and the same runs of the reference's own stepping (oracle/_ref,
the unmodified reference sources) with identical states.  The wave setup is
the reference's wave test (file_access.cpp:922-1045): a 1e-6 right-eigenvector
perturbation of the midpoint eigen-system of the background state, along x,
run for one period."""
import math

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from gpu_helpers import gpu_run, linear_wave as _wave, make_ctx, same
from pyoracle import Reference, reference_available

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("wave", [6, 5, 4], ids=["fast", "alfven", "slow"])
def test_linear_wave_convergence_order(wave):
    errs = []
    for n in (16, 32, 64):
        p, speed = _wave(n, wave)
        period = 1.0 / speed
        kw = dict(dt_min=1e-9, dt_max=period / 16.0, cfl=0.4)
        ctx = make_ctx(p, flags=0, **kw)
        r = gpu_run(ctx, period / 64.0, t_max=period)
        assert r["status"] == M.OK and abs(r["t"] - period) <= 1e-12 * period
        U = ctx.download()
        if reference_available():  # the reference's own main-loop stepping, same deck
            Ur = p.U.copy()
            rr = Reference().run(M.ENO_ROE, M.RK3, Ur, p.dx, p.dy, p.gamma, p.bc,
                                 period / 64.0, 1e-9, period / 16.0, 0.4, t_max=period)
            assert rr["steps"] == r["steps"] and rr["t"] == r["t"]
            assert same(U[:, 2:-2, 2:-2], Ur[:, 2:-2, 2:-2])
        # L1 error of the whole state after one period (the exact solution is U0)
        errs.append(np.abs(U[:, 2:-2, 2:-2] - p.U[:, 2:-2, 2:-2]).sum() * p.dx * p.dy)
    o1, o2 = math.log2(errs[0] / errs[1]), math.log2(errs[1] / errs[2])
    # the reference's own runs of this deck measure 2.33 and 2.60 for every wave,
    # and the device's errors are the same numbers
    assert abs(o1 - 2.33) < 0.01 and abs(o2 - 2.60) < 0.01, (errs, o1, o2)
