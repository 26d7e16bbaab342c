"""Shared helpers of the GPU parity tests (CUDA path through the C ABI)."""
import ctypes as C
import math

import numpy as np

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from pyoracle import load_oracle



def same(a, b):
    """Bitwise equality up to the sign of zero (NaNs compare equal)."""
    return np.array_equal(a, b, equal_nan=True)


def interior(a):
    return a[:, 2:-2, 2:-2]


def make_ctx(p, scheme=M.ENO_ROE, time_method=M.RK3, dt_min=0.0, dt_max=1.0, cfl=0.4,
             flags=M.FLAG_CHARACTERISTICS, U_dirichlet=None):
    c = M.Context(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, scheme=scheme, time_method=time_method,
                  dt_min=dt_min, dt_max=dt_max, cfl=cfl, flags=flags)
    c.upload(p.U if U_dirichlet is None else U_dirichlet)
    c.init_dirichlet()
    c.upload(p.U)
    return c


def gpu_run(ctx, dt0, nsteps=0, t_max=0.0, sor=None, hist_len=256):
    """The reference main loop (main.cpp:174-344, no output) on the device."""
    step, t, dt = 1, 0.0, dt0
    dts, divbs = [], []
    st = None
    while True:
        st, dt = ctx.step(dt)
        if st.status == M.ERR_TIME_UNDERFLOW or st.isError:
            break
        divbmax = -1.0
        if sor is not None and sor.sor_steps > 0 and step % sor.divb_skip_steps == 0:
            _, divbmax, _ = ctx.divb_clean(sor)
        t += dt
        if step <= hist_len:
            dts.append(dt)
            divbs.append(divbmax)
        done = (nsteps > 0 and step == nsteps) or (t_max > 0.0 and t >= t_max)
        if np.isnan(ctx.download()[0, 2, 2]):
            done = True
        step += 1
        if done:
            break
    return dict(status=st.status, is_error=int(st.isError), dt=dt, t=t, steps=step - 1,
                dt_hist=np.array(dts), divb_hist=np.array(divbs))


GAMMA = 5.0 / 3.0
BACKGROUND = (1.0, 0.0, 0.0, 0.0, 1.0, math.sqrt(2.0), 0.5, 1.0 / GAMMA)  # rho u v w Bx By Bz p


def _conserved(q):
    rho, u, v, w, bx, by, bz, p = q
    uu, bb = u * u + v * v + w * w, bx * bx + by * by + bz * bz
    return np.array([rho, u * rho, v * rho, w * rho, bx, by, bz,
                     p / (GAMMA - 1.0) + 0.5 * rho * uu + 0.5 * bb])


def linear_wave(n, wave, eps=1e-6, ny=4):
    """A 1e-6 right-eigenvector perturbation of the midpoint eigen-system of
    the background state along x on the periodic unit box (the reference's
    wave test, file_access.cpp:922-1045); returns the problem and |lambda|."""
    avg = _conserved(BACKGROUND)
    lam, lv, rv = np.zeros(8), np.zeros(64), np.zeros(64)
    npr = C.c_int(0)
    dp = C.POINTER(C.c_double)
    st = load_oracle().orc_eigens_f(C.c_double(GAMMA), avg.ctypes.data_as(dp),
                                    avg.ctypes.data_as(dp), lam.ctypes.data_as(dp),
                                    lv.ctypes.data_as(dp), rv.ctypes.data_as(dp), C.byref(npr))
    assert st == 0
    dx = 1.0 / n
    U = np.zeros((8, n + 4, ny + 4))
    x = -0.5 + np.arange(n) * dx  # cell i at x0 + i dx
    prof = np.cos(2.0 * math.pi * x)
    for k in range(8):
        U[k, 2:-2, 2:-2] = (avg[k] + eps * rv.reshape(8, 8)[wave][k] * prof)[:, None]
    return P.Problem(U, dx, dx, GAMMA, (M.PERIODIC,) * 4), abs(lam[wave])
