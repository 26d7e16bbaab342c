"""Shared helpers of the GPU parity tests (CUDA path through the C ABI)."""
import numpy as np

import mhd2d_b200 as M


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
