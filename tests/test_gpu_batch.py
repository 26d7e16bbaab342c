"""Batched runs (mhd_batch_*) against the oracle and against single contexts.

Every run of a batch must end bit-identical to the oracle's run of the same
problem (orc_run: the reference main loop without output), with the same
step count, simulated time and dt, whatever the mix of sizes, schemes,
boundary conditions and end times around it."""
import math

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import batch as B
from mhd2d_b200 import problems as P
from gpu_helpers import make_ctx, same
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _run_of(p, scheme, time_method=M.RK3, dt0=1e-3, t_end=0.05, dt_max=0.01, max_steps=0,
            cfl=0.4):
    return B.Run(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, scheme=scheme, time_method=time_method,
                 dt_min=1e-9, dt_max=dt_max, cfl=cfl, dt0=dt0, t_end=t_end, max_steps=max_steps)


def _mixed_problems():
    bw = P.brio_wu(64, 6)
    return [
        (P.explosion(40, 24), M.ENO_ROE, M.RK3, 0.02),
        (P.random_smooth(32, 48, seed=3), M.ENO_LF, M.RK3, 0.03),
        (P.random_blocky(20, 30, seed=5, bc=(M.NEUMANN,) * 4), M.ENO_LF, M.RK3, 0.02),
        (bw, M.ENO_ROE, M.RK3, 0.05),
        (P.ot_vortex(36), M.ENO_ROE, M.EULER, 0.05),
        (P.random_smooth(24, 20, seed=9, bc=(M.DIRICHLET, M.OPEN, M.PERIODIC, M.PERIODIC)),
         M.ENO_ROE, M.RK3, 0.02),
        (P.random_blocky(3, 37, seed=11, bc=(M.PERIODIC,) * 4), M.ENO_ROE, M.RK3, 0.01),
    ]


def _oracle_run(p, scheme, time_method, dt0, t_end, dt_max=0.01, max_steps=0):
    o = Oracle(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, scheme=scheme, time_method=time_method,
               dt_min=1e-9, dt_max=dt_max, cfl=0.4)
    U = p.U.copy()
    r = o.run(U, dt0, nsteps=max_steps, t_max=t_end)
    return U, r, o.retries()


def test_mixed_batch_matches_oracle_runs():
    probs = _mixed_problems()
    runs = [_run_of(p, s, tm, t_end=te) for p, s, tm, te in probs]
    with B.Batch(runs) as b:
        for i, (p, *_rest) in enumerate(probs):
            b.upload(i, p.U)
        left = b.run(check_every=30)
        assert left == 0
        for i, (p, s, tm, te) in enumerate(probs):
            U_ref, r, retries = _oracle_run(p, s, tm, 1e-3, te)
            st = b.state(i)
            U = b.download(i)
            assert st["steps"] == r["steps"], (i, st, r)
            assert st["t"] == r["t"] and st["dt"] == r["dt"], (i, st, r)
            assert st["status"].status == r["status"], (i, st, r)
            assert st["retries"] == retries, (i, st["retries"], retries)
            assert same(U[:, 2:-2, 2:-2], U_ref[:, 2:-2, 2:-2]), i


def test_batch_equals_single_context_steps():
    p = P.random_blocky(48, 40, seed=2)
    q = P.explosion(30, 50)
    runs = [_run_of(p, M.ENO_LF, max_steps=7, t_end=10.0), _run_of(q, M.ENO_ROE, max_steps=5,
                                                                   t_end=10.0)]
    with B.Batch(runs) as b:
        b.upload(0, p.U)
        b.upload(1, q.U)
        b.run()
        for i, (pp, s, n) in enumerate([(p, M.ENO_LF, 7), (q, M.ENO_ROE, 5)]):
            c = make_ctx(pp, scheme=s, dt_max=0.01, flags=0)
            dt = 1e-3
            for _ in range(n):
                stc, dt = c.step(dt)
                assert not stc.isError
            assert same(b.download(i)[:, 2:-2, 2:-2], c.download()[:, 2:-2, 2:-2])
            assert b.state(i)["dt"] == dt and b.state(i)["steps"] == n
            c.close()


def test_tune_leaves_runs_unchanged():
    probs = _mixed_problems()[:4]
    runs = [_run_of(p, s, tm, t_end=10.0, max_steps=6) for p, s, tm, _ in probs]
    out = []
    for tune in (False, True):
        with B.Batch(runs) as b:
            for i, (p, *_r) in enumerate(probs):
                b.upload(i, p.U)
            b.advance(5)
            if tune:
                info = b.tune(reps=1)
                assert info["tile"] in (B.TILE_7x32, B.TILE_3x32) and info["ms_per_stage"] > 0
            b.run()
            out.append([b.download(i) for i in range(len(runs))])
    for a, c in zip(*out):
        assert same(a[:, 2:-2, 2:-2], c[:, 2:-2, 2:-2])


@pytest.mark.parametrize("tile", [B.TILE_7x32, B.TILE_3x32])
def test_tile_shapes_agree(tile):
    probs = _mixed_problems()
    runs = [_run_of(p, s, tm, t_end=10.0, max_steps=4) for p, s, tm, _ in probs]
    res = []
    for t in (B.TILE_7x32, tile):
        with B.Batch(runs) as b:
            b.set_tile(t)
            for i, (p, *_r) in enumerate(probs):
                b.upload(i, p.U)
            b.run()
            res.append([b.download(i) for i in range(len(runs))])
    for a, c in zip(*res):
        assert same(a[:, 2:-2, 2:-2], c[:, 2:-2, 2:-2])


def test_failing_run_stops_alone():
    good = P.random_smooth(24, 24, seed=1)
    bad = P.random_smooth(24, 24, seed=1)
    bad.U[0, 10, 10] = -5.0  # negative density: getEigens_F error at the first integrate
    runs = [_run_of(good, M.ENO_ROE, t_end=10.0, max_steps=4), _run_of(bad, M.ENO_ROE, t_end=10.0)]
    with B.Batch(runs) as b:
        b.upload(0, good.U)
        b.upload(1, bad.U)
        assert b.run() == 0
        s0, s1 = b.state(0), b.state(1)
        assert s0["steps"] == 4 and s0["status"].status == M.OK
        assert s1["status"].status == M.ERR_NEGATIVE_DENSITY and s1["steps"] == 0
        U_ref, r, _ = _oracle_run(good, M.ENO_ROE, M.RK3, 1e-3, 10.0, max_steps=4)
        assert same(b.download(0)[:, 2:-2, 2:-2], U_ref[:, 2:-2, 2:-2])


def test_rearm_after_finish():
    p = P.random_smooth(20, 28, seed=4)
    runs = [_run_of(p, M.ENO_ROE, t_end=10.0, max_steps=3)]
    with B.Batch(runs) as b:
        b.upload(0, p.U)
        b.run()
        first = b.download(0)
        b.upload(0, p.U)  # re-arm the same run
        b.run()
        assert same(first, b.download(0)) and b.state(0)["steps"] == 3


# --- device-side initial states ----------------------------------------------------

def _to_conserved(q, gamma):
    rho, u, v, w, bx, by, bz, p = q
    uu = u * u + v * v + w * w
    bb = bx * bx + by * by + bz * bz
    return np.array([rho, u * rho, v * rho, w * rho, bx, by, bz,
                     p / (gamma - 1.0) + 0.5 * rho * uu + 0.5 * bb])


def test_device_explosion_matches_reference_setup():
    nx, ny, g = 37, 22, 5.0 / 3.0
    dx, dy = 1.0 / nx, 1.0 / ny
    with B.Batch([B.Run(nx, ny, dx, dy, g, (M.OPEN,) * 4, t_end=1.0)]) as b:
        b.init_explosion(0, r=0.1, rho_in=1.0, p_in=10.0, rho_out=0.125, p_out=1.0,
                         bx=2 ** -0.5, by=2 ** -0.5)
        U = b.download(0)
    NX, NY = nx + 4, ny + 4
    for i in range(2, nx + 2):
        for j in range(2, ny + 2):  # readProblemExplosion: centre at (NX/2, NY/2)
            inside = (i - NX // 2) ** 2 * dx * dx + (j - NY // 2) ** 2 * dy * dy < 0.1 * 0.1
            q = (1.0, 0, 0, 0, 2 ** -0.5, 2 ** -0.5, 0, 10.0) if inside else \
                (0.125, 0, 0, 0, 2 ** -0.5, 2 ** -0.5, 0, 1.0)
            assert np.array_equal(U[:, i, j], _to_conserved(q, g)), (i, j)


def test_device_wave_matches_reference_setup():
    from pyoracle import load_oracle
    import ctypes as C
    nx, ny, g = 24, 40, 5.0 / 3.0
    dx, dy = 1.0 / nx, 1.0 / ny
    lib = load_oracle()
    bg = (1.0, 0.0, 0.0, 0.0, 1.0, math.sqrt(2.0), 0.5, 1.0 / g)
    avg = _to_conserved(bg, g)
    for wave, kx, ky in [(0, 1, 0), (1, 1, 1), (3, 2, 1), (6, 0, 1), (4, 1, 2)]:
        with B.Batch([B.Run(nx, ny, dx, dy, g, (M.PERIODIC,) * 4, t_end=1.0)]) as b:
            b.init_wave(0, wave, kx, ky, eps=1e-6)
            U = b.download(0)
        lam = np.zeros(8); lv = np.zeros(64); rv = np.zeros(64); npr = C.c_int(0)
        dp = C.POINTER(C.c_double)
        st = lib.orc_eigens_f(C.c_double(g), avg.ctypes.data_as(dp), avg.ctypes.data_as(dp),
                              lam.ctypes.data_as(dp), lv.ctypes.data_as(dp),
                              rv.ctypes.data_as(dp), C.byref(npr))
        assert st == 0
        ev = rv.reshape(8, 8)[wave]
        ang = math.atan2(ky, kx)
        ct, s_ = math.cos(ang), math.sin(ang)
        for i in range(nx):
            for j in range(ny):
                x, y = -0.5 + i * dx, -0.5 + j * dy
                c = avg + 1e-6 * ev * math.cos(2 * math.pi * kx * x + 2 * math.pi * ky * y)
                u, v, w = c[1] / c[0], c[2] / c[0], c[3] / c[0]
                pr = (g - 1.0) * (c[7] - 0.5 * (c[1] ** 2 + c[2] ** 2 + c[3] ** 2) / c[0]
                                  - 0.5 * (c[4] ** 2 + c[5] ** 2 + c[6] ** 2))
                q = (c[0], ct * u - s_ * v, s_ * u + ct * v, w, ct * c[4] - s_ * c[5],
                     s_ * c[4] + ct * c[5], c[6], pr)
                ref = _to_conserved(q, g)
                # device cos / atan2 differ from the host libm in the last bits
                np.testing.assert_allclose(U[:, i + 2, j + 2], ref, rtol=1e-13, atol=1e-15)


def test_device_orszag_tang_and_plasma_sheet():
    n, g = 32, 5.0 / 3.0
    p = P.ot_vortex(n)
    with B.Batch([B.Run(n, n, p.dx, p.dy, g, p.bc, t_end=1.0)]) as b:
        b.init_orszag_tang(0)
        U = b.download(0)
    np.testing.assert_allclose(U[:, 2:-2, 2:-2], p.U[:, 2:-2, 2:-2], rtol=1e-14, atol=1e-15)
    nx, ny = 40, 20
    dx, dy = 4.0 / nx, 2.0 / ny
    amps = np.random.default_rng(1).normal(0, 1e-3, 16)
    with B.Batch([B.Run(nx, ny, dx, dy, g, (M.NEUMANN, M.NEUMANN, M.PERIODIC, M.PERIODIC),
                        t_end=1.0)]) as b:
        b.init_plasma_sheet(0, amps, delta=0.1)
        U = b.download(0)
    x = (-2.0 + np.arange(nx) * dx)[:, None]
    y = (-1.0 + np.arange(ny) * dy)[None, :]
    by = np.tanh(x / 0.1) * np.ones_like(y)
    pr = 1.25 - 0.5 * by * by
    rho = pr / 0.5
    v = sum(a * np.sin((k + 1) * np.pi * y) for k, a in enumerate(amps)) * np.exp(-x * x / 0.04)
    z = np.zeros_like(by)
    ref = P.to_conserved(rho, z, v, z, z, by, z, pr, g)
    np.testing.assert_allclose(U[:, 2:-2, 2:-2], ref[:, 2:-2, 2:-2], rtol=1e-13, atol=1e-16)


def test_generated_states_run_like_uploaded_ones():
    """A device-generated wave run equals the same state uploaded from the host."""
    nx, ny, g = 30, 18, 5.0 / 3.0
    run = B.Run(nx, ny, 1.0 / nx, 1.0 / ny, g, (M.PERIODIC,) * 4, scheme=M.ENO_LF, t_end=10.0,
                max_steps=5, dt_max=0.01)
    with B.Batch([run, run]) as b:
        b.init_wave(0, 5, 1, 1, eps=1e-6)
        U0 = b.download(0)
        b.upload(1, U0)
        b.run()
        assert same(b.download(0)[:, 2:-2, 2:-2], b.download(1)[:, 2:-2, 2:-2])
