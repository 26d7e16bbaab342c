"""Discrete adjoint of the ENO-Roe step (mhd_adj_*) against the tangent-linear
oracle (oracle/tlm.cpp: forward-mode derivative of the same discrete map with
the same frozen branches) and against frozen-stencil central differences of
the GPU replay."""
import os

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from mhd2d_b200.adjoint import Adjoint
from gpu_helpers import make_ctx, same
from pyoracle import tlm_run

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _interior_dirs(shape, n, seed):
    d = np.random.default_rng(seed).normal(0, 1, (n,) + shape)
    d[:, :, :2], d[:, :, -2:], d[:, :, :, :2], d[:, :, :, -2:] = 0, 0, 0, 0
    return d


def _adjoint(p, nsteps, dt0=1e-3, dt_max=0.01, tm=M.RK3, K=4, cfl=0.4, dt_min=1e-9, store=-1,
             contract=True):
    a = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, time_method=tm, dt_min=dt_min,
                dt_max=dt_max, cfl=cfl, checkpoint_every=K)
    a.set_store(store)
    a.set_contract(contract)
    a.upload(p.U)
    J = a.forward(nsteps, dt0)
    return a, J


def _dot(g, d):
    return float((g[:, 2:-2, 2:-2] * d[:, 2:-2, 2:-2]).sum())


CASES = [
    ("sheet", lambda: P.plasma_sheet(32, 16, np.random.default_rng(1).normal(0, 1e-2, 6))),
    ("smooth-periodic", lambda: P.random_smooth(24, 20, seed=2)),
    ("smooth-open", lambda: P.random_smooth(20, 24, seed=3, bc=(M.OPEN,) * 4)),
    ("smooth-mixed", lambda: P.random_smooth(22, 18, seed=4,
                                            bc=(M.DIRICHLET, M.NEUMANN, M.NEUMANN, M.OPEN))),
    ("blocky-neumann", lambda: P.random_blocky(20, 20, seed=6, bc=(M.NEUMANN,) * 4)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_recording_forward_and_replay_match_context(name, make):
    p = make()
    a, J = _adjoint(p, 6)
    c = make_ctx(p, dt_min=1e-9, dt_max=0.01, flags=0)
    dt = 1e-3
    for _ in range(6):
        st, dt = c.step(dt)
        assert not st.isError
    Uc = c.download()
    assert same(a.download(1)[:, 2:-2, 2:-2], Uc[:, 2:-2, 2:-2])
    assert a.info()["dt"] == dt
    assert a.replay() == J  # frozen replay of the recorded initial state
    assert same(a.download(2)[:, 2:-2, 2:-2], Uc[:, 2:-2, 2:-2])


# Tolerance against the tangent-linear oracle (relative, per direction).  The
# uncontracted reverse sweep rounds like the oracle; the contracted one (the
# default) differs by rounding that the near-degenerate eigen-system of the
# current sheet (B_perp ~ 0) amplifies to ~4e-8.
TLM_RTOL = {False: 1e-9, True: 1e-7}


@pytest.mark.parametrize("contract", [False, True], ids=["uncontracted", "contracted"])
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_adjoint_matches_tangent_linear(name, make, contract):
    p = make()
    nsteps = 6
    a, J = _adjoint(p, nsteps, contract=contract)
    a.backward()
    g = a.gradient()
    d = _interior_dirs(p.U.shape, 4, seed=7)
    r = tlm_run(p.U, d, p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, nsteps=nsteps, dt0=1e-3,
                dt_min=1e-9, dt_max=0.01)
    assert r["steps"] == nsteps
    assert abs(r["J"] - J) <= 1e-12 * abs(J)
    for q in range(d.shape[0]):
        adj = _dot(g, d[q])
        assert abs(adj - r["dJ"][q]) <= TLM_RTOL[contract] * max(abs(r["dJ"][q]), 1e-30), \
            (q, adj, r["dJ"][q])


def test_contract_setting_keeps_the_recording():
    """mhd_adj_set_contract switches the reverse sweep on an existing
    recording: each setting reproduces a fresh run's gradient bit for bit,
    and the two differ by rounding only."""
    p = P.plasma_sheet(32, 16, np.random.default_rng(1).normal(0, 1e-2, 6))
    a, _ = _adjoint(p, 6, contract=False)
    a.backward()
    g_plain = a.gradient()
    a.set_contract(True)
    a.backward()
    g_fma = a.gradient()
    b, _ = _adjoint(p, 6, contract=True)
    b.backward()
    assert same(g_fma, b.gradient())
    c, _ = _adjoint(p, 6, contract=False)
    c.backward()
    assert same(g_plain, c.gradient())
    scale = np.abs(g_plain).max()
    assert np.abs(g_fma - g_plain).max() <= 1e-7 * scale


def test_sheet_amplitude_gradient_matches_tangent_linear():
    amps = np.random.default_rng(5).normal(0, 1e-3, 16)
    p = P.plasma_sheet(40, 20, amps)
    a, J = _adjoint(p, 12)
    a.sheet = (p.extra["x0"], p.extra["y0"], 16)
    a.backward()
    dJda = a.sheet_gradient()
    T = P.plasma_sheet_tangents(p)
    r = tlm_run(p.U, T, p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, nsteps=12, dt0=1e-3,
                dt_min=1e-9, dt_max=0.01)
    scale = np.abs(r["dJ"]).max()
    assert np.all(np.abs(dJda - r["dJ"]) <= 1e-9 * scale), (dJda, r["dJ"])


@pytest.mark.parametrize("bc", [(M.PERIODIC,) * 4, (M.OPEN, M.OPEN, M.NEUMANN, M.NEUMANN)])
def test_frozen_stencil_central_differences(bc):
    """(J(U0 + h d) - J(U0 - h d)) / 2h of the frozen replay, h = 1e-7, against
    the adjoint's dJ/dU0 . d, within 1e-6 relative, on a smooth state."""
    p = P.random_smooth(48, 40, seed=9, bc=bc)
    a, J = _adjoint(p, 20, K=6)
    a.backward()
    g = a.gradient()
    h = 1e-7
    for d in _interior_dirs(p.U.shape, 3, seed=11):
        fd = (a.replay(p.U + h * d) - a.replay(p.U - h * d)) / (2 * h)
        adj = _dot(g, d)
        assert abs(fd - adj) <= 1e-6 * abs(adj), (fd, adj)


def test_plasma_sheet_amplitude_differences():
    """The current sheet starts with B_x = 0, where the slow speed
    c_s = sqrt(c^2 - sqrt(c^4 - a^2 c_a^2)) ~ |B_x| a / sqrt(2 rho c^2) has a
    kink (and its computed value a rounding-level cancellation): the discrete
    map is not differentiable there, so central differences in the
    amplitudes a_k agree with the frozen-branch derivative only to ~1e-3 at
    h = 1e-5 and not better at smaller h.  The tangent-linear comparison
    above checks the same derivative to 1e-9."""
    amps = np.random.default_rng(9).normal(0, 1e-3, 16)
    p = P.plasma_sheet(64, 32, amps)
    a, J = _adjoint(p, 30, K=8)
    a.backward()
    g = a.gradient()
    T = P.plasma_sheet_tangents(p)
    h = 1e-5
    for k in (0, 3):
        fd = (a.replay(p.U + h * T[k]) - a.replay(p.U - h * T[k])) / (2 * h)
        adj = _dot(g, T[k])
        assert abs(fd - adj) <= 5e-3 * abs(adj), (k, fd, adj)


def test_checkpoint_interval_does_not_change_the_gradient():
    p = P.random_blocky(24, 16, seed=8, bc=(M.PERIODIC, M.PERIODIC, M.NEUMANN, M.NEUMANN))
    grads = []
    for K in (1, 3, 100):
        for store in (0, -1):  # replayed segments / stage inputs kept by the recording
            a, _ = _adjoint(p, 7, K=K, store=store)
            a.backward()
            grads.append(a.gradient())
            info = a.info()
            assert info["checkpoints"] == -(-7 // K)
            assert info["replayed_segments"] == (info["checkpoints"] if store == 0 else 0)
    for g in grads[1:]:
        assert same(grads[0], g)


def test_stage_store_keeps_the_last_segments():
    p = P.random_blocky(24, 16, seed=8, bc=(M.PERIODIC, M.PERIODIC, M.NEUMANN, M.NEUMANN))
    grads, infos = [], []
    # a 2 MB store holds the stage inputs (86 KB each here) of the last segment only;
    # without kept masks the replayed segments record their ENO codes again
    for keep_masks in (True, False):
        for store in (0, 2 << 20, -1):
            a = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=1e-9, dt_max=0.01,
                        checkpoint_every=3)
            a.set_masks(keep_masks)
            a.set_store(store)
            a.upload(p.U)
            a.forward(7, 1e-3)
            a.backward()
            grads.append(a.gradient())
            infos.append(a.info())
            if not keep_masks:
                with pytest.raises(M.MhdError):
                    a.replay()
    for off in (0, 3):
        assert infos[off]["stored_stages"] == 0 and infos[off]["replayed_segments"] == 3
        assert 0 < infos[off + 1]["stored_stages"] < infos[off + 1]["stages"]
        assert 0 < infos[off + 1]["replayed_segments"] < 3
        assert infos[off + 2]["stored_stages"] == infos[off + 2]["stages"]
        assert infos[off + 2]["replayed_segments"] == 0
    for g in grads[1:]:
        assert same(grads[0], g)


def test_retry_steps_and_euler_match_tangent_linear():
    d = np.load(os.path.join(GOLD, "run_explosion_retry.npz"))
    p = P.Problem(d["U_in"].copy(), float(d["dx"]), float(d["dy"]), float(d["gamma"]),
                  tuple(int(b) for b in d["bc"]))
    n = int(d["nsteps"])
    kw = dict(dt0=float(d["dt0"]), dt_max=float(d["dt_max"]), cfl=float(d["cfl"]),
              dt_min=float(d["dt_min"]))
    a, J = _adjoint(p, n, **kw)
    assert a.info()["retries"] > 0  # the case really restarts RK3 stage loops
    a.backward()
    g = a.gradient()
    dirs = _interior_dirs(p.U.shape, 3, seed=12)
    r = tlm_run(p.U, dirs, p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, nsteps=n, dt0=kw["dt0"],
                dt_min=kw["dt_min"], dt_max=kw["dt_max"], cfl=kw["cfl"])
    for q in range(3):
        assert abs(_dot(g, dirs[q]) - r["dJ"][q]) <= 1e-9 * abs(r["dJ"][q])
    a0, _ = _adjoint(p, n, store=0, **kw)  # the retried stages replayed from checkpoints
    a0.backward()
    assert same(a0.gradient(), g)
    a1 = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=kw["dt_min"], dt_max=kw["dt_max"],
                 cfl=kw["cfl"], checkpoint_every=4)
    a1.set_masks(False)  # ... with their masks recorded again by the replays
    a1.set_store(0)
    a1.upload(p.U)
    a1.forward(n, kw["dt0"])
    a1.backward()
    assert same(a1.gradient(), g)
    pe = P.random_smooth(20, 20, seed=13)
    a, J = _adjoint(pe, 5, tm=M.EULER)
    a.backward()
    g = a.gradient()
    dirs = _interior_dirs(pe.U.shape, 2, seed=14)
    r = tlm_run(pe.U, dirs, pe.nx, pe.ny, pe.dx, pe.dy, pe.gamma, pe.bc, nsteps=5, dt0=1e-3,
                time_method=1, dt_min=1e-9, dt_max=0.01)
    for q in range(2):
        assert abs(_dot(g, dirs[q]) - r["dJ"][q]) <= 1e-9 * abs(r["dJ"][q])


def test_device_plasma_sheet_and_its_gradient():
    amps = np.random.default_rng(2).normal(0, 1e-3, 16)
    p = P.plasma_sheet(48, 24, amps)
    a = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=1e-9, dt_max=0.01,
                checkpoint_every=5)
    a.init_plasma_sheet(amps)
    U0 = a.download(0)
    np.testing.assert_allclose(U0[:, 2:-2, 2:-2], p.U[:, 2:-2, 2:-2], rtol=1e-13, atol=1e-17)
    a.forward(8, 1e-3)
    a.backward()
    dJda = a.sheet_gradient()
    # the same state uploaded from the host gives the same dJ/da
    b = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=1e-9, dt_max=0.01,
                checkpoint_every=5)
    b.upload(U0)
    b.forward(8, 1e-3)
    b.backward()
    b.sheet = a.sheet
    assert same(dJda, b.sheet_gradient())
    # frozen central differences in the amplitudes (replays of the device setup)
    h = 1e-7
    for k in (0, 7):
        ap, am = amps.copy(), amps.copy()
        ap[k] += h
        am[k] -= h
        fd = (a.replay_plasma_sheet(ap) - a.replay_plasma_sheet(am)) / (2 * h)
        assert abs(fd - dJda[k]) <= 1e-6 * np.abs(dJda).max(), (k, fd, dJda[k])


def test_autograd_function_wrapper():
    import torch

    from adjoint_autograd import kinetic_energy_after_steps
    p = P.random_smooth(32, 24, seed=4)
    a = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=1e-9, dt_max=0.01,
                checkpoint_every=3)
    U0 = torch.tensor(p.U, dtype=torch.float64, requires_grad=True)
    J = kinetic_energy_after_steps(U0, a, 9, 1e-3)
    J.backward()
    d = _interior_dirs(p.U.shape, 1, seed=21)[0]
    h = 1e-7
    fd = (a.replay(p.U + h * d) - a.replay(p.U - h * d)) / (2 * h)
    adj = float((U0.grad.numpy() * d).sum())
    assert abs(fd - adj) <= 1e-6 * abs(adj)


def test_group_forward_and_backward_match_separate_runs():
    from mhd2d_b200.adjoint import backward_group, forward_group
    probs = [P.plasma_sheet(32, 16, np.random.default_rng(3).normal(0, 1e-2, 6)),
             P.random_smooth(24, 20, seed=2),
             P.random_blocky(20, 20, seed=6, bc=(M.NEUMANN,) * 4),
             P.random_smooth(22, 18, seed=4, bc=(M.DIRICHLET, M.NEUMANN, M.NEUMANN, M.OPEN))]
    nsteps = [7, 5, 6, 4]
    setups = [(True, -1), (False, 0), (False, 2 << 20), (True, 0)]  # (keep masks, store)

    def make(i):
        p = probs[i]
        a = Adjoint(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, dt_min=1e-9, dt_max=0.01,
                    checkpoint_every=3)
        a.set_masks(setups[i][0])
        a.set_store(setups[i][1])
        a.upload(p.U)
        return a

    solo = []
    for i in range(len(probs)):
        a = make(i)
        J = a.forward(nsteps[i], 1e-3)
        a.backward()
        solo.append((J, a.gradient(), a.download(1)))
    group = [make(i) for i in range(len(probs))]
    Js, ms_f = forward_group(group, nsteps, 1e-3)
    ms_b = backward_group(group)
    assert ms_f > 0 and ms_b > 0
    for i, a in enumerate(group):
        assert Js[i] == solo[i][0]
        assert same(a.download(1), solo[i][2])
        assert same(a.gradient(), solo[i][1])
        assert a.info()["steps"] == nsteps[i]
