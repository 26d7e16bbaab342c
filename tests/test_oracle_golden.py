"""Pin the oracle (oracle/mhd_oracle.c) to the reference.

Every golden vector under tests/golden/ was produced by the unmodified
reference hot path (tests/golden/make_golden.py); the oracle must reproduce
each one bit for bit.  Where the reference library itself is built
(oracle/_ref), extra seeded cases compare the two directly.
"""
import glob
import os

import numpy as np
import pytest

from pyoracle import Oracle, Reference, SorParams, load_oracle, oracle_update_dt, reference_available
from mhd2d_b200 import problems as P

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def same(a, b):
    """Bitwise equality up to the sign of zero (NaNs compare equal)."""
    return np.array_equal(a, b, equal_nan=True)


def _files(prefix):
    fs = sorted(glob.glob(os.path.join(GOLD, prefix + "*.npz")))
    assert fs, f"no golden files {prefix}*"
    return fs


@pytest.mark.parametrize("path", _files("integrate_"), ids=os.path.basename)
def test_integrate_matches_reference(path):
    d = np.load(path)
    U = d["U_in"].copy()
    nx, ny = U.shape[1] - 4, U.shape[2] - 4
    o = Oracle(nx, ny, float(d["dx"]), float(d["dy"]), float(d["gamma"]), d["bc"],
               scheme=int(d["scheme"]))
    o.init_dirichlet(d["U_in"].copy())
    st, err, UL, ideal = o.integrate(U)
    assert st == int(d["status"]) and err == int(d["is_error"])
    if err:
        return  # the reference stops mid-sweep: only the status is defined
    s = (slice(None), slice(2, nx + 2), slice(2, ny + 2))
    assert same(U, d["U_out"])
    assert same(UL[s], d["UL"][s])
    assert ideal == float(d["dtIdeal"])
    cx, cy, LUx, LUy = o.characteristics()
    for name, a in (("cx", cx), ("cy", cy), ("LUx", LUx), ("LUy", LUy)):
        assert same(a, d[name]), name


@pytest.mark.parametrize("path", _files("run_"), ids=os.path.basename)
def test_run_matches_reference(path):
    d = np.load(path)
    U = d["U_in"].copy()
    nx, ny = U.shape[1] - 4, U.shape[2] - 4
    sp = None
    if d["sor"].size:
        v = d["sor"]
        sp = SorParams(int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), int(v[5]),
                       float(v[6]))
    o = Oracle(nx, ny, float(d["dx"]), float(d["dy"]), float(d["gamma"]), d["bc"],
               scheme=int(d["scheme"]), time_method=int(d["time_method"]),
               dt_min=float(d["dt_min"]), dt_max=float(d["dt_max"]), cfl=float(d["cfl"]))
    r = o.run(U, float(d["dt0"]), nsteps=int(d["nsteps"]), t_max=float(d["t_max"]), sor=sp,
              red_black=0, hist_len=256)
    assert r["status"] == int(d["status"]) and r["steps"] == int(d["steps"])
    assert same(r["dt_hist"], d["dt_hist"])
    assert same(r["divb_hist"], d["divb_hist"])
    assert r["dt"] == float(d["dt"]) and r["t"] == float(d["t"])
    assert same(U, d["U_out"])


def test_run_fixture_exercises_retry():
    d = np.load(os.path.join(GOLD, "run_explosion_retry.npz"))
    nx, ny = d["U_in"].shape[1] - 4, d["U_in"].shape[2] - 4
    o = Oracle(nx, ny, float(d["dx"]), float(d["dy"]), float(d["gamma"]), d["bc"],
               dt_min=float(d["dt_min"]), dt_max=float(d["dt_max"]), cfl=float(d["cfl"]))
    o.run(d["U_in"].copy(), float(d["dt0"]), nsteps=int(d["nsteps"]))
    assert o.retries() > 0


@pytest.mark.parametrize("path", _files("sor_"), ids=os.path.basename)
def test_sor_matches_reference(path):
    d = np.load(path)
    U = d["U_in"].copy()
    nx, ny = U.shape[1] - 4, U.shape[2] - 4
    v = d["sor"]
    sp = SorParams(int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), int(v[5]),
                   float(v[6]))
    o = Oracle(nx, ny, float(d["dx"]), float(d["dy"]), 5.0 / 3.0, d["bc"])
    st, err, _ = o.divb_sor(U, sp, red_black=0)
    assert st == int(d["status"]) and err == int(d["is_error"])
    assert same(U, d["U_out"])
    m, t = Oracle(nx, ny, float(d["dx"]), float(d["dy"]), 5.0 / 3.0, d["bc"]).divb_calc(U.copy())
    assert m == d["divb_out"][0] and t == d["divb_out"][1]


def test_update_dt_table():
    d = np.load(os.path.join(GOLD, "update_dt.npz"))["table"]
    lib = load_oracle()
    for dtmin, dtmax, cfl, dt, ideal, st, err, newdt in d:
        s, e, nd = oracle_update_dt(dtmin, dtmax, cfl, dt, ideal, lib=lib)
        assert (s, e) == (int(st), int(err))
        assert nd == newdt


def test_red_black_sor_reaches_same_divergence_level():
    """The red-black ordering (what the GPU runs) converges to the same
    max|div B| level as the reference's lexicographic sweep."""
    p = P.random_smooth(24, 20, seed=3, bc=(1, 1, 1, 1))
    sp = SorParams(1, 10, 100000.0, 1e-11, 1e-10, 1, 1.7)
    outs = []
    for rb in (0, 1):
        U = p.U.copy()
        o = Oracle(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc)
        st, err, sw = o.divb_sor(U, sp, red_black=rb)
        assert st == 0 and not err
        outs.append((U, o.divb_calc(U.copy())[0], sw))
    m_lex, m_rb = outs[0][1], outs[1][1]
    assert m_rb < 1e-8 and m_lex < 1e-8
    s = (slice(4, 6), slice(2, -2), slice(2, -2))
    assert np.max(np.abs(outs[0][0][s] - outs[1][0][s])) < 1e-7


needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_oracle_vs_reference_random(seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(6, 20)), int(rng.integers(6, 20))
    bc = tuple(int(b) for b in rng.integers(1, 5, size=4))
    p = (P.random_smooth if seed % 2 else P.random_blocky)(nx, ny, seed=100 + seed, bc=bc)
    ref = Reference()
    for scheme in (2, 3):
        U1 = p.U.copy()
        r = ref.integrate(scheme, U1, p.dx, p.dy, p.gamma, bc, U_dirichlet=p.U.copy(), chars=True)
        o = Oracle(nx, ny, p.dx, p.dy, p.gamma, bc, scheme=scheme)
        o.init_dirichlet(p.U.copy())
        U2 = p.U.copy()
        st, err, UL, ideal = o.integrate(U2)
        assert st == r["status"] and err == r["is_error"]
        s = (slice(None), slice(2, nx + 2), slice(2, ny + 2))
        assert same(U1, U2) and same(UL[s], r["UL"][s]) and ideal == r["dtIdeal"]


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_oracle_central_fd_vs_reference_random(seed):
    """Central FD2 on random square-or-wider grids (ny <= nx: the reference's
    corner test reads flux entries it never wrote when ny > nx), corners
    filled or left at zero, every boundary mix."""
    rng = np.random.default_rng(50 + seed)
    nx = int(rng.integers(6, 20))
    ny = int(rng.integers(4, nx + 1))
    bc = tuple(int(b) for b in rng.integers(1, 5, size=4))
    p = (P.random_smooth if seed % 2 else P.random_blocky)(nx, ny, seed=200 + seed, bc=bc)
    if seed % 3:  # ghost corners get their nearest interior state
        for i in (0, 1, nx + 2, nx + 3):
            for j in (0, 1, ny + 2, ny + 3):
                p.U[:, i, j] = p.U[:, min(max(i, 2), nx + 1), min(max(j, 2), ny + 1)]
    U1 = p.U.copy()
    r = Reference().integrate(1, U1, p.dx, p.dy, p.gamma, bc, U_dirichlet=p.U.copy())
    o = Oracle(nx, ny, p.dx, p.dy, p.gamma, bc, scheme=1)
    o.init_dirichlet(p.U.copy())
    U2 = p.U.copy()
    st, err, UL, ideal = o.integrate(U2)
    assert st == r["status"] and err == r["is_error"]
    assert same(U1, U2)
    if st != 6:
        s = (slice(None), slice(2, nx + 2), slice(2, ny + 2))
        assert same(UL[s], r["UL"][s]) and ideal == r["dtIdeal"]


def test_fixed_lf_alpha_hook():
    """The window hook of the oracle: integrating with the coefficients of
    lf_alpha_grid (on the filled state) gives the ordinary ENO-LF result;
    other coefficients change it."""
    from pyoracle import Oracle, lf_alpha_grid
    from mhd2d_b200 import problems as P

    p = P.ot_vortex(40)
    o = Oracle(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, scheme=3)
    U = p.U.copy()
    _, _, UL, ideal = o.integrate(U)
    aF, aG = lf_alpha_grid(U, p.gamma)
    o2 = Oracle(p.nx, p.ny, p.dx, p.dy, p.gamma, p.bc, scheme=3)
    o2.set_lf_alpha(aF, aG)
    _, _, UL2, ideal2 = o2.integrate(p.U.copy())
    assert np.array_equal(UL, UL2) and ideal == ideal2
    o2.set_lf_alpha(1.1 * aF, 1.1 * aG)
    _, _, UL3, _ = o2.integrate(p.U.copy())
    assert not np.array_equal(UL, UL3)
