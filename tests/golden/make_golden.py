"""Generate the golden vectors under tests/golden/ from the UNMODIFIED reference.

Runs the reference hot path (oracle/_ref/libmhdref.so, built by
`make -C oracle ref` from the reference sources) on small seeded states and
stores inputs and outputs as compressed .npz files:

* integrate_*.npz — one SpatialMethodEnoRoe/EnoLF/CentralFD2::integrate call: state in,
  state out (ghosts filled), UL, dtIdeal, status, characteristics;
* run_*.npz       — the main loop for a few steps (RK3 / Euler, dt control
  with retries, optional SOR cleaning): final state, dt and div B history;
* sor_*.npz       — one divBCorrectionSOR call (lexicographic sweep);
* update_dt.npz   — a table of TimeIntegrationMethod::updateDt cases.

Usage:  python tests/golden/make_golden.py [name-prefix ...]
        (needs the reference build; with prefixes only the matching files are
        written, so the others keep their bytes)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "mhd2d-solver_b200"))

from pyoracle import Reference, sor_params  # noqa: E402
from mhd2d_b200 import problems as P  # noqa: E402

BCS = [(1, 1, 1, 1), (3, 3, 3, 3), (4, 4, 4, 4), (2, 2, 2, 2), (1, 1, 3, 3), (4, 3, 1, 2)]


def integrate_cases():
    cases = []
    for n, bc in enumerate(BCS):
        cases.append((f"smooth_bc{n}", P.random_smooth(12, 10, seed=10 + n, bc=bc)))
        cases.append((f"blocky_bc{n}", P.random_blocky(12, 10, seed=20 + n, bc=bc)))
    cases.append(("briowu", P.brio_wu(32, 8)))
    cases.append(("otvortex", P.ot_vortex(16)))
    cases.append(("explosion", P.explosion(16)))
    # a clamped (negative) pressure at the last y interface, (nx+1, ny+1)
    p = P.random_blocky(10, 9, seed=31, bc=(3, 3, 3, 3))
    i = p.nx + 1
    p.U[7, i, p.ny] = 0.0
    p.U[7, i, p.ny + 1] = 0.0
    cases.append(("negpressure_last", p))
    # a clamped pressure elsewhere only (the last interface is fine)
    p = P.random_blocky(10, 9, seed=33, bc=(1, 1, 1, 1))
    p.U[7, 4, 5] = 0.0
    p.U[7, 4, 6] = 0.0
    cases.append(("negpressure_inner", p))
    # non-positive density: the midpoint of two cells must be <= 0 for the
    # ENO-Roe check, a single cell suffices for the ENO-LF cell eigenvalues
    p = P.random_smooth(10, 9, seed=32, bc=(1, 1, 1, 1))
    p.U[0, 5, 6] = -5.0
    cases.append(("negdensity", p))
    return cases


def fill_corners(p):
    """Ring corners of a central-FD state: the reference's corner test uses
    the x bounds for j too, so with ny < nx it evaluates the ghost corners
    (1, ny+2) and (nx+2, ny+2), which no boundary fill writes; give every
    ghost corner the state of its nearest interior cell."""
    U = p.U
    nx, ny = p.nx, p.ny
    for i in (0, 1, nx + 2, nx + 3):
        for j in (0, 1, ny + 2, ny + 3):
            U[:, i, j] = U[:, min(max(i, 2), nx + 1), min(max(j, 2), ny + 1)]
    return p


def cfd_integrate_cases():
    """Central FD2 (scheme 1): smooth states with nx >= ny (with ny > nx the
    reference reads flux entries it never wrote), its fatal negative
    pressure and density, and an unfilled ring corner."""
    cases = []
    for n, bc in enumerate(BCS):
        cases.append((f"cfd_smooth_bc{n}", fill_corners(P.random_smooth(12, 10, seed=60 + n, bc=bc))))
    cases.append(("cfd_otvortex", P.ot_vortex(16)))
    cases.append(("cfd_explosion", P.explosion(16)))
    p = fill_corners(P.random_smooth(11, 9, seed=66, bc=(1, 1, 1, 1)))
    p.U[7, 4, 5] = 0.0
    p.U[7, 7, 3] = 0.0
    cases.append(("cfd_negpressure", p))
    p = fill_corners(P.random_smooth(11, 9, seed=67, bc=(3, 3, 3, 3)))
    p.U[0, 6, 4] = -1.0
    p.U[0, 3, 7] = -2.0
    cases.append(("cfd_negdensity", p))
    cases.append(("cfd_zerocorner", P.random_smooth(12, 10, seed=68, bc=(1, 1, 1, 1))))
    return cases


def run_cases():
    sp = sor_params(1, 5, 20000, 1e-9, 1e-9, True, 1.7)
    return [
        # name, problem, scheme, time method, dt0, dt_min, dt_max, cfl, nsteps, t_max, sor
        ("briowu_roe", P.brio_wu(32, 8), 2, 2, 0.0078125, 1e-6, 0.0078125, 0.4, 0, 0.04, None),
        ("briowu_lf", P.brio_wu(32, 8), 3, 2, 0.0078125, 1e-6, 0.0078125, 0.4, 0, 0.04, None),
        # the Brio-Wu shock tube at its full size and end time (256 x 8, t = 0.2, ~410 steps)
        ("briowu_full_roe", P.brio_wu(256, 8), 2, 2, 0.0078125, 1e-6, 0.0078125, 0.4, 0, 0.2,
         None),
        ("briowu_full_lf", P.brio_wu(256, 8), 3, 2, 0.0078125, 1e-6, 0.0078125, 0.4, 0, 0.2,
         None),
        ("ot_roe", P.ot_vortex(16), 2, 2, 0.03125, 1e-6, 0.03125, 0.4, 5, 0.0, None),
        ("ot_lf", P.ot_vortex(16), 3, 2, 0.03125, 1e-6, 0.03125, 0.4, 5, 0.0, None),
        ("explosion_retry", P.explosion(16), 2, 2, 0.02, 1e-9, 0.02, 0.4, 4, 0.0, None),
        ("blocky_euler", P.random_blocky(14, 12, seed=40, bc=(4, 3, 1, 2)), 3, 1, 0.01, 1e-9,
         0.01, 0.3, 4, 0.0, None),
        ("blocky_const", P.random_blocky(14, 12, seed=41, bc=(2, 2, 3, 3)), 2, 2, 0.002, 0.0,
         0.002, 0.0, 3, 0.0, None),
        ("ot_roe_sor", P.ot_vortex(16), 2, 2, 0.03125, 1e-6, 0.03125, 0.4, 3, 0.0, sp),
        ("smooth_lf_sor", P.random_smooth(16, 12, seed=42, bc=(3, 3, 1, 1)), 3, 2, 0.02, 1e-7,
         0.02, 0.4, 2, 0.0, sp),
        ("cfd_ot_rk3", P.ot_vortex(16), 1, 2, 0.0078125, 1e-6, 0.0078125, 0.2, 6, 0.0, None),
        ("cfd_smooth_euler", fill_corners(P.random_smooth(14, 12, seed=43, bc=(1, 1, 4, 4))), 1,
         1, 0.002, 1e-9, 0.002, 0.2, 4, 0.0, None),
    ]


def main():
    ref = Reference()
    out = {}
    for name, prob in integrate_cases():
        for scheme in (2, 3):
            U = prob.U.copy()
            r = ref.integrate(scheme, U, prob.dx, prob.dy, prob.gamma, prob.bc,
                              U_dirichlet=prob.U.copy(), chars=True)
            out[f"integrate_{name}_{scheme}"] = dict(
                U_in=prob.U, U_out=U, UL=r["UL"], dtIdeal=r["dtIdeal"], status=r["status"],
                is_error=r["is_error"], cx=r["cx"], cy=r["cy"], LUx=r["LUx"], LUy=r["LUy"],
                dx=prob.dx, dy=prob.dy, gamma=prob.gamma, bc=np.array(prob.bc), scheme=scheme)
    for name, prob in cfd_integrate_cases():
        U = prob.U.copy()
        r = ref.integrate(1, U, prob.dx, prob.dy, prob.gamma, prob.bc,
                          U_dirichlet=prob.U.copy(), chars=True)
        out[f"integrate_{name}_1"] = dict(
            U_in=prob.U, U_out=U, UL=r["UL"], dtIdeal=r["dtIdeal"], status=r["status"],
            is_error=r["is_error"], cx=r["cx"], cy=r["cy"], LUx=r["LUx"], LUy=r["LUy"],
            dx=prob.dx, dy=prob.dy, gamma=prob.gamma, bc=np.array(prob.bc), scheme=1,
            message=r.get("message", ""))
    for (name, prob, scheme, tm, dt0, dtmin, dtmax, cfl, nsteps, tmax, sp) in run_cases():
        ref = Reference(fresh=True)
        U = prob.U.copy()
        r = ref.run(scheme, tm, U, prob.dx, prob.dy, prob.gamma, prob.bc, dt0, dtmin, dtmax, cfl,
                    nsteps=nsteps, t_max=tmax, sor=sp, hist_len=256)
        spv = np.array([sp.divb_skip_steps, sp.sor_steps, sp.sor_rsteps, sp.sor_rmax,
                        sp.sor_divbmax, sp.omega_use_static, sp.omega]) if sp else np.zeros(0)
        out[f"run_{name}"] = dict(
            U_in=prob.U, U_out=U, status=r["status"], is_error=r["is_error"], dt=r["dt"], t=r["t"],
            steps=r["steps"], dt_hist=r["dt_hist"], divb_hist=r["divb_hist"], dx=prob.dx,
            dy=prob.dy, gamma=prob.gamma, bc=np.array(prob.bc), scheme=scheme, time_method=tm,
            dt0=dt0, dt_min=dtmin, dt_max=dtmax, cfl=cfl, nsteps=nsteps, t_max=tmax, sor=spv)
    for n, bc in enumerate([(1, 1, 1, 1), (3, 3, 1, 1), (4, 4, 4, 4), (2, 3, 4, 1)]):
        prob = P.random_smooth(14, 12, seed=50 + n, bc=bc)
        ref = Reference(fresh=True)
        sp = sor_params(1, 5, 5000, 1e-8, 1e-9, n % 2 == 0, 1.6)
        U = prob.U.copy()
        st, err = ref.divb_sor(U, prob.dx, prob.dy, prob.bc, sp)
        m0, t0 = Reference().divb_calc(prob.U.copy(), prob.dx, prob.dy, prob.bc)
        m1, t1 = Reference().divb_calc(U.copy(), prob.dx, prob.dy, prob.bc)
        out[f"sor_{n}"] = dict(U_in=prob.U, U_out=U, status=st, is_error=err, dx=prob.dx,
                               dy=prob.dy, bc=np.array(prob.bc), divb_in=[m0, t0],
                               divb_out=[m1, t1],
                               sor=np.array([1, 5, 5000, 1e-8, 1e-9, n % 2 == 0, 1.6]))
    rng = np.random.default_rng(7)
    rows = []
    ref = Reference()
    for _ in range(200):
        dt = 2.0 ** rng.integers(-14, 0)
        ideal = 10 ** rng.uniform(-5, 0)
        cfl = [0.0, 0.2, 0.4, 0.9][rng.integers(0, 4)]
        dtmin = [0.0, 1e-6, 1e-3][rng.integers(0, 3)]
        dtmax = 2.0 ** rng.integers(-8, 1)
        st, err, newdt = ref.update_dt(dtmin, dtmax, cfl, dt, ideal)
        rows.append([dtmin, dtmax, cfl, dt, ideal, st, err, newdt])
    out["update_dt"] = dict(table=np.array(rows))
    only = sys.argv[1:]
    n = 0
    for key, d in out.items():
        if only and not any(key.startswith(p) for p in only):
            continue
        np.savez_compressed(os.path.join(HERE, key + ".npz"), **d)
        n += 1
    print(f"wrote {n} golden files to {HERE}")


if __name__ == "__main__":
    main()
