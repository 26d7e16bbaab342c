"""CPU jobs of the configuration-size parity tests, run in worker processes
(a `spawn` pool, so no worker inherits a CUDA context).

Every job runs the unmodified reference (oracle/_ref/libmhdref.so) or the
oracle restatement from a problem description and returns the end state and
the run's bookkeeping; the parent compares them with the device runs.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (os.path.join(ROOT, "mhd2d-solver_b200"), os.path.join(ROOT, "oracle"), HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def problem(kind, n):
    from mhd2d_b200 import problems as P

    if kind == "ot":
        return P.ot_vortex(n)
    if kind == "explosion":
        return P.explosion(n)
    raise ValueError(kind)


def reference_run(kind, n, scheme, dt0, dt_min, dt_max, cfl, nsteps=0, t_max=0.0):
    """The reference's own main loop (no output) on problem `kind` of side n."""
    from pyoracle import Reference

    p = problem(kind, n)
    U = p.U.copy()
    r = Reference(fresh=True).run(scheme, 2, U, p.dx, p.dy, p.gamma, p.bc, dt0, dt_min, dt_max,
                                  cfl, nsteps=nsteps, t_max=t_max)
    return dict(U=U, steps=r["steps"], t=r["t"], dt=r["dt"], status=r["status"],
                is_error=r["is_error"])


def oracle_run(U0, nx, ny, dx, dy, gamma, bc, scheme, time_method, dt0, dt_min, dt_max, cfl,
               t_max, max_steps=0):
    """The oracle's main loop (the reference's semantics) from state U0."""
    from pyoracle import Oracle

    o = Oracle(nx, ny, dx, dy, gamma, bc, scheme=scheme, time_method=time_method, dt_min=dt_min,
               dt_max=dt_max, cfl=cfl)
    U = U0.copy()
    o.init_dirichlet(U)
    r = o.run(U, dt0, nsteps=max_steps, t_max=t_max)
    return dict(U=U, steps=r["steps"], t=r["t"], dt=r["dt"], status=r["status"],
                retries=o.retries())
