"""Batched runs (mhd_batch_* in include/mhd2d_b200.h).

The reference runs one problem per process (main.cpp); running many is
starting several copies with different INI files.  ``Batch`` holds many
independent runs of uneven grid sizes, schemes, boundary conditions and end
times on one GPU and advances all of them together, each following the
reference main loop (step, t += dt, stop at t >= t_end, on a NaN or on a
fatal status).  Each run's result is bit-identical to the same problem
advanced alone through a ``Context``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import (ENO_ROE, OK, RK3, STATUS_NAMES, BatchDesc, BatchState, MhdError, TStatus, _p,
               library)

PROBLEM_EXPLOSION, PROBLEM_WAVE, PROBLEM_ORSZAG_TANG, PROBLEM_PLASMA_SHEET = 1, 2, 3, 4
PROBLEM_SHOCK_TUBE, PROBLEM_SHEET_LOBES = 5, 6
TILE_7x32, TILE_3x32 = 0, 1
WAVES = ("negative fast magnetosonic", "negative alfven", "negative slow magnetosonic",
         "entropy", "positive slow magnetosonic", "positive alfven",
         "positive fast magnetosonic")


@dataclass
class Run:
    """One run of a batch (the [problem] / [time] / [method] keys that matter)."""

    nx: int
    ny: int
    dx: float
    dy: float
    gamma: float
    bc: tuple
    scheme: int = ENO_ROE
    time_method: int = RK3
    dt_min: float = 1e-9
    dt_max: float = 1.0
    cfl: float = 0.4
    dt0: float = 1e-3
    t_end: float = 1.0
    max_steps: int = 0

    def desc(self):
        d = BatchDesc()
        d.nx, d.ny, d.dx, d.dy, d.gamma = self.nx, self.ny, self.dx, self.dy, self.gamma
        for s in range(4):
            d.bc[s] = int(self.bc[s])
        d.scheme, d.time_method = self.scheme, self.time_method
        d.dt_min, d.dt_max, d.cfl = self.dt_min, self.dt_max, self.cfl
        d.dt0, d.t_end, d.max_steps = self.dt0, self.t_end, self.max_steps
        return d


class Batch:
    def __init__(self, runs, device=0):
        self.lib = library()
        self.runs = list(runs)
        arr = (BatchDesc * len(self.runs))(*[r.desc() for r in self.runs])
        h = C.c_void_p()
        st = self.lib.mhd_batch_create(len(self.runs), arr, device, C.byref(h))
        if st != OK:
            msg = ""
            if h:
                msg = self._message(h)
                self.lib.mhd_batch_destroy(h)
            raise MhdError(f"mhd_batch_create failed: {STATUS_NAMES.get(st, st)} {msg}")
        self.h = h

    def _message(self, h=None):
        buf = C.create_string_buffer(1024)
        e = C.c_int(0)
        self.lib.mhd_batch_last_error(h or self.h, buf, 1024, C.byref(e))
        return buf.value.decode()

    def _check(self, st, what):
        if st != OK:
            raise MhdError(f"{what}: {STATUS_NAMES.get(st, st)} {self._message()}")
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.runs)

    def shape(self, i):
        r = self.runs[i]
        return (8, r.nx + 4, r.ny + 4)

    # -- data ------------------------------------------------------------------------
    def upload(self, i, U):
        self._check(self.lib.mhd_batch_upload(self.h, i, _p(np.ascontiguousarray(U))), "upload")

    def download(self, i, out=None):
        out = np.empty(self.shape(i)) if out is None else out
        self._check(self.lib.mhd_batch_download(self.h, i, _p(out)), "download")
        return out

    def init_problem(self, i, kind, params=()):
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        ptr = _p(p) if p.size else None
        self._check(self.lib.mhd_batch_init_problem(self.h, i, kind, ptr, int(p.size)),
                    "init_problem")

    def init_explosion(self, i, r=0.1, rho_in=1.0, p_in=10.0, rho_out=0.125, p_out=1.0,
                       bx=2 ** -0.5, by=2 ** -0.5):
        self.init_problem(i, PROBLEM_EXPLOSION, [0.0, 0.0, r, rho_in, p_in, rho_out, p_out, bx, by])

    def init_wave(self, i, wave, kx, ky, eps=1e-6, rho=1.0, u=0.0, v=0.0, w=0.0, bx=1.0,
                  by=2 ** 0.5, bz=0.5, p=None, lx=1.0, ly=1.0, x0=-0.5, y0=-0.5):
        p = 1.0 / self.runs[i].gamma if p is None else p
        self.init_problem(i, PROBLEM_WAVE, [x0, y0, lx, ly, rho, u, v, w, bx, by, bz, p, eps,
                                            float(wave), float(kx), float(ky)])

    def init_orszag_tang(self, i):
        self.init_problem(i, PROBLEM_ORSZAG_TANG, [])

    def init_plasma_sheet(self, i, amps, delta=0.1, x0=-2.0, y0=-1.0):
        a = list(amps)
        self.init_problem(i, PROBLEM_PLASMA_SHEET, [x0, y0, delta, float(len(a))] + a)

    def init_shock_tube(self, i, lx, ly, angle, left, right):
        """readProblemShockTube: left / right are natural states (rho, u, v,
        w, Bx, By, Bz, p); the run's dx, dy must be lx / nx, ly / ny."""
        self.init_problem(i, PROBLEM_SHOCK_TUBE, [lx, ly, angle] + list(left) + list(right))

    def init_sheet_lobes(self, i, lx, ly, start_x, start_y, head, foot, thickness, tanh_profile,
                         linear_transition, points, left, right, up, down):
        """readProblemPlasmaSheet (the reference's lobe / sheet setup): the four
        natural states (rho, u, v, w, Bx, By, Bz, p) of the left and right sheet
        halves and the upper and lower lobes."""
        p = [lx, ly, start_x, start_y, head, foot, thickness, float(bool(tanh_profile)),
             float(bool(linear_transition)), float(points)]
        self.init_problem(i, PROBLEM_SHEET_LOBES, p + list(left) + list(right) + list(up)
                          + list(down))

    # -- stepping --------------------------------------------------------------------
    def advance(self, stages, check_every=0):
        """Advance every active run by up to `stages` stages; returns the active count."""
        n = C.c_int(0)
        self._check(self.lib.mhd_batch_advance(self.h, int(stages), int(check_every),
                                               C.byref(n)), "advance")
        return n.value

    def run(self, max_stages=10 ** 9, check_every=48):
        """Advance until every run stopped (or max_stages)."""
        return self.advance(max_stages, check_every)

    def state(self, i):
        s = BatchState()
        self._check(self.lib.mhd_batch_get_state(self.h, i, C.byref(s)), "get_state")
        return {"t": s.t, "dt": s.dt, "steps": s.steps, "active": bool(s.active),
                "status": TStatus(s.status not in (0, 1, 2, 7), s.status), "phase": s.phase,
                "retries": s.retries, "neg_pressure": s.neg_pressure}

    def states(self):
        return [self.state(i) for i in range(len(self))]

    def tune(self, reps=2):
        t, c, ms = C.c_int(0), C.c_int(0), C.c_double(0)
        self._check(self.lib.mhd_batch_tune(self.h, reps, C.byref(t), C.byref(c), C.byref(ms)),
                    "tune")
        return {"tile": t.value, "ctas_per_sm": c.value, "ms_per_stage": ms.value}

    def set_tile(self, tile, ctas_per_sm=0):
        self._check(self.lib.mhd_batch_set_tile(self.h, tile, ctas_per_sm), "set_tile")

    def stream(self):
        s = C.c_void_p()
        self.lib.mhd_batch_stream(self.h, C.byref(s))
        return s.value or 0

    def launches(self):
        n = C.c_longlong(0)
        self.lib.mhd_batch_launches(self.h, C.byref(n))
        return n.value

    def cells(self):
        return np.array([r.nx * r.ny for r in self.runs], dtype=np.int64)

    def steps(self):
        return np.array([self.state(i)["steps"] for i in range(len(self))], dtype=np.int64)


@dataclass
class MixedRun:
    """One run of the mixed benchmark batch and its device-side initial state."""

    run: Run
    kind: str       # "explosion" or "wave"
    wave: int = 0
    kx: int = 1
    ky: int = 0

    def init(self, b, i):
        if self.kind == "explosion":
            b.init_explosion(i)
        else:
            b.init_wave(i, self.wave, self.kx, self.ky, eps=1e-6)


def shard_runs(costs, world, rank):
    """Indices of the runs rank `rank` of `world` takes: the runs are
    independent, so they are spread over the GPUs with no exchange at all.
    Longest processing time first: runs in decreasing cost (ties by index),
    each to the rank with the least cost so far (ties by rank).  Every rank
    computes the same assignment from the same costs."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    load = [0.0] * world
    mine = []
    for i in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += float(costs[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def mixed_runs(n=512, seed=0, side_min=64, side_max=1024, gamma=5.0 / 3.0):
    """The mixed batch of independent runs (seeded):

    * grid sides drawn log-uniformly in [side_min, side_max], nx and ny
      independently;
    * ENO-LF or ENO-Roe with probability 1/2, RK3, CFL 0.4, t_end ~ U[0.1, 1];
    * half 2-D explosions on [-0.5, 0.5]^2 with open sides (rho 1, p 10
      inside r < 0.1; rho 0.125, p 1 outside; B = (1, 1, 0)/sqrt 2);
    * half linear waves on the periodic unit box (rho 1, p 1/gamma,
      B = (1, sqrt 2, 0.5), a 1e-6 right-eigenvector perturbation of one of
      the 7 waves), integer wave vector (kx, ky) close to an angle drawn
      uniformly in [0, pi/2).
    """
    import math
    rng = np.random.default_rng(seed)
    lo, hi = math.log(side_min), math.log(side_max)
    out = []
    for r in range(n):
        nx = int(round(math.exp(rng.uniform(lo, hi))))
        ny = int(round(math.exp(rng.uniform(lo, hi))))
        scheme = 3 if rng.uniform() < 0.5 else 2
        t_end = float(rng.uniform(0.1, 1.0))
        common = dict(scheme=scheme, time_method=RK3, dt_min=1e-10, dt_max=2.0 ** -6,
                      cfl=0.4, dt0=2.0 ** -10, t_end=t_end)
        if r % 2 == 0:
            run = Run(nx, ny, 1.0 / nx, 1.0 / ny, gamma, (4, 4, 4, 4), **common)
            out.append(MixedRun(run, "explosion"))
        else:
            run = Run(nx, ny, 1.0 / nx, 1.0 / ny, gamma, (1, 1, 1, 1), **common)
            ang = rng.uniform(0.0, 0.5 * math.pi)
            kx, ky = int(round(4 * math.cos(ang))), int(round(4 * math.sin(ang)))
            if kx == 0 and ky == 0:
                kx = 1
            out.append(MixedRun(run, "wave", int(rng.integers(0, 7)), kx, ky))
    return out
