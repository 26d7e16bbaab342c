"""Initial states for tests and benchmarks (host-side numpy).

Every state is the reference's conserved-variable block
``U[k][i][j]`` (k = rho, mx, my, mz, Bx, By, Bz, E), float64, shape
``(8, nx+4, ny+4)`` with two ghost cells per side.  Natural variables are
converted with the reference's formula (conversions.cpp:59-77):
``E = p/(gamma-1) + rho*|u|^2/2 + |B|^2/2``.

The problem descriptions follow the reference's problem setups
(file_access.cpp) and the benchmark configurations of this project:

* ``ot_vortex``   — Orszag-Tang vortex on [0, 2pi]^2, periodic
                    (file_access.cpp:578-613);
* ``brio_wu``     — Brio-Wu shock tube as a 2-D grid, Neumann on all sides
                    (file_access.cpp:302-395 with angle 0);
* ``explosion``   — circular blast, open boundaries;
* ``random_smooth`` / ``random_blocky`` — seeded synthetic states for
                    parity tests (smooth and discontinuous);
* ``plasma_sheet`` — the current sheet of the adjoint benchmark
                    (By = tanh(x/delta), a velocity perturbation with
                    amplitudes a_k) and its tangents dU0/da_k.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PERIODIC, DIRICHLET, NEUMANN, OPEN = 1, 2, 3, 4


@dataclass
class Problem:
    U: np.ndarray
    dx: float
    dy: float
    gamma: float
    bc: tuple  # left, right, bottom, top
    name: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def nx(self):
        return self.U.shape[1] - 4

    @property
    def ny(self):
        return self.U.shape[2] - 4


def to_conserved(rho, u, v, w, bx, by, bz, p, gamma):
    """Natural -> conserved variables, same association as conversions.cpp:59-77."""
    nx, ny = rho.shape
    U = np.zeros((8, nx + 4, ny + 4))
    s = (slice(2, nx + 2), slice(2, ny + 2))
    U[0][s] = rho
    U[1][s] = u * rho
    U[2][s] = v * rho
    U[3][s] = w * rho
    U[4][s] = bx
    U[5][s] = by
    U[6][s] = bz
    uu = u * u + v * v + w * w
    bb = bx * bx + by * by + bz * bz
    U[7][s] = p / (gamma - 1.0) + 0.5 * rho * uu + 0.5 * bb
    return U


def ot_vortex(nx, ny=None, gamma=5.0 / 3.0):
    ny = nx if ny is None else ny
    dx, dy = 2.0 * math.pi / nx, 2.0 * math.pi / ny
    x = (np.arange(nx) * dx)[:, None] * np.ones((1, ny))
    y = np.ones((nx, 1)) * (np.arange(ny) * dy)[None, :]
    one = np.ones((nx, ny))
    U = to_conserved(gamma * gamma * one, -np.sin(y), np.sin(x), 0 * one, -np.sin(y),
                     np.sin(2 * x), 0 * one, gamma * one, gamma)
    return Problem(U, dx, dy, gamma, (PERIODIC,) * 4, "ot_vortex")


def brio_wu(nx=256, ny=8, gamma=2.0, lx=2.0, ly=0.5):
    dx, dy = lx / nx, ly / ny
    left = (1.0, 0.0, 0.0, 0.0, 0.75, 1.0, 0.0, 1.0)
    right = (0.125, 0.0, 0.0, 0.0, 0.75, -1.0, 0.0, 0.1)
    x0 = 0.5 * lx - 0.5 * dx
    is_left = (np.arange(nx) * dx < x0)[:, None] * np.ones((1, ny), dtype=bool)
    q = [np.where(is_left, a, b) for a, b in zip(left, right)]
    U = to_conserved(*q, gamma)
    return Problem(U, dx, dy, gamma, (NEUMANN,) * 4, "brio_wu")


def explosion(nx, ny=None, gamma=5.0 / 3.0, radius=0.1, bc=(OPEN,) * 4):
    ny = nx if ny is None else ny
    dx, dy = 1.0 / nx, 1.0 / ny
    x = (-0.5 + (np.arange(nx) + 0.5) * dx)[:, None]
    y = (-0.5 + (np.arange(ny) + 0.5) * dy)[None, :]
    inside = (x * x + y * y) < radius * radius
    one = np.ones((nx, ny))
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 10.0, 1.0)
    b = 1.0 / math.sqrt(2.0)
    U = to_conserved(rho, 0 * one, 0 * one, 0 * one, b * one, b * one, 0 * one, p, gamma)
    return Problem(U, dx, dy, gamma, tuple(bc), "explosion")


def random_smooth(nx, ny, seed=0, gamma=5.0 / 3.0, bc=(PERIODIC,) * 4, amp=0.2):
    rng = np.random.default_rng(seed)
    dx, dy = 1.0 / nx, 1.0 / ny
    x = (np.arange(nx) + 0.5)[:, None] * dx
    y = (np.arange(ny) + 0.5)[None, :] * dy

    def wave(base, a):
        kx, ky = rng.integers(1, 3, size=2)
        ph = rng.uniform(0, 2 * math.pi, size=2)
        return base + a * np.sin(2 * math.pi * kx * x + ph[0]) * np.cos(2 * math.pi * ky * y + ph[1])

    rho = wave(1.0, amp)
    u, v, w = wave(0.1, amp), wave(-0.1, amp), wave(0.05, amp)
    bx, by, bz = wave(0.7, amp), wave(0.4, amp), wave(0.2, amp)
    p = wave(1.0, amp)
    U = to_conserved(rho, u, v, w, bx, by, bz, p, gamma)
    return Problem(U, dx, dy, gamma, tuple(bc), f"random_smooth[{seed}]")


def random_blocky(nx, ny, seed=0, gamma=5.0 / 3.0, bc=(PERIODIC,) * 4, nblocks=4):
    """Piecewise-constant random blocks: shocks / contacts on both axes."""
    rng = np.random.default_rng(seed)
    dx, dy = 1.0 / nx, 1.0 / ny
    bi = np.minimum((np.arange(nx) * nblocks) // nx, nblocks - 1)
    bj = np.minimum((np.arange(ny) * nblocks) // ny, nblocks - 1)

    def field(lo, hi):
        vals = rng.uniform(lo, hi, size=(nblocks, nblocks))
        return vals[bi][:, bj]

    rho = field(0.2, 2.0)
    u, v, w = field(-0.5, 0.5), field(-0.5, 0.5), field(-0.3, 0.3)
    bx, by, bz = field(-1.0, 1.0), field(-1.0, 1.0), field(-0.5, 0.5)
    p = field(0.1, 2.0)
    U = to_conserved(rho, u, v, w, bx, by, bz, p, gamma)
    return Problem(U, dx, dy, gamma, tuple(bc), f"random_blocky[{seed}]")


def plasma_sheet(nx, ny, amps, delta=0.1, gamma=5.0 / 3.0, lx=4.0, ly=2.0, x0=-2.0, y0=-1.0,
                 bc=(NEUMANN, NEUMANN, PERIODIC, PERIODIC)):
    """By = tanh(x/delta), Bx = Bz = 0, T = 0.5, p = 1.25 - By^2/2, rho = p/T,
    v = sum_k a_k sin(k pi y) exp(-x^2/0.04); cell i at x0 + i dx (the
    reference's coordinate convention, file_access.cpp:598-599)."""
    dx, dy = lx / nx, ly / ny
    x = (x0 + np.arange(nx) * dx)[:, None] * np.ones((1, ny))
    y = np.ones((nx, 1)) * (y0 + np.arange(ny) * dy)[None, :]
    by = np.tanh(x / delta)
    p = 1.25 - 0.5 * by * by
    rho = p / 0.5
    env = np.exp(-x * x / 0.04)
    v = np.zeros_like(x)
    for k, a in enumerate(amps, start=1):
        v = v + a * np.sin(k * math.pi * y) * env
    z = np.zeros_like(x)
    U = to_conserved(rho, z, v, z, z, by, z, p, gamma)
    return Problem(U, dx, dy, gamma, tuple(bc), "plasma_sheet",
                   extra={"amps": list(amps), "delta": delta, "x0": x0, "y0": y0})


def plasma_sheet_tangents(p):
    """dU0/da_k of plasma_sheet, shape (K, 8, nx+4, ny+4)."""
    nx, ny = p.nx, p.ny
    x = (p.extra["x0"] + np.arange(nx) * p.dx)[:, None] * np.ones((1, ny))
    y = np.ones((nx, 1)) * (p.extra["y0"] + np.arange(ny) * p.dy)[None, :]
    rho = p.U[0, 2:-2, 2:-2]
    v = p.U[2, 2:-2, 2:-2] / rho
    env = np.exp(-x * x / 0.04)
    K = len(p.extra["amps"])
    T = np.zeros((K,) + p.U.shape)
    for k in range(1, K + 1):
        s = np.sin(k * math.pi * y) * env
        T[k - 1, 2, 2:-2, 2:-2] = rho * s
        T[k - 1, 7, 2:-2, 2:-2] = rho * v * s
    return T
