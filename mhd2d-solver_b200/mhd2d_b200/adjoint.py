"""Discrete adjoint of the ENO-Roe time step (mhd_adj_* in include/mhd2d_b200.h).

``Adjoint`` owns one run: an initial state, a recording forward run of
``nsteps`` steps (the same stepping as a ``Context``), and the reverse sweep
that gives dJ/dU0 for J = the kinetic energy sum |m|^2/(2 rho) dx dy of the
final state, with the recorded ENO choices and dt frozen.  ``replay`` runs
the frozen forward map from another initial state (for finite differences).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import OK, RK3, STATUS_NAMES, AdjStats, MhdError, _p, library
from .batch import PROBLEM_PLASMA_SHEET


class Adjoint:
    def __init__(self, nx, ny, dx, dy, gamma, bc, time_method=RK3, dt_min=1e-9, dt_max=1.0,
                 cfl=0.4, checkpoint_every=64, device=0):
        self.lib = library()
        self.nx, self.ny = int(nx), int(ny)
        self.shape = (8, self.nx + 4, self.ny + 4)
        h = C.c_void_p()
        bcs = (C.c_int * 4)(*[int(b) for b in bc])
        st = self.lib.mhd_adj_create(self.nx, self.ny, dx, dy, gamma, bcs, time_method, dt_min,
                                     dt_max, cfl, checkpoint_every, device, C.byref(h))
        if st != OK:
            if h:
                self.lib.mhd_adj_destroy(h)
            raise MhdError(f"mhd_adj_create failed: {STATUS_NAMES.get(st, st)}")
        self.h = h
        self.sheet = None  # (x0, y0, K) of a device-generated plasma sheet

    def _check(self, st, what):
        if st != OK:
            buf = C.create_string_buffer(1024)
            e = C.c_int(0)
            self.lib.mhd_adj_last_error(self.h, buf, 1024, C.byref(e))
            raise MhdError(f"{what}: {STATUS_NAMES.get(st, st)} {buf.value.decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_store(self, max_bytes=-1):
        """Device memory for kept stage inputs (-1 automatic, 0 none: replay every segment)."""
        self._check(self.lib.mhd_adj_set_store(self.h, int(max_bytes)), "set_store")

    def set_masks(self, keep_all=True):
        """Keep the ENO codes of every stage (True) or of stored stages only."""
        self._check(self.lib.mhd_adj_set_masks(self.h, 1 if keep_all else 0), "set_masks")

    def set_contract(self, enable=True):
        """Reverse sweep with FMA contraction (True, the default) or with the
        parity build's rounding throughout (False).  The recording is kept."""
        self._check(self.lib.mhd_adj_set_contract(self.h, 1 if enable else 0), "set_contract")

    # -- initial state ---------------------------------------------------------------
    def upload(self, U0):
        self._check(self.lib.mhd_adj_upload(self.h, _p(np.ascontiguousarray(U0))), "upload")

    @staticmethod
    def _sheet_params(amps, delta, x0, y0):
        a = [float(x) for x in amps]
        return np.array([x0, y0, delta, float(len(a))] + a)

    def init_plasma_sheet(self, amps, delta=0.1, x0=-2.0, y0=-1.0):
        p = self._sheet_params(amps, delta, x0, y0)
        self._check(self.lib.mhd_adj_init_problem(self.h, PROBLEM_PLASMA_SHEET, _p(p), p.size),
                    "init_problem")
        self.sheet = (x0, y0, len(p) - 4)

    # -- runs ------------------------------------------------------------------------
    def forward(self, nsteps, dt0):
        J = C.c_double(0)
        self._check(self.lib.mhd_adj_forward(self.h, int(nsteps), float(dt0), C.byref(J)),
                    "forward")
        return J.value

    def replay(self, U0=None):
        J = C.c_double(0)
        arg = None if U0 is None else _p(np.ascontiguousarray(U0))
        self._check(self.lib.mhd_adj_replay(self.h, arg, C.byref(J)), "replay")
        return J.value

    def replay_plasma_sheet(self, amps, delta=0.1, x0=-2.0, y0=-1.0):
        p = self._sheet_params(amps, delta, x0, y0)
        J = C.c_double(0)
        self._check(self.lib.mhd_adj_replay_problem(self.h, PROBLEM_PLASMA_SHEET, _p(p), p.size,
                                                    C.byref(J)), "replay_problem")
        return J.value

    def backward(self):
        self._check(self.lib.mhd_adj_backward(self.h), "backward")

    def gradient(self):
        out = np.empty(self.shape)
        self._check(self.lib.mhd_adj_gradient(self.h, _p(out)), "gradient")
        return out

    def sheet_gradient(self, K=None, x0=None, y0=None):
        sx0, sy0, sK = self.sheet if self.sheet else (-2.0, -1.0, 16)
        K = sK if K is None else K
        out = np.zeros(K)
        self._check(self.lib.mhd_adj_sheet_gradient(self.h, sx0 if x0 is None else x0,
                                                    sy0 if y0 is None else y0, K, _p(out)),
                    "sheet_gradient")
        return out

    def download(self, which=1):
        """which: 0 initial state, 1 final state of the recording, 2 working state."""
        out = np.empty(self.shape)
        self._check(self.lib.mhd_adj_download(self.h, which, _p(out)), "download")
        return out

    def info(self):
        s = AdjStats()
        self._check(self.lib.mhd_adj_info(self.h, C.byref(s)), "info")
        return {f: getattr(s, f) for f, _ in AdjStats._fields_}


def _group_handles(adjs):
    hs = (C.c_void_p * len(adjs))(*[a.h for a in adjs])
    return hs


def _group_error(adjs, st, what):
    for a in adjs:
        buf = C.create_string_buffer(1024)
        e = C.c_int(0)
        a.lib.mhd_adj_last_error(a.h, buf, 1024, C.byref(e))
        if e.value:
            raise MhdError(f"{what}: {STATUS_NAMES.get(st, st)} {buf.value.decode()}")
    raise MhdError(f"{what}: {STATUS_NAMES.get(st, st)}")


def forward_group(adjs, nsteps, dt0):
    """Recording forwards of several Adjoint objects at once (mhd_adj_forward_group).
    nsteps, dt0: one value or one per object.  Returns (list of J, device ms)."""
    n = len(adjs)
    lib = library()
    ns = np.broadcast_to(np.asarray(nsteps, dtype=np.int32), (n,)).copy()
    d0 = np.broadcast_to(np.asarray(dt0, dtype=np.float64), (n,)).copy()
    J = np.zeros(n)
    ms = C.c_double(0.0)
    st = lib.mhd_adj_forward_group(n, _group_handles(adjs), ns.ctypes.data_as(C.POINTER(C.c_int)),
                                   _p(d0), _p(J), C.byref(ms))
    if st != OK:
        _group_error(adjs, st, "forward_group")
    return [float(x) for x in J], ms.value


def backward_group(adjs):
    """Reverse sweeps of several recorded Adjoint objects at once.  Returns device ms."""
    lib = library()
    ms = C.c_double(0.0)
    st = lib.mhd_adj_backward_group(len(adjs), _group_handles(adjs), C.byref(ms))
    if st != OK:
        _group_error(adjs, st, "backward_group")
    return ms.value
