"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes bindings for the two CPU checkers:

* ``Oracle``     -> oracle/_build/libmhdoracle.so, the C restatement of the
                    reference hot path (mhd_oracle.c), always buildable;
* ``Reference``  -> oracle/_ref/libmhdref.so, the unmodified reference
                    sources (piccolo255/mhd2d-solver) linked with
                    ref_harness.cpp; present only where the reference
                    checkout was available at build time.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only to check or time the CPU side.  Arrays are the
reference's [k][i][j] blocks: float64, shape (8, nx+4, ny+4), C order.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libmhdoracle.so")
TLM_SO = os.path.join(HERE, "_build", "libmhdtlm.so")
REF_SO = os.path.join(HERE, "_ref", "libmhdref.so")
REF_BENCH = os.path.join(HERE, "_ref", "ref_bench")
REFIO_SO = os.path.join(HERE, "_ref", "libmhdrefio.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class SorParams(C.Structure):
    """Mirror of ``orc_sor_params`` / ``ref_sor_params`` ([divb corrector] keys)."""

    _fields_ = [
        ("divb_skip_steps", C.c_int),
        ("sor_steps", C.c_int),
        ("sor_rsteps", C.c_double),
        ("sor_rmax", C.c_double),
        ("sor_divbmax", C.c_double),
        ("omega_use_static", C.c_int),
        ("omega", C.c_double),
    ]


def sor_params(skip=1, steps=10, rsteps=100000, rmax=1e-10, divbmax=1e-10,
               use_static=True, omega=1.7):
    return SorParams(skip, steps, float(rsteps), rmax, divbmax, int(use_static), omega)


def _bc(bc):
    arr = (C.c_int * 4)(*[int(b) for b in bc])
    return arr


def load_oracle():
    if not os.path.exists(ORACLE_SO):
        raise FileNotFoundError(f"{ORACLE_SO} missing: run `make -C oracle`")
    lib = C.CDLL(ORACLE_SO)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                               C.c_double, _ip, C.c_double, C.c_double, C.c_double]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_init_dirichlet.argtypes = [C.c_void_p, _dp]
    lib.orc_apply_bc.argtypes = [C.c_void_p, _dp, _ip]
    lib.orc_integrate.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip]
    lib.orc_get_characteristics.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    lib.orc_update_dt.argtypes = [C.c_double, C.c_double, C.c_double, _dp, C.c_double, _ip]
    lib.orc_step.argtypes = [C.c_void_p, _dp, _dp, _ip]
    lib.orc_divb_calc.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.orc_divb_sor.argtypes = [C.c_void_p, C.POINTER(SorParams), _dp, C.c_int, _ip, _ip]
    lib.orc_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.POINTER(SorParams), C.c_int,
                            _dp, _dp, _dp, _ip, _dp, _dp, C.c_int, _ip]
    lib.orc_eigens_f.argtypes = [C.c_double, _dp, _dp, _dp, _dp, _dp, _ip]
    lib.orc_eigenvalues_at.argtypes = [C.c_double, _dp, _dp, _ip]
    lib.orc_lf_alpha_grid.argtypes = [C.c_double, C.c_int, C.c_int, _dp, _dp, _dp]
    lib.orc_set_lf_alpha.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_set_lf_alpha.restype = None
    lib.orc_retries.argtypes = [C.c_void_p]
    lib.orc_retries.restype = C.c_longlong
    return lib


TLM_NT = 17  # tangent directions of one tlm_run call (tlm.cpp)


def tlm_run(U0, dU0, nx, ny, dx, dy, gamma, bc, nsteps, dt0, time_method=2, dt_min=0.0,
            dt_max=1.0, cfl=0.4, scheme=2):
    """Tangent-linear run of the oracle (tlm.cpp): J and dJ/dU0 . dU0[r] for each
    of up to 17 directions dU0[r] (shape (ndir, 8, nx+4, ny+4)), frozen branches."""
    if not os.path.exists(TLM_SO):
        raise FileNotFoundError(f"{TLM_SO} missing: run `make -C oracle`")
    lib = C.CDLL(TLM_SO)
    lib.tlm_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                            C.c_double, _ip, C.c_double, C.c_double, C.c_double, C.c_int,
                            C.c_double, _dp, C.c_int, _dp, _dp, _dp, _dp, _ip]
    U0 = np.ascontiguousarray(U0, dtype=np.float64)
    dU0 = np.ascontiguousarray(dU0, dtype=np.float64).reshape(-1, *U0.shape)
    nd = dU0.shape[0]
    if nd > TLM_NT:
        raise ValueError("at most 17 directions per call")
    J = C.c_double(0.0)
    dJ = np.zeros(max(nd, 1))
    Uout = np.zeros_like(U0)
    steps = C.c_int(0)
    st = lib.tlm_run(scheme, time_method, nx, ny, dx, dy, gamma, _bc(bc), dt_min, dt_max, cfl,
                     nsteps, dt0, _p(U0), nd, _p(dU0), C.byref(J), _p(dJ), _p(Uout),
                     C.byref(steps))
    return dict(status=st, J=J.value, dJ=dJ[:nd], U=Uout, steps=steps.value)


def reference_available():
    return os.path.exists(REF_SO)


def grid_writer_available():
    return os.path.exists(REFIO_SO)


_refio = None


def ref_grid_records(U, dx, dy, gamma, bc, start_x=0.0, start_y=0.0, natural=True,
                     conservation=True, binary_double=True):
    """The bytes the reference's outputGridData writes for state U (its
    binary grid dump, file_access.cpp:1193-1325), from oracle/_ref/libmhdrefio.so.
    U is copied first: the writer overwrites B ghosts in place."""
    global _refio
    if _refio is None:
        if not os.path.exists(REFIO_SO):
            raise FileNotFoundError(f"{REFIO_SO} missing: run `make -C oracle ref`")
        lib = C.CDLL(REFIO_SO)
        lib.ref_grid_records.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_double, _ip, _dp, C.c_int, C.c_int,
                                         C.c_int, C.c_void_p, C.c_longlong]
        lib.ref_grid_records.restype = C.c_longlong
        _refio = lib
    W = np.ascontiguousarray(U, dtype=np.float64).copy()
    _, NX, NY = W.shape
    fields = 7 + (4 if natural else 0) + (4 if conservation else 0)
    cap = fields * (NX - 4) * (NY - 4) * 8
    buf = (C.c_char * cap)()
    n = _refio.ref_grid_records(NX - 4, NY - 4, dx, dy, gamma, start_x, start_y, _bc(bc), _p(W),
                                int(natural), int(conservation), int(binary_double), buf, cap)
    if n < 0:
        raise RuntimeError("ref_grid_records failed")
    return bytes(buf[:n])


def load_reference(fresh=False):
    """Load the reference library.  ``fresh=True`` loads a private copy so the
    reference's function-static SOR potential starts from zero."""
    if not os.path.exists(REF_SO):
        raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle ref`")
    path = REF_SO
    if fresh:
        d = tempfile.mkdtemp(prefix="mhdref_")
        path = os.path.join(d, "libmhdref.so")
        shutil.copy(REF_SO, path)
    lib = C.CDLL(path)
    lib.ref_integrate.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                  _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip,
                                  C.c_char_p, C.c_int]
    lib.ref_update_dt.argtypes = [C.c_double, C.c_double, C.c_double, _dp, C.c_double, _ip]
    lib.ref_divb_calc.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _ip, _dp, _dp, _dp]
    lib.ref_nongrid_data.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _ip,
                                     _dp, _dp]
    lib.ref_nongrid_data.restype = None
    lib.ref_divb_sor.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _ip,
                                 C.POINTER(SorParams), _dp, _ip]
    lib.ref_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                            C.c_double, _ip, C.c_double, C.c_double, C.c_double, C.c_int,
                            C.c_double, C.POINTER(SorParams), _dp, _dp, _dp, _ip, _dp, _dp,
                            C.c_int, _dp, _dp, _dp, _dp, _ip, C.c_char_p, C.c_int]
    return lib


class Oracle:
    """One oracle context: mirrors a reference method + stepper pair."""

    def __init__(self, nx, ny, dx, dy, gamma, bc, scheme=2, time_method=2,
                 dt_min=0.0, dt_max=1.0, cfl=0.4, lib=None):
        self.lib = lib or load_oracle()
        self.nx, self.ny = nx, ny
        self.ctx = self.lib.orc_create(scheme, time_method, nx, ny, dx, dy, gamma, _bc(bc),
                                       dt_min, dt_max, cfl)

    def __del__(self):
        if getattr(self, "ctx", None):
            self.lib.orc_destroy(self.ctx)
            self.ctx = None

    def shape(self):
        return (8, self.nx + 4, self.ny + 4)

    def init_dirichlet(self, U):
        self.lib.orc_init_dirichlet(self.ctx, _p(U))

    def apply_bc(self, U):
        e = C.c_int(0)
        st = self.lib.orc_apply_bc(self.ctx, _p(U), C.byref(e))
        return st, e.value

    def retries(self):
        return int(self.lib.orc_retries(self.ctx))

    def set_lf_alpha(self, aF=None, aG=None):
        """Fix the ENO-LF dissipation coefficients (aF [8][ny+4], aG [8][nx+4])
        for the following integrations; no arguments: computed again."""
        if aF is None:
            self.lib.orc_set_lf_alpha(self.ctx, None, None)
        else:
            self.lib.orc_set_lf_alpha(self.ctx, _p(np.ascontiguousarray(aF)),
                                      _p(np.ascontiguousarray(aG)))

    def integrate(self, U, UL=None):
        UL = np.zeros(self.shape()) if UL is None else UL
        d = C.c_double(0.0)
        e = C.c_int(0)
        st = self.lib.orc_integrate(self.ctx, _p(U), _p(UL), C.byref(d), C.byref(e))
        return st, e.value, UL, d.value

    def characteristics(self):
        out = [np.zeros(self.shape()) for _ in range(4)]
        self.lib.orc_get_characteristics(self.ctx, *[_p(a) for a in out])
        return out

    def step(self, U, dt):
        d = C.c_double(dt)
        e = C.c_int(0)
        st = self.lib.orc_step(self.ctx, _p(U), C.byref(d), C.byref(e))
        return st, e.value, d.value

    def divb_calc(self, U):
        m, t = C.c_double(0), C.c_double(0)
        self.lib.orc_divb_calc(self.ctx, _p(U), C.byref(m), C.byref(t))
        return m.value, t.value

    def divb_sor(self, U, sp, red_black=0):
        sw, e = C.c_int(0), C.c_int(0)
        st = self.lib.orc_divb_sor(self.ctx, C.byref(sp), _p(U), red_black, C.byref(sw),
                                   C.byref(e))
        return st, e.value, sw.value

    def run(self, U, dt, nsteps=0, t_max=0.0, sor=None, red_black=0, hist_len=0):
        d, t = C.c_double(dt), C.c_double(0.0)
        n, e = C.c_int(0), C.c_int(0)
        dth = np.zeros(max(hist_len, 1))
        dbh = np.zeros(max(hist_len, 1))
        st = self.lib.orc_run(self.ctx, nsteps, t_max, C.byref(sor) if sor else None, red_black,
                              _p(U), C.byref(d), C.byref(t), C.byref(n), _p(dth), _p(dbh),
                              hist_len, C.byref(e))
        return dict(status=st, is_error=e.value, dt=d.value, t=t.value, steps=n.value,
                    dt_hist=dth[:min(n.value, hist_len)], divb_hist=dbh[:min(n.value, hist_len)])


def lf_alpha_grid(U, gamma, lib=None):
    """ENO-LF dissipation coefficients of a whole grid whose ghost layers
    are filled: (aF [8][ny+4], aG [8][nx+4])."""
    lib = lib or load_oracle()
    _, NX, NY = U.shape
    aF, aG = np.zeros((8, NY)), np.zeros((8, NX))
    st = lib.orc_lf_alpha_grid(gamma, NX - 4, NY - 4, _p(U), _p(aF), _p(aG))
    if st:
        raise RuntimeError(f"lf_alpha_grid: status {st}")
    return aF, aG


def oracle_update_dt(dt_min, dt_max, cfl, dt, ideal, lib=None):
    lib = lib or load_oracle()
    d, e = C.c_double(dt), C.c_int(0)
    st = lib.orc_update_dt(dt_min, dt_max, cfl, C.byref(d), ideal, C.byref(e))
    return st, e.value, d.value


class Reference:
    """Thin wrapper of the reference library calls (fresh objects per call)."""

    def __init__(self, fresh=False):
        self.lib = load_reference(fresh=fresh)

    def integrate(self, scheme, U, dx, dy, gamma, bc, U_dirichlet=None, chars=False):
        _, NX, NY = U.shape
        nx, ny = NX - 4, NY - 4
        UL = np.zeros_like(U)
        d, e = C.c_double(0.0), C.c_int(0)
        msg = C.create_string_buffer(512)
        ch = [np.zeros_like(U) for _ in range(4)] if chars else [None] * 4
        Ud = U.copy() if U_dirichlet is None else U_dirichlet
        st = self.lib.ref_integrate(scheme, nx, ny, dx, dy, gamma, _bc(bc), _p(Ud), _p(U), _p(UL),
                                    C.byref(d), _p(ch[0]), _p(ch[1]), _p(ch[2]), _p(ch[3]),
                                    C.byref(e), msg, 512)
        return dict(status=st, is_error=e.value, UL=UL, dtIdeal=d.value,
                    cx=ch[0], cy=ch[1], LUx=ch[2], LUy=ch[3], message=msg.value.decode())

    def update_dt(self, dt_min, dt_max, cfl, dt, ideal):
        d, e = C.c_double(dt), C.c_int(0)
        st = self.lib.ref_update_dt(dt_min, dt_max, cfl, C.byref(d), ideal, C.byref(e))
        return st, e.value, d.value

    def divb_calc(self, U, dx, dy, bc):
        _, NX, NY = U.shape
        m, t = C.c_double(0), C.c_double(0)
        self.lib.ref_divb_calc(NX - 4, NY - 4, dx, dy, _bc(bc), _p(U), C.byref(m), C.byref(t))
        return m.value, t.value

    def nongrid_data(self, U, dx, dy, gamma, bc):
        """(u_max, divb_max, divb_sum, mass, momentum, energy, entropy) of the reference's
        non-grid output record (fills periodic B ghosts of U, as divBCalculation does)."""
        _, NX, NY = U.shape
        out = np.zeros(7)
        self.lib.ref_nongrid_data(NX - 4, NY - 4, dx, dy, gamma, _bc(bc), _p(U), _p(out))
        return tuple(float(x) for x in out)

    def divb_sor(self, U, dx, dy, bc, sp):
        _, NX, NY = U.shape
        e = C.c_int(0)
        st = self.lib.ref_divb_sor(NX - 4, NY - 4, dx, dy, _bc(bc), C.byref(sp), _p(U), C.byref(e))
        return st, e.value

    def run(self, scheme, time_method, U, dx, dy, gamma, bc, dt, dt_min, dt_max, cfl,
            nsteps=0, t_max=0.0, sor=None, hist_len=0, chars=False):
        _, NX, NY = U.shape
        d, t = C.c_double(dt), C.c_double(0.0)
        n, e = C.c_int(0), C.c_int(0)
        dth = np.zeros(max(hist_len, 1))
        dbh = np.zeros(max(hist_len, 1))
        ch = [np.zeros_like(U) for _ in range(4)] if chars else [None] * 4
        msg = C.create_string_buffer(512)
        st = self.lib.ref_run(scheme, time_method, NX - 4, NY - 4, dx, dy, gamma, _bc(bc),
                              dt_min, dt_max, cfl, nsteps, t_max, C.byref(sor) if sor else None,
                              _p(U), C.byref(d), C.byref(t), C.byref(n), _p(dth), _p(dbh),
                              hist_len, _p(ch[0]), _p(ch[1]), _p(ch[2]), _p(ch[3]),
                              C.byref(e), msg, 512)
        return dict(status=st, is_error=e.value, dt=d.value, t=t.value, steps=n.value,
                    dt_hist=dth[:min(n.value, hist_len)], divb_hist=dbh[:min(n.value, hist_len)],
                    cx=ch[0], cy=ch[1], LUx=ch[2], LUy=ch[3], message=msg.value.decode())
