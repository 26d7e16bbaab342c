"""Python binding of libmhd2d_b200.so (the C ABI in include/mhd2d_b200.h).

The classes mirror the reference solver's plugin interface for the time-step
hot path (piccolo255/mhd2d-solver):

* ``SpatialMethodEnoRoe`` / ``SpatialMethodEnoLF``  — SpatialIntegrationMethod
  (spatialintegrationmethod.hpp:6-65): ``initializeDirichletBoundaries``,
  ``integrate(U, UL) -> (t_status, dtIdeal)``, ``getCharacteristicsX/Y``;
* ``TimeIntegrationRK3`` / ``TimeIntegrationEuler`` — TimeIntegrationMethod
  (timeintegrationmethod.hpp:6-53): ``step(U, cx, cy, LUx, LUy, borderFlux,
  dtCurrent) -> (t_status, dtCurrent)``;
* ``divBCalculation`` / ``divBCorrectionSOR`` — the div_b_fix.cpp functions.

``Context`` is the lower-level device-resident handle (upload once, step many
times, download when needed).  States are numpy float64 arrays of shape
(8, nx+4, ny+4), the reference's U[0][0] block.  There is no CPU fallback:
importing fails loudly when the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libmhd2d_b200.so")

# ReturnStatus (enums.hpp)
OK, NO_CHANGE, UPDATED = 0, 1, 2
ERR_NOT_IMPLEMENTED, ERR_TIME_UNDERFLOW, ERR_NOT_CONVERGED = 3, 4, 5
ERR_NEGATIVE_DENSITY, ERR_NEGATIVE_PRESSURE = 6, 7
ERR_WRONG_PARAMETER, ERR_CUDA = 10, 100
STATUS_NAMES = {0: "OK", 1: "NoChange", 2: "Updated", 3: "ErrorNotImplemented",
                4: "ErrorTimeUnderflow", 5: "ErrorNotConverged", 6: "ErrorNegativeDensity",
                7: "ErrorNegativePressure", 8: "ErrorFileNotFound", 9: "ErrorFailedToParse",
                10: "ErrorWrongParameter", 100: "ErrorCuda"}

PERIODIC, DIRICHLET, NEUMANN, OPEN = 1, 2, 3, 4
CENTRAL_FD, ENO_ROE, ENO_LF = 1, 2, 3
EULER, RK3 = 1, 2
FLAG_CHARACTERISTICS, FLAG_FAST_MATH = 0x1, 0x2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class AdjStats(C.Structure):
    """mhd_adj_stats."""

    _fields_ = [("steps", C.c_int), ("stages", C.c_int), ("checkpoints", C.c_int),
                ("retries", C.c_int), ("t", C.c_double), ("dt", C.c_double),
                ("ms_forward", C.c_double), ("ms_backward", C.c_double),
                ("ms_replay", C.c_double), ("launches", C.c_longlong),
                ("stored_stages", C.c_int), ("replayed_segments", C.c_int)]


class BatchDesc(C.Structure):
    """mhd_batch_desc: one run of a batch."""

    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("gamma", C.c_double), ("bc", C.c_int * 4), ("scheme", C.c_int),
                ("time_method", C.c_int), ("dt_min", C.c_double), ("dt_max", C.c_double),
                ("cfl", C.c_double), ("dt0", C.c_double), ("t_end", C.c_double),
                ("max_steps", C.c_int)]


class BatchState(C.Structure):
    """mhd_batch_state: progress of one run."""

    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("steps", C.c_int), ("active", C.c_int),
                ("status", C.c_int), ("phase", C.c_int), ("retries", C.c_longlong),
                ("neg_pressure", C.c_longlong)]


class SorParams(C.Structure):
    """mhd_sor_params: the [divb corrector] keys (file_access.cpp:273-299)."""

    _fields_ = [("divb_skip_steps", C.c_int), ("sor_steps", C.c_int),
                ("sor_rsteps", C.c_double), ("sor_rmax", C.c_double),
                ("sor_divbmax", C.c_double), ("omega_use_static", C.c_int),
                ("omega", C.c_double)]


class RunParams(C.Structure):
    """mhd_run_params: the main loop's stop rule, cleaning and non-grid output cadence."""

    _fields_ = [("time_mode", C.c_int), ("steps", C.c_int), ("t_max", C.c_double),
                ("dt0", C.c_double), ("sor", SorParams), ("nongrid_mode", C.c_int),
                ("nongrid_steps", C.c_int), ("nongrid_t", C.c_double)]


class NongridRecord(C.Structure):
    """mhd_nongrid_record: step, t, dt and the 7 numbers of mhd_nongrid_data."""

    _fields_ = [("step", C.c_int), ("t", C.c_double), ("dt", C.c_double),
                ("values", C.c_double * 7)]


class GridPackParams(C.Structure):
    """mhd_grid_pack_params."""

    _fields_ = [("natural", C.c_int), ("conservation", C.c_int), ("single", C.c_int),
                ("start_x", C.c_double), ("start_y", C.c_double)]


class RunResult(C.Structure):
    """mhd_run_result."""

    _fields_ = [("steps", C.c_int), ("t", C.c_double), ("dt", C.c_double), ("status", C.c_int),
                ("is_error", C.c_int), ("nan_stop", C.c_int), ("records", C.c_int),
                ("sor_sweeps", C.c_longlong)]


def set_tile_tma(enable=None):
    """Stage flux tiles by TMA (True) or per-element async copies (False); None keeps the
    setting.  Returns the number of TMA-staged flux launches so far."""
    n = C.c_longlong(0)
    st = library().mhd_set_tile_tma(-1 if enable is None else int(bool(enable)), C.byref(n))
    if st != OK:
        raise MhdError(f"mhd_set_tile_tma: {STATUS_NAMES.get(st, st)}")
    return n.value


def sor_params(skip=1, steps=10, rsteps=100000, rmax=1e-10, divbmax=1e-10, use_static=True,
               omega=1.7):
    return SorParams(skip, steps, float(rsteps), rmax, divbmax, int(use_static), omega)


def library():
    """Load libmhd2d_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built: run `make -C mhd2d-solver_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "mhd_ctx_create": [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _ip,
                           C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                           C.POINTER(vp)],
        "mhd_ctx_destroy": [vp],
        "mhd_last_error": [vp, C.c_char_p, C.c_size_t, _ip],
        "mhd_upload": [vp, _dp],
        "mhd_download": [vp, _dp],
        "mhd_download_ul": [vp, _dp],
        "mhd_init_dirichlet": [vp],
        "mhd_set_dirichlet": [vp, _dp, _dp, _dp, _dp],
        "mhd_integrate": [vp, _dp],
        "mhd_integrate_host": [vp, _dp, _dp, _dp],
        "mhd_set_stepper": [vp, C.c_int, C.c_double, C.c_double, C.c_double],
        "mhd_step": [vp, _dp],
        "mhd_step_host": [vp, _dp, _dp],
        "mhd_steps": [vp, C.c_int, _dp, _dp],
        "mhd_set_step_graph": [vp, C.c_int],
        "mhd_get_characteristics": [vp, _dp, _dp, _dp, _dp],
        "mhd_divb_calc": [vp, _dp, _dp],
        "mhd_nongrid_data": [vp, _dp],
        "mhd_grid_pack": [vp, C.POINTER(GridPackParams), C.c_void_p, C.c_size_t,
                          C.POINTER(C.c_size_t)],
        "mhd_set_tile_tma": [C.c_int, C.POINTER(C.c_longlong)],
        "mhd_set_sor_fused": [vp, C.c_int],
        "mhd_set_sor_rows": [vp, C.c_int],
        "mhd_set_sor_graph": [vp, C.c_int],
        "mhd_set_step_host_banded": [vp, C.c_int],
        "mhd_run": [vp, C.POINTER(RunParams), C.POINTER(NongridRecord), C.c_int,
                    C.POINTER(RunResult)],
        "mhd_divb_sor": [vp, C.POINTER(SorParams), _ip],
        "mhd_divb_clean": [vp, C.POINTER(SorParams), _dp, _ip],
        "mhd_get_counters": [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
        "mhd_layout": [vp, _ip, _ip],
        "mhd_stream": [vp, C.POINTER(vp)],
        "mhd_time_integrate": [vp, C.c_int, _dp],
        "mhd_fp64_peak": [C.c_int, _dp],
        "mhd_divb_calc_noalloc": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.c_double, _ip, C.c_void_p, C.c_void_p],
        "mhd_batch_create": [C.c_int, C.POINTER(BatchDesc), C.c_int, C.POINTER(vp)],
        "mhd_batch_destroy": [vp],
        "mhd_batch_last_error": [vp, C.c_char_p, C.c_size_t, _ip],
        "mhd_batch_upload": [vp, C.c_int, _dp],
        "mhd_batch_download": [vp, C.c_int, _dp],
        "mhd_batch_advance": [vp, C.c_int, C.c_int, _ip],
        "mhd_batch_get_state": [vp, C.c_int, C.POINTER(BatchState)],
        "mhd_batch_tune": [vp, C.c_int, _ip, _ip, _dp],
        "mhd_batch_set_tile": [vp, C.c_int, C.c_int],
        "mhd_batch_init_problem": [vp, C.c_int, C.c_int, _dp, C.c_int],
        "mhd_batch_stream": [vp, C.POINTER(vp)],
        "mhd_batch_launches": [vp, C.POINTER(C.c_longlong)],
        "mhd_adj_create": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _ip, C.c_int,
                           C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(vp)],
        "mhd_adj_destroy": [vp],
        "mhd_adj_set_store": [vp, C.c_longlong],
        "mhd_adj_set_masks": [vp, C.c_int],
        "mhd_adj_set_contract": [vp, C.c_int],
        "mhd_adj_last_error": [vp, C.c_char_p, C.c_size_t, _ip],
        "mhd_adj_upload": [vp, _dp],
        "mhd_adj_init_problem": [vp, C.c_int, _dp, C.c_int],
        "mhd_adj_forward": [vp, C.c_int, C.c_double, _dp],
        "mhd_adj_replay": [vp, _dp, _dp],
        "mhd_adj_replay_problem": [vp, C.c_int, _dp, C.c_int, _dp],
        "mhd_adj_backward": [vp],
        "mhd_adj_gradient": [vp, _dp],
        "mhd_adj_sheet_gradient": [vp, C.c_double, C.c_double, C.c_int, _dp],
        "mhd_adj_download": [vp, C.c_int, _dp],
        "mhd_adj_info": [vp, C.POINTER(AdjStats)],
        "mhd_adj_forward_group": [C.c_int, C.POINTER(vp), C.POINTER(C.c_int),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)],
        "mhd_adj_backward_group": [C.c_int, C.POINTER(vp), C.POINTER(C.c_double)],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = lib
    return lib


def _p(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("state arrays must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


@dataclass
class TStatus:
    """t_status (mhd2d.hpp:121-125)."""

    isError: bool
    status: int
    message: str = ""

    @property
    def name(self):
        return STATUS_NAMES.get(self.status, str(self.status))


class MhdError(RuntimeError):
    pass


class Context:
    """Device-resident state + method + stepper (one mhd_ctx)."""

    def __init__(self, nx, ny, dx, dy, gamma, bc, scheme=ENO_ROE, time_method=RK3,
                 dt_min=0.0, dt_max=1.0, cfl=0.4, flags=0, device=0, halo=2):
        self.lib = library()
        self.nx, self.ny = int(nx), int(ny)
        self.shape = (8, self.nx + 4, self.ny + 4)
        self.flags = flags
        h = C.c_void_p()
        bcs = (C.c_int * 4)(*[int(b) for b in bc])
        st = self.lib.mhd_ctx_create(self.nx, self.ny, halo, dx, dy, gamma, bcs, scheme,
                                     time_method, dt_min, dt_max, cfl, flags, device, C.byref(h))
        if st != OK:
            raise MhdError(f"mhd_ctx_create failed: {STATUS_NAMES.get(st, st)}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- status -----------------------------------------------------------------------
    def last_status(self, st):
        buf = C.create_string_buffer(1024)
        e = C.c_int(0)
        self.lib.mhd_last_error(self.h, buf, 1024, C.byref(e))
        return TStatus(bool(e.value), int(st), buf.value.decode())

    def _check(self, st, what):
        if st == ERR_CUDA:
            raise MhdError(f"{what}: {self.last_status(st).message}")
        return st

    # -- data -------------------------------------------------------------------------
    def upload(self, U):
        self._check(self.lib.mhd_upload(self.h, _p(np.ascontiguousarray(U))), "upload")

    def download(self, out=None):
        out = np.empty(self.shape) if out is None else out
        self._check(self.lib.mhd_download(self.h, _p(out)), "download")
        return out

    def download_ul(self, out=None):
        out = np.zeros(self.shape) if out is None else out
        self._check(self.lib.mhd_download_ul(self.h, _p(out)), "download_ul")
        return out

    def init_dirichlet(self):
        self._check(self.lib.mhd_init_dirichlet(self.h), "init_dirichlet")

    # -- hot path ---------------------------------------------------------------------
    def set_stepper(self, time_method, dt_min, dt_max, cfl):
        st = self._check(self.lib.mhd_set_stepper(self.h, time_method, dt_min, dt_max, cfl),
                         "set_stepper")
        if st != OK:
            raise MhdError(self.last_status(st).message)

    def integrate(self):
        d = C.c_double(0.0)
        st = self._check(self.lib.mhd_integrate(self.h, C.byref(d)), "integrate")
        return self.last_status(st), d.value

    def integrate_host(self, U, UL=None):
        UL = np.zeros(self.shape) if UL is None else UL
        d = C.c_double(0.0)
        st = self._check(self.lib.mhd_integrate_host(self.h, _p(U), _p(UL), C.byref(d)),
                         "integrate_host")
        return self.last_status(st), UL, d.value

    def step(self, dt):
        d = C.c_double(dt)
        st = self._check(self.lib.mhd_step(self.h, C.byref(d)), "step")
        return self.last_status(st), d.value

    def step_host(self, U, dt):
        d = C.c_double(dt)
        st = self._check(self.lib.mhd_step_host(self.h, _p(U), C.byref(d)), "step_host")
        return self.last_status(st), d.value

    def steps(self, n, dt, record=False):
        d = C.c_double(dt)
        dts = np.zeros(max(n, 1)) if record else None
        st = self._check(self.lib.mhd_steps(self.h, n, C.byref(d), _p(dts)), "steps")
        return self.last_status(st), d.value, (dts[:n] if record else None)

    def characteristics(self):
        out = [np.zeros(self.shape) for _ in range(4)]
        st = self._check(self.lib.mhd_get_characteristics(self.h, *[_p(a) for a in out]),
                         "characteristics")
        if st == NO_CHANGE:  # central FD keeps none: the arrays stay as they are
            return out
        if st != OK:
            raise MhdError(self.last_status(st).message)
        return out

    def divb_calc(self):
        m, t = C.c_double(0), C.c_double(0)
        self._check(self.lib.mhd_divb_calc(self.h, C.byref(m), C.byref(t)), "divb_calc")
        return m.value, t.value

    def nongrid_data(self):
        """(u_max, divb_max, divb_sum, mass, momentum, energy, entropy) of the state."""
        out = np.zeros(7)
        self._check(self.lib.mhd_nongrid_data(self.h, _p(out)), "nongrid_data")
        return tuple(float(x) for x in out)

    def grid_records(self, natural=True, conservation=True, single=False, start_x=0.0,
                     start_y=0.0):
        """The reference's binary grid dump of the state (mhd_grid_pack), as bytes."""
        gp = GridPackParams(int(natural), int(conservation), int(single), start_x, start_y)
        n = C.c_size_t(0)
        self._check(self.lib.mhd_grid_pack(self.h, C.byref(gp), None, 0, C.byref(n)),
                    "grid_pack")
        buf = (C.c_char * n.value)()
        st = self.lib.mhd_grid_pack(self.h, C.byref(gp), buf, n.value, None)
        if st != OK:
            raise MhdError(f"grid_pack: {self.last_status(st).message}")
        return bytes(buf)

    def divb_sor(self, params):
        sw = C.c_int(0)
        st = self._check(self.lib.mhd_divb_sor(self.h, C.byref(params), C.byref(sw)), "divb_sor")
        return self.last_status(st), sw.value

    def run(self, dt0, steps=0, t_max=0.0, sor=None, nongrid_steps=0, nongrid_t=0.0,
            max_records=1024):
        """The reference main loop on the device (mhd_run): `steps` steps (constant time
        mode) or until t_max.  Returns (RunResult as a dict, list of record dicts)."""
        p = RunParams()
        p.time_mode = 1 if steps > 0 else 2
        p.steps, p.t_max, p.dt0 = int(steps), float(t_max), float(dt0)
        p.sor = sor if sor is not None else sor_params(steps=0)
        p.nongrid_mode = 1 if nongrid_steps > 0 else (2 if nongrid_t > 0.0 else 0)
        p.nongrid_steps, p.nongrid_t = int(nongrid_steps), float(nongrid_t)
        recs = (NongridRecord * max(1, max_records))()
        r = RunResult()
        self._check(self.lib.mhd_run(self.h, C.byref(p), recs, max_records, C.byref(r)), "run")
        res = {f: getattr(r, f) for f, _ in RunResult._fields_}
        out = [dict(step=q.step, t=q.t, dt=q.dt, values=tuple(q.values))
               for q in recs[:min(r.records, max_records)]]
        return res, out

    def divb_clean(self, params):
        m, sw = C.c_double(0), C.c_int(0)
        st = self._check(self.lib.mhd_divb_clean(self.h, C.byref(params), C.byref(m),
                                                 C.byref(sw)), "divb_clean")
        return self.last_status(st), m.value, sw.value

    def set_step_graph(self, enable):
        """steps() as one CUDA graph launch (default on) or one host round trip per step."""
        self._check(self.lib.mhd_set_step_graph(self.h, int(bool(enable))), "set_step_graph")

    def set_step_host_banded(self, enable):
        """step_host: banded host copy overlapping the first operator (default on) or one copy."""
        self._check(self.lib.mhd_set_step_host_banded(self.h, int(bool(enable))),
                    "set_step_host_banded")

    def set_sor_graph(self, enable):
        """SOR sweep loop as one CUDA graph launch (default on) or host-issued passes."""
        self._check(self.lib.mhd_set_sor_graph(self.h, int(bool(enable))), "set_sor_graph")

    def set_sor_fused(self, enable):
        """Two-launch SOR sweeps where the grid allows them (default on)."""
        self._check(self.lib.mhd_set_sor_fused(self.h, int(bool(enable))), "set_sor_fused")

    def set_sor_rows(self, mode):
        """SOR rows per thread step: 0 by grid size, 1 one row (reused loads), 2 two rows."""
        self._check(self.lib.mhd_set_sor_rows(self.h, int(mode)), "set_sor_rows")

    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        self.lib.mhd_stream(self.h, C.byref(s))
        return s.value or 0

    def time_integrate(self, n):
        """Average device ms of `n` back-to-back spatial operators."""
        ms = C.c_double(0.0)
        st = self._check(self.lib.mhd_time_integrate(self.h, n, C.byref(ms)), "time_integrate")
        if st != OK:
            raise MhdError(self.last_status(st).message)
        return ms.value

    def counters(self):
        a, b = C.c_longlong(0), C.c_longlong(0)
        self.lib.mhd_get_counters(self.h, C.byref(a), C.byref(b))
        return {"neg_pressure": a.value, "launches": b.value}


# ---------------------------------------------------------------------------------------
# Reference-shaped interface (host buffers in, host buffers out).

class _SpatialMethod:
    scheme = ENO_ROE
    min_buffer = 2

    def __init__(self, nx, ny, bufferWidth, dx, dy, boundary, gamma, characteristics=True,
                 fast_math=False, device=0):
        if bufferWidth < self.min_buffer:
            raise ValueError("Buffer is too small for this method; need at least "
                             f"{self.min_buffer} extra grids")
        flags = (FLAG_CHARACTERISTICS if characteristics else 0) | (FLAG_FAST_MATH if fast_math else 0)
        self.ctx = Context(nx, ny, dx, dy, gamma, boundary, scheme=self.scheme, time_method=RK3,
                           flags=flags, device=device)
        self.characteristics = characteristics

    def initializeDirichletBoundaries(self, U):
        self.ctx.upload(U)
        self.ctx.init_dirichlet()

    def integrate(self, U, UL, borderFlux=None):
        """SpatialIntegrationMethod::integrate: U gets its ghost cells, UL = L(U)."""
        st, _, d = self.ctx.integrate_host(U, UL)
        return st, d

    def getCharacteristicsX(self, cx, LUx):
        if self.scheme == CENTRAL_FD:
            return False
        a = self.ctx.characteristics()
        cx[...] = a[0]
        LUx[...] = a[2]
        return True

    def getCharacteristicsY(self, cy, LUy):
        if self.scheme == CENTRAL_FD:
            return False
        a = self.ctx.characteristics()
        cy[...] = a[1]
        LUy[...] = a[3]
        return True


class SpatialMethodEnoRoe(_SpatialMethod):
    scheme = ENO_ROE


class SpatialMethodEnoLF(_SpatialMethod):
    scheme = ENO_LF


class SpatialMethodCentralFD2(_SpatialMethod):
    """SpatialMethodCentralFD2 (spatialmethodcentralfd2.cpp): second-order
    central differences; keeps no characteristics."""
    scheme = CENTRAL_FD
    min_buffer = 1


class _TimeMethod:
    time_method = RK3

    def __init__(self, nx, ny, bufferWidth, dtMin, dtMax, cflNumber, method):
        """Takes over the method's device context, like the reference's
        std::move of the method into the stepper (main.cpp:141-151)."""
        self.method = method
        self.ctx = method.ctx
        self.ctx.set_stepper(self.time_method, dtMin, dtMax, cflNumber)

    def step(self, U, cx=None, cy=None, LUx=None, LUy=None, borderFlux=None, dtCurrent=0.0):
        st, dt = self.ctx.step_host(U, dtCurrent)
        if not st.isError and self.method.characteristics:
            a = self.ctx.characteristics()
            for dst, src in ((cx, a[0]), (cy, a[1]), (LUx, a[2]), (LUy, a[3])):
                if dst is not None:
                    dst[...] = src
        return st, dt


class TimeIntegrationRK3(_TimeMethod):
    time_method = RK3


class TimeIntegrationEuler(_TimeMethod):
    time_method = EULER


def divBCalculation(ctx: Context, U):
    """divBCalculation on a host state (periodic B ghosts are filled in U)."""
    ctx.upload(U)
    m, t = ctx.divb_calc()
    U[...] = ctx.download()
    return m, t


def divBCorrectionSOR(ctx: Context, U, params):
    """divBCorrectionSOR on a host state; the context keeps the potential."""
    ctx.upload(U)
    st, sweeps = ctx.divb_sor(params)
    U[...] = ctx.download()
    return st, sweeps


def fp64_peak_tflops(device=0):
    """Measured FP64 FMA throughput of the device (TFLOP/s)."""
    t = C.c_double(0.0)
    st = library().mhd_fp64_peak(device, C.byref(t))
    if st != OK:
        raise MhdError(f"mhd_fp64_peak failed: {STATUS_NAMES.get(st, st)}")
    return t.value
