"""C ABI checks that need no GPU: the library loads, exports every entry
point include/mhd2d_b200.h declares, and rejects bad parameters before it
touches the device (the reference's constructor errors)."""
import ctypes as C
import os
import re

import pytest

import mhd2d_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mhd2d_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*int\s+(mhd_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("mhd_ctx_create", "mhd_integrate", "mhd_step", "mhd_divb_sor", "mhd_divb_calc",
              "mhd_get_characteristics", "mhd_upload", "mhd_download"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = M.library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    lib = M.library()
    for s in declared_symbols():
        assert getattr(lib, s).argtypes is not None, f"{s} has no ctypes signature"


@pytest.mark.parametrize("kw,val", [("halo", 1), ("nx", 1), ("scheme", 0), ("scheme", 4),
                                    ("time_method", 3), ("bc", (1, 1, 0, 1)), ("bc", (5, 1, 1, 1)),
                                    ("dx", 0.0), ("dy", -1.0)])
def test_ctx_create_rejects_bad_parameters(kw, val):
    args = dict(nx=8, ny=8, halo=2, dx=0.1, dy=0.1, gamma=1.4, bc=(1, 1, 1, 1), scheme=2,
                time_method=2, dt_min=0.0, dt_max=1.0, cfl=0.4, flags=0, device=0)
    args[kw] = val
    lib = M.library()
    h = C.c_void_p()
    bc = (C.c_int * 4)(*args["bc"])
    st = lib.mhd_ctx_create(args["nx"], args["ny"], args["halo"], args["dx"], args["dy"],
                            args["gamma"], bc, args["scheme"], args["time_method"],
                            args["dt_min"], args["dt_max"], args["cfl"], args["flags"],
                            args["device"], C.byref(h))
    assert st == M.ERR_WRONG_PARAMETER
    assert not h.value


def test_null_context_is_rejected():
    lib = M.library()
    d = C.c_double(0.0)
    assert lib.mhd_integrate(None, C.byref(d)) == M.ERR_WRONG_PARAMETER
    assert lib.mhd_step(None, C.byref(d)) == M.ERR_WRONG_PARAMETER
    assert lib.mhd_ctx_destroy(None) == M.OK


def test_status_codes_match_reference_enum():
    # enums.hpp: ReturnStatus order
    names = ["OK", "NoChange", "Updated", "ErrorNotImplemented", "ErrorTimeUnderflow",
             "ErrorNotConverged", "ErrorNegativeDensity", "ErrorNegativePressure",
             "ErrorFileNotFound", "ErrorFailedToParse", "ErrorWrongParameter"]
    for code, name in enumerate(names):
        assert M.STATUS_NAMES[code] == name
