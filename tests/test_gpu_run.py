"""mhd_run: the reference main loop (main.cpp:174-344) as one native call on
the device, against the golden main-loop runs of the reference, against the
same loop driven step by step from Python (gpu_run), and its non-grid output
records against mhd_nongrid_data at the same steps."""
import os

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from gpu_helpers import gpu_run, interior, make_ctx, same

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gold(prefix):
    return sorted(os.path.join(GOLD, f) for f in os.listdir(GOLD)
                  if f.startswith(prefix) and f.endswith(".npz"))


def _problem(d):
    return P.Problem(d["U_in"].copy(), float(d["dx"]), float(d["dy"]), float(d["gamma"]),
                     tuple(int(b) for b in d["bc"]))


@pytest.mark.parametrize("path", _gold("run_"), ids=os.path.basename)
def test_run_matches_golden_and_stepwise_loop(path):
    d = np.load(path)
    p = _problem(d)
    sp = None
    if d["sor"].size:
        v = d["sor"]
        sp = M.SorParams(int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), int(v[5]),
                         float(v[6]))
    kw = dict(scheme=int(d["scheme"]), time_method=int(d["time_method"]),
              dt_min=float(d["dt_min"]), dt_max=float(d["dt_max"]), cfl=float(d["cfl"]), flags=0)
    nsteps, t_max = int(d["nsteps"]), float(d["t_max"])
    a = make_ctx(p, **kw)
    res, recs = a.run(float(d["dt0"]), steps=nsteps, t_max=t_max, sor=sp)
    assert res["records"] == 0 and recs == []
    b = make_ctx(p, **kw)
    r = gpu_run(b, float(d["dt0"]), nsteps=nsteps, t_max=t_max, sor=sp)
    assert res["status"] == int(d["status"]) == r["status"]
    assert res["steps"] == int(d["steps"]) == r["steps"]
    assert (res["t"], res["dt"]) == (r["t"], r["dt"])
    U = a.download()
    assert same(U, b.download())
    if sp is None:
        assert same(U, d["U_out"])
    # with non-grid records (step 0 and every 2nd step): the record's div B pass fills
    # periodic B ghosts, as the reference's outputNonGridData does, and nothing else changes
    c = make_ctx(p, **kw)
    res2, recs = c.run(float(d["dt0"]), steps=nsteps, t_max=t_max, sor=sp, nongrid_steps=2)
    assert (res2["status"], res2["steps"], res2["t"], res2["dt"]) == \
        (res["status"], res["steps"], res["t"], res["dt"])
    assert same(interior(c.download()), interior(U))
    assert res2["records"] == 1 + res2["steps"] // 2
    assert [q["step"] for q in recs] == list(range(0, res2["steps"] + 1, 2))
    e = make_ctx(p, **kw)
    assert recs[0]["values"] == e.nongrid_data()
    if sp is None and res2["steps"] >= 2:
        e.steps(2, float(d["dt0"]))
        assert recs[1]["values"] == e.nongrid_data()


def test_run_by_time_cadence_and_nan_stop():
    p = P.ot_vortex(64)
    a = make_ctx(p, dt_min=1e-9, dt_max=2.0 ** -5, flags=0)
    res, recs = a.run(2.0 ** -8, t_max=0.3, nongrid_t=0.1)
    assert res["t"] >= 0.3 and not res["nan_stop"]
    ts = [q["t"] for q in recs]
    assert ts[0] == 0.0 and len(recs) == res["records"]
    # one record each time t first reaches a multiple of 0.1 (main.cpp:291-295)
    for k, t in enumerate(ts[1:], start=1):
        assert t >= 0.1 * k - 1e-12
    assert recs[-1]["t"] == res["t"]
    # the blocky ENO-LF Neumann case that runs into NaNs stops like the step loop
    q = P.random_blocky(20, 30, seed=5, bc=(M.NEUMANN,) * 4)
    kw = dict(scheme=M.ENO_LF, dt_min=1e-9, dt_max=0.01, cfl=0.4, flags=0)
    a = make_ctx(q, **kw)
    res, _ = a.run(1e-3, t_max=0.02)
    b = make_ctx(q, **kw)
    r = gpu_run(b, 1e-3, t_max=0.02)
    assert res["nan_stop"] == 1
    assert (res["steps"], res["t"], res["dt"]) == (r["steps"], r["t"], r["dt"])
    assert same(interior(a.download()), interior(b.download()))
