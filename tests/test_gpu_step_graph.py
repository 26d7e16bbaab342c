"""mhd_steps as one CUDA graph launch (a while node over the steps, the RK3
retry loop as a nested while node driven by the device-side controller)
against the step-by-step host loop and the reference's golden runs."""
import os
import time

import numpy as np
import pytest

import mhd2d_b200 as M
from mhd2d_b200 import problems as P
from gpu_helpers import make_ctx, same

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _problem(d):
    return P.Problem(d["U_in"].copy(), float(d["dx"]), float(d["dy"]),
                     float(d.get("gamma", 5.0 / 3.0)), tuple(int(b) for b in d["bc"]))


def _steps(p, graph, n, dt0, flags=0, **kw):
    ctx = make_ctx(p, flags=flags, **kw)
    ctx.set_step_graph(graph)
    st, dt, dts = ctx.steps(n, dt0, record=True)
    U = ctx.download()
    chars = ctx.characteristics() if flags & M.FLAG_CHARACTERISTICS else None
    ctx.close()
    return st, dt, dts, U, chars


@pytest.mark.parametrize("name", ["run_ot_roe", "run_ot_lf", "run_explosion_retry",
                                  "run_blocky_euler", "run_blocky_const"])
def test_graph_steps_match_golden_and_host_loop(name):
    """Fixed-count golden runs (RK3 with dt changes and retries, Euler,
    constant dt): the graph loop ends bit-identical to the reference's run
    and to the host loop, with the same dt of every step."""
    d = np.load(os.path.join(GOLD, name + ".npz"))
    p = _problem(d)
    n = int(d["nsteps"])
    kw = dict(scheme=int(d["scheme"]), time_method=int(d["time_method"]),
              dt_min=float(d["dt_min"]), dt_max=float(d["dt_max"]), cfl=float(d["cfl"]))
    g = _steps(p, True, n, float(d["dt0"]), **kw)
    h = _steps(p, False, n, float(d["dt0"]), **kw)
    assert g[0].status == h[0].status == int(d["status"])
    assert g[1] == h[1] == float(d["dt"])
    assert same(g[2], h[2]) and same(g[2], d["dt_hist"][:n])
    assert same(g[3], h[3]) and same(g[3], d["U_out"])


def test_graph_steps_stop_at_a_failing_step_like_the_host_loop():
    d = np.load(os.path.join(GOLD, "integrate_negdensity_2.npz"))
    p = _problem(d)
    g = _steps(p, True, 3, 0.01)
    h = _steps(p, False, 3, 0.01)
    assert g[0].status == h[0].status == M.ERR_NEGATIVE_DENSITY and g[0].isError
    assert g[1] == h[1] == 0.01
    assert same(g[3], h[3])


def test_graph_steps_keep_characteristics():
    p = P.random_smooth(40, 36, seed=5, bc=(M.PERIODIC, M.PERIODIC, M.NEUMANN, M.OPEN))
    g = _steps(p, True, 4, 1e-3, flags=M.FLAG_CHARACTERISTICS, dt_max=0.01)
    h = _steps(p, False, 4, 1e-3, flags=M.FLAG_CHARACTERISTICS, dt_max=0.01)
    assert same(g[3], h[3]) and same(g[2], h[2])
    for a, b in zip(g[4], h[4]):
        assert same(a, b)


def test_graph_steps_brio_wu_full_and_time():
    """Config 1 (Brio-Wu 256 x 8, 410 steps): the graph loop and the host
    loop give the same state; the graph loop waits on the host once."""
    d = np.load(os.path.join(GOLD, "run_briowu_full_roe.npz"))
    p = _problem(d)
    n = int(d["steps"])
    kw = dict(scheme=int(d["scheme"]), dt_min=float(d["dt_min"]), dt_max=float(d["dt_max"]),
              cfl=float(d["cfl"]))
    out = {}
    for graph in (True, False):
        ctx = make_ctx(p, flags=0, **kw)
        ctx.set_step_graph(graph)
        ctx.steps(2, float(d["dt0"]))  # warm-up (graph capture)
        ctx.upload(p.U)
        t0 = time.perf_counter()
        st, dt, dts = ctx.steps(n, float(d["dt0"]), record=True)
        out[graph] = (time.perf_counter() - t0, ctx.download(), dts, st.status)
        ctx.close()
    assert out[True][3] == out[False][3] == M.OK
    assert same(out[True][1], out[False][1]) and same(out[True][1], d["U_out"])
    assert same(out[True][2], out[False][2])
    print(f"Brio-Wu 256x8, {n} steps: graph {out[True][0] * 1e3:.1f} ms, "
          f"host loop {out[False][0] * 1e3:.1f} ms")
