"""The FLOP-per-cell constants bench.py uses for the roofline are the
op-counting oracle's numbers (oracle/opcount.cpp, structural zeros
excluded), extrapolated in 1/n from two grid sizes to 4096^2."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_build", "opcount")


def _count(n):
    out = subprocess.run([EXE, str(n)], capture_output=True, text=True, check=True, timeout=300)
    return json.loads(out.stdout)


@pytest.mark.skipif(not os.path.exists(EXE), reason="run `make -C oracle opcount`")
def test_bench_flop_constants_match_opcount():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    a, b = _count(128), _count(256)
    for code, name in ((2, "eno_roe"), (3, "eno_lf")):
        for key, table in (("integrate_nonzero", bench.FLOPS_PER_CELL_INTEGRATE),
                           ("step_nonzero", bench.FLOPS_PER_CELL_STEP)):
            f128, f256 = a[name][key], b[name][key]
            slope = (f128 - f256) * 256.0  # f(n) = f_inf + slope / n
            f_inf = f256 - slope / 256.0
            f4096 = f_inf + slope / 4096.0
            assert abs(f4096 - table[code]) < 1.0, (name, key, f4096, table[code])
            assert f4096 < a[name][key.replace("nonzero", "dense")]
