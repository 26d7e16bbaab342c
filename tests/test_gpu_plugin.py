"""Drop-in check through the reference's own C++ interfaces.

mhd2d-solver_b200/_build/plugin_check (built from the plugin subclasses, the
reference's hot-path objects and libmhd2d_b200.so) runs the same problem
three ways - the reference stepper with the reference method, the reference
stepper with CudaSpatialMethodEnoRoe/EnoLF, and CudaTimeIntegrationRK3 with
the Cuda method - and exits non-zero unless all three agree bit for bit
(state, characteristic outputs and the final dt)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "mhd2d-solver_b200", "_build", "plugin_check")


@pytest.mark.skipif(not os.path.exists(EXE), reason="plugin_check not built (needs the reference headers)")
@pytest.mark.parametrize("scheme", [2, 3])
@pytest.mark.parametrize("problem,steps", [("ot", 6), ("bw", 12), ("dir", 5)])
def test_plugin_subclasses_match_reference(scheme, problem, steps):
    r = subprocess.run([EXE, str(scheme), problem, str(steps)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
