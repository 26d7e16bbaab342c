"""Non-grid output record (outputNonGridData, file_access.cpp:1680-1736): the
reference harness (the reference's own toNaturalData and divBCalculation)
against a numpy restatement of the record's sums, on the CPU."""
import numpy as np
import pytest

from mhd2d_b200 import problems as P
from pyoracle import Reference, reference_available

needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed,bc", [(1, (1, 1, 1, 1)), (2, (3, 3, 4, 4)), (3, (2, 1, 3, 1))])
def test_reference_record_matches_numpy_sums(seed, bc):
    p = P.random_smooth(23, 17, seed=seed, bc=bc)
    U = p.U.copy()
    out = Reference().nongrid_data(U, p.dx, p.dy, p.gamma, bc)
    I = p.U[:, 2:-2, 2:-2]
    rho, m, B, E = I[0], I[1:4], I[4:7], I[7]
    u = m / rho
    uu = (u * u).sum(0)
    pres = (p.gamma - 1.0) * (E - 0.5 * (m * m).sum(0) / rho - 0.5 * (B * B).sum(0))
    dxdy = p.dx * p.dy
    want = [np.sqrt(uu.max()), None, None, rho.sum() * dxdy, (rho * np.sqrt(uu)).sum() * dxdy,
            E.sum() * dxdy, np.log(pres * rho ** -p.gamma).sum() * dxdy]
    for k in (0, 3, 4, 5, 6):
        assert abs(out[k] - want[k]) <= 1e-12 * abs(want[k]), (k, out[k], want[k])
    assert out[1] >= 0.0 and out[2] >= 0.0
