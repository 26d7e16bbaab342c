"""Device problem generators of the reference's shock tube and plasma sheet
(MHD_PROBLEM_SHOCK_TUBE, MHD_PROBLEM_SHEET_LOBES) against the reference's own
INI reader and setups (oracle/_ref/ref_setup: inputData compiled unmodified),
bit for bit on the interior cells.

The decks are the reduced example decks (tests/golden/decks) and variants of
them written here: an oblique shock-tube interface, and plasma sheets with
the tanh profile, wider linear transitions, the jump transition and an
elliptic sheet front (head != foot)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from mhd2d_b200 import batch as B
from ini_decks import problem_of
from gpu_helpers import same

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_SETUP = os.path.join(ROOT, "oracle", "_ref", "ref_setup")
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_decks import rewrite  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(REF_SETUP),
                                                  reason="oracle/_ref/ref_setup not built")]

DECKS = os.path.join(HERE, "golden", "decks")
VARIANTS = {
    "bw_plain": ("bw_lf.ini", {}),
    "bw_oblique": ("bw_lf.ini", {("problem", "Nx"): "40", ("problem", "Ny"): "24",
                                 ("problem", "interface angle"): "30"}),
    "bw_steep": ("bw_lf.ini", {("problem", "Nx"): "24", ("problem", "Ny"): "40",
                               ("problem", "interface angle"): "-65"}),
    "sheet_plain": ("sheet_lf.ini", {}),
    "sheet_tanh_wide": ("sheet_lf.ini", {("problem", "Nx"): "96", ("problem", "Ny"): "24",
                                         ("problem", "sheet profile"): "tanh",
                                         ("problem", "transition points"): "2",
                                         ("problem", "sheet start"): "4.0",
                                         ("problem", "sheet start foot"): "-2.0",
                                         ("problem", "Bx_l"): "0.3",
                                         ("problem", "By_r"): "-0.4"}),
    "sheet_jump": ("sheet_lf.ini", {("problem", "Nx"): "48", ("problem", "Ny"): "24",
                                    ("problem", "transition type"): "jump",
                                    ("problem", "sheet thickness"): "2.5"}),
}


def _reference_state(deck, tmp_path):
    out = tmp_path / "state.bin"
    r = subprocess.run([REF_SETUP, str(deck), str(out)], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    nx, ny = np.frombuffer(raw[:8], dtype=np.int32)
    dx, dy, gamma = np.frombuffer(raw[8:32], dtype=np.float64)
    bc = tuple(int(b) for b in np.frombuffer(raw[32:48], dtype=np.int32))
    U = np.frombuffer(raw[48:], dtype=np.float64).reshape(8, nx + 4, ny + 4)
    return int(nx), int(ny), float(dx), float(dy), float(gamma), bc, U


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_device_setup_matches_reference(name, tmp_path):
    src, changes = VARIANTS[name]
    with open(os.path.join(DECKS, src)) as f:
        text = rewrite(f.read(), changes) if changes else f.read()
    deck = tmp_path / "deck.ini"
    deck.write_text(text)
    nx, ny, dx, dy, gamma, bc, U_ref = _reference_state(deck, tmp_path)
    kind, params, pnx, pny, pdx, pdy, pgamma, pbc = problem_of(str(deck))
    assert (pnx, pny, pdx, pdy, pgamma, pbc) == (nx, ny, dx, dy, gamma, bc)
    run = B.Run(nx, ny, dx, dy, gamma, bc, dt_max=0.01, t_end=1.0)
    with B.Batch([run]) as b:
        if kind == "shock tube":
            b.init_shock_tube(0, *params[:3], params[3:11], params[11:19])
        else:
            b.init_sheet_lobes(0, *params[:10], params[10:18], params[18:26], params[26:34],
                               params[34:42])
        U = b.download(0)
    assert same(U[:, 2:-2, 2:-2], U_ref[:, 2:-2, 2:-2])
