"""The drop-in program (mhd2d-solver_b200/_build/mhd2d_run): the reference's
INI decks drive the plugin classes through the reference's own reader,
problem setups, conversions and writers, compiled unmodified with the
project-written Boost stand-in headers.

The checker is the reference's own whole program (oracle/_ref/mhd2d, its
unmodified sources).  Each reduced deck (tests/golden/decks, written by
tests/golden/make_decks.py from the reference's example decks) runs in a
directory of its own through both programs, and the output files (grid
dumps, non-grid records, characteristics, binary hint files) are compared:

* --backend=cpu (the reference's classes under the drop-in main loop):
  byte-identical files, on the CPU;
* --backend=cuda --divb=host (the CUDA method and stepper, the reference's
  div B cleaning on the host state): byte-identical files, on the GPU;
* --backend=cuda --divb=device (the cleaning on the GPU too, red-black SOR):
  the same files with the same records; the solutions differ by what the
  two SOR orderings leave behind at the decks' loose sweep tolerance (rmax
  1e-5), so the conserved totals are compared to 1e-5 relative (the
  explosion deck's total momentum, which the B corrections feed through the
  Lorentz force, moves by 1.1e-6) and the cleaned max |div B| must not exceed
  ten times the reference's (or the deck's divbmax target).
"""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECKS = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "decks", "*.ini")))
REF_PROG = os.path.join(ROOT, "oracle", "_ref", "mhd2d")
RUN = os.path.join(ROOT, "mhd2d-solver_b200", "_build", "mhd2d_run")

needs_programs = pytest.mark.skipif(
    not (os.path.exists(REF_PROG) and os.path.exists(RUN)),
    reason="oracle/_ref/mhd2d or mhd2d_run not built (needs the reference checkout)")


def _run(argv, deck, where):
    os.makedirs(where)
    shutil.copy(deck, os.path.join(where, "deck.ini"))
    r = subprocess.run(argv + ["deck.ini"], cwd=where, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, (argv, r.stdout[-2000:], r.stderr[-2000:])
    files = {}
    for name in sorted(os.listdir(where)):
        if name != "deck.ini":
            with open(os.path.join(where, name), "rb") as f:
                files[name] = f.read()
    assert files, "no output files"
    return files, r.stdout


def _reference(deck, tmp_path):
    return _run([REF_PROG], deck, str(tmp_path / "reference"))


def _ngdat(blob):
    rows = [ln.split() for ln in blob.decode().splitlines() if ln and not ln.startswith("#")]
    return np.array([[float(v) for v in r] for r in rows])


@needs_programs
@pytest.mark.parametrize("deck", DECKS, ids=os.path.basename)
def test_cpu_backend_matches_reference_program(deck, tmp_path):
    ref, _ = _reference(deck, tmp_path)
    got, out = _run([RUN, "--backend=cpu"], deck, str(tmp_path / "dropin"))
    assert "Backend            : cpu" in out
    assert list(got) == list(ref)
    for name in ref:
        assert got[name] == ref[name], name


@pytest.mark.gpu
@needs_programs
@pytest.mark.parametrize("deck", DECKS, ids=os.path.basename)
def test_cuda_backend_host_divb_matches_reference_program(deck, tmp_path):
    ref, _ = _reference(deck, tmp_path)
    got, out = _run([RUN, "--backend=cuda", "--divb=host"], deck, str(tmp_path / "dropin"))
    assert "Backend            : cuda" in out
    assert list(got) == list(ref)
    for name in ref:
        assert got[name] == ref[name], name


@pytest.mark.gpu
@needs_programs
@pytest.mark.parametrize("deck", DECKS, ids=os.path.basename)
def test_cuda_backend_device_divb(deck, tmp_path):
    ref, _ = _reference(deck, tmp_path)
    got, out = _run([RUN, "--backend=cuda", "--divb=device"], deck, str(tmp_path / "dropin"))
    assert "div B on the device" in out
    assert list(got) == list(ref)
    ng = [n for n in ref if n.endswith(".ngdat")]
    assert ng
    a, b = _ngdat(got[ng[0]]), _ngdat(ref[ng[0]])
    assert a.shape == b.shape
    assert np.array_equal(a[:, :2], b[:, :2])  # record index and step
    np.testing.assert_allclose(a[:, 2:4], b[:, 2:4], rtol=1e-12)  # t, dt
    np.testing.assert_allclose(a[:, 7:10], b[:, 7:10], rtol=1e-5)  # mass, momentum, energy
    assert np.all(a[:, 5] <= np.maximum(10.0 * b[:, 5], 1e-6) + 1e-12)  # max |div B|
