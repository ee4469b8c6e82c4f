"""The reference-side binding: DRAGON's own Grid2D / Grid3D, compiled from
the reference sources, with unsplit_step overridden by the C ABI
(tests/refside/gpugrid.hpp, the binding INTEGRATION.md shows), driven by the
reference's own Grid::advance (CFL.cpp:151-213: its BoundaryList, its CFL
time, its catch-and-halve retry) and compared bit for bit with the plain
reference grid on the same initial state.

The binaries are built in the container that holds the reference sources
(tests/refside/Makefile, run by the build entry point) and travel prebuilt.
"""
import os
import subprocess

import pytest

from conftest import ROOT, cuda_ok

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tests", "refside", "_build")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def run(binary, case):
    exe = os.path.join(BUILD, binary)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference sources: make -C tests/refside)")
    p = subprocess.run([exe, case], capture_output=True, text=True, timeout=600)
    line = [x for x in p.stdout.splitlines() if x.startswith(case + " ")]
    assert line, p.stdout + p.stderr
    fields = dict(kv.split("=") for kv in line[-1].split()[2:])
    return p.returncode, line[-1], {k: int(v) for k, v in fields.items()}


@pytest.mark.parametrize("case", ["kh2d", "walls2d", "blast3d"])
def test_reference_advance_through_binding_hydro(case):
    rc, line, f = run("refside_hydro", case)
    assert rc == 0 and " bitwise " in line, line
    assert f["calls"] > 3 and f["failures"] == 0, line


def test_reference_retry_through_binding():
    """Fixed dt without a CFL limit: device steps fail, the binding throws,
    and the reference's advance halves dt and retries until it succeeds."""
    rc, line, f = run("refside_hydro", "retry2d")
    assert rc == 0 and " bitwise " in line, line
    assert f["failures"] > 0 and f["calls"] > f["failures"], line


@pytest.mark.parametrize("case", ["ot2d", "blast3d_mhd"])
def test_reference_advance_through_binding_mhd(case):
    rc, line, f = run("refside_mhd", case)
    assert rc == 0 and " bitwise " in line, line
    assert f["calls"] > 3 and f["failures"] == 0, line
