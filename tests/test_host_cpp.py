"""The C++23 host API (include/dragon/dragon.hpp, dragon_b200/libdragon_host*.so).

A C++ program written like code against the reference (tests/host_cpp/
host_test.cpp: Grid2D, grid[i, j], grid.boundary = Boundary::Reflective("X") +
Boundary::Periodic("YZ"), a user GhostFill, grid.advance(dt)) runs each case
through the C ABI; its arrays must equal the oracle's bit for bit. The boundary
composition checks need no GPU.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cuda_ok

from dragon_b200 import boundary as bd
from dragon_b200 import build as dbuild
from dragon_b200 import problems

SRC = os.path.join(ROOT, "tests", "host_cpp", "host_test.cpp")


@pytest.fixture(scope="module")
def host_test(tmp_path_factory):
    dbuild.build()
    out = tmp_path_factory.mktemp("host_cpp")
    exes = {}
    for mhd in (False, True):
        exe = str(out / ("host_test_mhd" if mhd else "host_test"))
        lib = "dragon_host_mhd" if mhd else "dragon_host"
        libdir = os.path.join(ROOT, "dragon_b200")
        cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", *(["-DMHD"] if mhd else []),
               "-I" + os.path.join(ROOT, "include"), SRC, "-L" + libdir, "-l" + lib, "-ldragon_gpu",
               "-Wl,-rpath," + libdir, "-o", exe]
        subprocess.run(cmd, check=True)
        exes[mhd] = exe
    return exes, out


def test_cpp_boundary_composition(host_test):
    exes, _ = host_test
    for exe in exes.values():
        r = subprocess.run([exe, "boundary"], capture_output=True, text=True)
        assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_host_libraries_link_the_c_abi():
    """Both host builds exist and resolve against libdragon_gpu.so."""
    dbuild.build()
    for name in ("libdragon_host.so", "libdragon_host_mhd.so"):
        path = os.path.join(ROOT, "dragon_b200", name)
        r = subprocess.run(["ldd", path], capture_output=True, text=True)
        assert "libdragon_gpu.so" in r.stdout and "not found" not in r.stdout, r.stdout


def oracle(dim, n, d, ghosts, mhd=False, **kw):
    from oracle import port, refgrid
    if refgrid.available("mhd" if mhd else "hydro"):
        return refgrid.RefGrid(dim, n, d, ghosts=ghosts, mhd=mhd, **kw)
    return port.PortGrid(dim, n, d, ghosts=ghosts, mhd=mhd, **kw)


def run_cpp(host_test, case, arrays, mhd=False):
    exes, out = host_test
    np.concatenate([a.ravel() for a in arrays]).astype(np.float64).tofile(str(out / f"{case}.in.bin"))
    r = subprocess.run([exes[mhd], "run", case, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.fromfile(str(out / f"{case}.out.bin"), dtype=np.float64), r.stdout


@pytest.mark.gpu
def test_cpp_sod_1d_to_t02(host_test):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    w0, dx = problems.sod_1d(512, ghosts=2)
    got, stdout = run_cpp(host_test, "sod1d", [w0])
    R = oracle(1, (512,), (dx,), 2, riemann=2, limiter=0)
    R.set_prim(w0)
    res = R.advance(0.2)
    np.testing.assert_array_equal(got.reshape(w0.shape), R.get_prim())
    steps = res[0] if isinstance(res, tuple) else None
    if steps is not None:
        assert f"steps {steps} " in stdout, stdout


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh2d", "kh2d_walls", "kh2d_inflow", "kh2d_device_inflow"])
def test_cpp_kh_2d(host_test, case):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    w0, dx, dy = problems.kelvin_helmholtz_2d(64, ghosts=2, seed=21, ny=48)
    w0 = np.pad(w0[2:-2, 2:-2], [(2, 2), (2, 2), (0, 0)], mode="edge")
    got, _ = run_cpp(host_test, case, [w0])
    R = oracle(2, (64, 48), (dx, dy), 2, riemann=2, limiter=2)
    R.set_prim(w0)
    if case == "kh2d":
        R.set_boundary([(bd.PERIODIC, 63, 1, None)])
        for _ in range(5):
            R.step_cfl()
    elif case == "kh2d_walls":
        R.set_boundary([(bd.REFLECTIVE, bd.X, 1, None), (bd.PERIODIC, bd.Y | bd.Z, 1, None)])
        R.advance(0.02)
    else:
        jet = [3.0, 2.5, 0.8, 0.0, 0.0]
        R.set_boundary([(bd.PERIODIC, bd.Y, 1, None), (bd.FIXED, bd.X_negative, 1, jet)])
        R.advance(0.02)
    np.testing.assert_array_equal(got.reshape(w0.shape), R.get_prim())


@pytest.mark.gpu
def test_cpp_orszag_tang_mhd(host_test):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    n, g = 32, 3
    w0, B0, dx, dy = problems.orszag_tang_2d(n, ghosts=g)
    got, _ = run_cpp(host_test, "ot2d", [w0, B0], mhd=True)
    R = oracle(2, (n, n), (dx, dy), g, mhd=True, riemann=5)
    R.set_prim(w0)
    R.set_faceB(B0)
    R.set_boundary([(bd.PERIODIC, 63, 1, None)])
    R.initialize_B_fields()
    for _ in range(5):
        R.step_cfl()
    nw = w0.size
    np.testing.assert_array_equal(got[:nw].reshape(w0.shape), R.get_prim())
    np.testing.assert_array_equal(got[nw:].reshape(B0.shape), R.get_faceB())


@pytest.mark.gpu
def test_cpp_hoard_restart(host_test):
    """DRAGONHOARD from C++ (include/dragon/hoard.hpp): frames written through
    writeToFileAsync / writeToFile, the newest found by restartFileName, a
    fresh grid restarted from it: t, cycle and spacing come back, and three
    more steps on both grids end bit for bit in the same state."""
    rng = np.random.default_rng(21)
    w0 = np.zeros((68, 52, 5))
    w0[..., 0] = rng.uniform(0.5, 2.0, w0.shape[:2])
    w0[..., 1] = rng.uniform(1.0, 2.0, w0.shape[:2])
    w0[..., 2:4] = rng.uniform(-0.3, 0.3, w0.shape[:2] + (2,))
    got, stdout = run_cpp(host_test, "hoard2d", [w0])
    assert "frame_00003.h5 t 0.5 cycle 3 dx 0.015625 dy 0.020833333333333332" in stdout
    half = got.size // 2
    np.testing.assert_array_equal(got[half:], got[:half])
    assert np.all(np.isfinite(got))


@pytest.mark.gpu
def test_cpp_blast_3d(host_test):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    n = 16
    w0, d = problems.blast_3d(n, ghosts=2, p_in=10.0)
    w0 = np.pad(w0[2:-2, 2:-2, 2:-2], [(2, 2)] * 3 + [(0, 0)], mode="edge")
    got, _ = run_cpp(host_test, "blast3d", [w0])
    R = oracle(3, (n, n, n), (1.0 / n,) * 3, 2, riemann=2)
    R.set_prim(w0)
    for _ in range(3):
        R.step_cfl()
    np.testing.assert_array_equal(got.reshape(w0.shape), R.get_prim())
