"""The C++ DistGrid (include/dragon/dist.hpp, libdragon_dist*.so).

tests/host_cpp/dist_test.cpp runs a DistGrid with P ranks as threads of one
process, each holding its slab on the visible GPU and exchanging halos through
host memory (their kernels never wait on one another), and checks the gathered
arrays against the serial grid bit for bit. A one-rank NCCL communicator runs
the NCCL transport (the periodic wrap of a single slab and the all-reduces).
The program is compiled on the CPU side too, so the library links there.
"""
import os
import subprocess

import pytest

from conftest import ROOT, cuda_ok

from dragon_b200 import build as dbuild

SRC = os.path.join(ROOT, "tests", "host_cpp", "dist_test.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def dist_test(tmp_path_factory):
    dbuild.build()
    out = tmp_path_factory.mktemp("dist_cpp")
    exes = {}
    libdir = os.path.join(ROOT, "dragon_b200")
    for mhd in (False, True):
        sfx = "_mhd" if mhd else ""
        exe = str(out / f"dist_test{sfx}")
        cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", *(["-DMHD"] if mhd else []),
               "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"), SRC, "-L" + libdir,
               f"-ldragon_dist{sfx}", f"-ldragon_host{sfx}", "-ldragon_gpu", "-L" + os.path.join(CUDA, "lib64"),
               "-lcudart", "-lnccl", "-lpthread", "-Wl,-rpath," + libdir, "-Wl,-rpath," + os.path.join(CUDA, "lib64"),
               "-o", exe]
        subprocess.run(cmd, check=True)
        exes[mhd] = exe
    return exes


def test_cpp_dist_builds_and_links(dist_test):
    for exe in dist_test.values():
        r = subprocess.run(["ldd", exe], capture_output=True, text=True)
        assert "libdragon_dist" in r.stdout and "not found" not in r.stdout, r.stdout


def _run(exe, *args):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)
    last = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else ""
    assert r.returncode == 0 and last.startswith("ok"), r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["kh", "walls", "blast3d", "fills"])
@pytest.mark.parametrize("ranks", [1, 2, 3])
def test_cpp_dist_threads_match_serial(dist_test, case, ranks):
    """P slabs against the serial grid, bit for bit; "fills" carries device
    user fills (NVRTC), one of them depending on the global x position."""
    if not cuda_ok():
        pytest.fail("CUDA device required")
    _run(dist_test[False], "threads", str(ranks), case)


@pytest.mark.gpu
@pytest.mark.parametrize("ranks", [1, 2, 3])
def test_cpp_dist_mhd_threads_match_serial(dist_test, ranks):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    _run(dist_test[True], "threads", str(ranks), "ot")


@pytest.mark.gpu
def test_cpp_dist_nccl_single_rank(dist_test):
    if not cuda_ok():
        pytest.fail("CUDA device required")
    _run(dist_test[False], "nccl1", "kh")
    _run(dist_test[True], "nccl1", "ot")
