"""DistGrid with GPU slabs == the serial GPU grid, bit for bit.

The ranks are gloo processes whose slabs are GPU grids on the one visible GPU;
their kernels never wait on one another (the exchange runs on the host between
launches). The halo copies and the step rollback are also checked directly
through the C ABI, with host and with device buffers.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, cuda_ok

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(ROOT, "tests"))
import dist_worker  # noqa: E402
from test_dist import ALL_CASES, run_ranks  # noqa: E402

from dragon_b200 import _lib  # noqa: E402
from dragon_b200 import grid as gr  # noqa: E402
from dragon_b200 import problems  # noqa: E402
from dragon_b200.boundary import Periodic  # noqa: E402


@pytest.fixture(autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("world", [1, 2])
def test_gpu_dist_matches_serial(world, tmp_path):
    got = run_ranks(world, ALL_CASES, tmp_path, slab="gpu")
    for name in ALL_CASES:
        w, B = dist_worker.serial_run(name, backend="gpu")
        np.testing.assert_array_equal(got[name]["w"], w, err_msg=name)
        if B is not None:
            np.testing.assert_array_equal(got[name]["B"], B, err_msg=name)


@pytest.mark.parametrize("world", [2, 3])
def test_gpu_dist_device_fills(world, tmp_path):
    """Device user fills (NVRTC) on the slabs of a distributed grid: each slab
    runs them on the faces of the global box it touches, with its global
    origin in the fill context, and the distributed run equals the serial
    grid's bit for bit (one fill depends on the global x position)."""
    got = run_ranks(world, ["kh2d_device_fills"], tmp_path, slab="gpu")
    w, _ = dist_worker.serial_run("kh2d_device_fills", backend="gpu")
    np.testing.assert_array_equal(got["kh2d_device_fills"]["w"], w)
    assert int(got["kh2d_device_fills"]["retries"]) == 0


def _ot_grid(n=20):
    """A 2D MHD grid (n x n+4, 3 ghosts) holding distinct values everywhere."""
    G = gr.Grid2D(n, n + 4, 1.0 / n, 1.0 / n, ghosts=3, config=gr.Config(mhd=True))
    rng = np.random.default_rng(11)
    G.w[...] = rng.uniform(0.5, 2.0, size=G.w.shape)
    G.B[...] = rng.uniform(-1.0, 1.0, size=G.B.shape)
    return G


@pytest.mark.parametrize("faces", [0, 1])
@pytest.mark.parametrize("corners", [0, 1])
def test_halo_pack_unpack(faces, corners):
    import torch
    G = _ot_grid()
    L, h, g = G._lib, G._h, G.ghosts
    ref = (G.B if faces else G.w).copy()
    first, layers = -2, 4
    cnt = ctypes.c_longlong()
    _lib.check(L.dragon_gpu_halo_size(h, 0, layers, faces, corners, ctypes.byref(cnt)))
    ny = G.n[1] + faces
    ty = slice(0, ny + 2 * g) if corners else slice(g, g + ny)
    blk = np.moveaxis(ref[first + g:first + g + layers, ty], -1, 0).ravel()
    assert cnt.value == blk.size
    G._to_device()
    host = np.zeros(cnt.value)
    _lib.check(L.dragon_gpu_halo_pack(h, 0, first, layers, faces, corners, host.ctypes.data_as(ctypes.c_void_p), 0))
    np.testing.assert_array_equal(host, blk)
    dev = torch.zeros(cnt.value, dtype=torch.float64, device="cuda")
    _lib.check(L.dragon_gpu_halo_pack(h, 0, first, layers, faces, corners, ctypes.c_void_p(dev.data_ptr()), 1))
    np.testing.assert_array_equal(dev.cpu().numpy(), blk)
    # unpack a marked block one layer up, from the device buffer
    dev.mul_(-1.0)
    torch.cuda.synchronize()
    _lib.check(L.dragon_gpu_halo_unpack(h, 0, first + 1, layers, faces, corners, ctypes.c_void_p(dev.data_ptr()), 1))
    G._device_ran()
    got = G.B if faces else G.w
    want = ref.copy()
    want[first + 1 + g:first + 1 + g + layers, ty] = -np.moveaxis(blk.reshape((ref.shape[-1], layers, -1)), 0, -1)
    np.testing.assert_array_equal(got, want)


def test_halo_rejects_out_of_range():
    G = _ot_grid()
    buf = np.zeros(1 << 16)
    p = buf.ctypes.data_as(ctypes.c_void_p)
    assert G._lib.dragon_gpu_halo_pack(G._h, 0, -4, 2, 0, 1, p, 0) == 1       # below the ghosts
    assert G._lib.dragon_gpu_halo_pack(G._h, 0, G.n[0] + 2, 2, 0, 1, p, 0) == 1  # past them
    assert G._lib.dragon_gpu_halo_pack(G._h, 2, 0, 1, 0, 1, p, 0) == 1       # no third axis
    H = gr.Grid2D(16, 16, 1 / 16, 1 / 16, ghosts=2)
    assert H._lib.dragon_gpu_halo_pack(H._h, 0, 0, 1, 1, 1, p, 0) == 1       # no face B


def test_step_rollback_restores_state():
    w, dx, dy = problems.kelvin_helmholtz_2d(32, ghosts=2, seed=3)
    G = gr.Grid2D(32, 32, dx, dy, ghosts=2, config=gr.Config(riemann=gr.RIEMANN_HLLC))
    G.w[...] = w
    G.boundary = Periodic()
    G.apply_boundary()
    before = G.w.copy()
    G.unsplit_step(G.cfl_time())
    assert not np.array_equal(G.w, before)
    _lib.check(G._lib.dragon_gpu_step_rollback(G._h))
    G._device_ran()
    np.testing.assert_array_equal(G.w, before)
    # only the last committed step can be undone, once
    assert G._lib.dragon_gpu_step_rollback(G._h) == 1
