"""The GPU path against the golden fixtures the reference itself produced
(tests/golden/make_golden.py): bit for bit where no pow is involved; the
exact solver (CUDA pow) within 1e-12 relative L1 with the same dt sequence to
1e-12."""
import os

import numpy as np
import pytest

from conftest import ROOT, cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import problems  # noqa: E402

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def test_sod_1d_512():
    g = load("sod_1d_512")
    G = dg.Grid1D(512, float(g["dx"]), ghosts=2, config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MINMOD))
    G.w[...] = g["w0"]
    G.advance(float(g["t"]))
    np.testing.assert_array_equal(G.w, g["w"])


def test_kh_2d_32():
    g = load("kh_2d_32")
    G = dg.Grid2D(32, 32, float(g["dx"]), float(g["dy"]), ghosts=2,
                  config=dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER))
    G.w[...] = g["w0"]
    G.boundary = dg.Periodic()
    G.advance(float(g["t"]))
    np.testing.assert_array_equal(G.w, g["w"])


def test_ot_2d_24():
    g = load("ot_2d_24")
    G = dg.Grid2D(24, 24, float(g["dx"]), float(g["dy"]), ghosts=3,
                  config=dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, limiter=dg.LIMITER_MC))
    G.w[...] = g["w0"]
    G.B[...] = g["B0"]
    G.boundary = dg.Periodic()
    G.initialize_B_fields()
    np.testing.assert_array_equal(G.w, g["w_init"])
    np.testing.assert_array_equal(G.B, g["B_init"])
    G.advance(float(g["t"]))
    np.testing.assert_array_equal(G.w, g["w"])
    np.testing.assert_array_equal(G.B, g["B"])


def test_blast_3d_10():
    g = load("blast_3d_10")
    d = float(g["d"])
    G = dg.Grid3D(10, 10, 10, d, d, d, ghosts=2, config=dg.Config(riemann=dg.RIEMANN_EXACT, limiter=dg.LIMITER_MC))
    G.w[...] = g["w0"]
    dts = []
    for _ in range(3):  # the reference's step: ghost fill, CFL dt, advance(dt)
        G.apply_boundary()
        dts.append(G.cfl_time())
        G.advance(dts[-1])
    np.testing.assert_allclose(dts, g["dts"], rtol=1e-12)
    l1 = problems.rel_l1(G.w, g["w"])
    assert np.all(l1 <= 1e-12), l1
