"""The C restatement of the reference (oracle/dragon_oracle.c) reproduces the
golden fixtures that the reference itself produced (tests/golden/make_golden.py)
bit for bit: the oracle is pinned even where the reference cannot be built."""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import port

GOLD = os.path.join(ROOT, "tests", "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def test_sod_1d_512():
    g = load("sod_1d_512")
    P = port.PortGrid(dim=1, n=(512,), d=(float(g["dx"]),), ghosts=2, riemann=2, limiter=0)
    P.set_prim(g["w0"])
    P.advance(float(g["t"]))
    np.testing.assert_array_equal(P.get_prim(), g["w"])


def test_kh_2d_32():
    g = load("kh_2d_32")
    P = port.PortGrid(dim=2, n=(32, 32), d=(float(g["dx"]), float(g["dy"])), ghosts=2, riemann=2, limiter=2)
    P.set_prim(g["w0"])
    P.set_boundary([(4, 63, 1, None)])
    P.advance(float(g["t"]))
    np.testing.assert_array_equal(P.get_prim(), g["w"])


def test_ot_2d_24():
    g = load("ot_2d_24")
    P = port.PortGrid(dim=2, n=(24, 24), d=(float(g["dx"]), float(g["dy"])), ghosts=3, mhd=True, riemann=5, limiter=1)
    P.set_prim(g["w0"])
    P.set_faceB(g["B0"])
    P.set_boundary([(4, 63, 1, None)])
    P.initialize_B_fields()
    np.testing.assert_array_equal(P.get_prim(), g["w_init"])
    np.testing.assert_array_equal(P.get_faceB(), g["B_init"])
    P.advance(float(g["t"]))
    np.testing.assert_array_equal(P.get_prim(), g["w"])
    np.testing.assert_array_equal(P.get_faceB(), g["B"])


def test_blast_3d_10():
    g = load("blast_3d_10")
    d = float(g["d"])
    P = port.PortGrid(dim=3, n=(10, 10, 10), d=(d, d, d), ghosts=2, riemann=0, limiter=1)
    P.set_prim(g["w0"])
    dts = [P.step_cfl() for _ in range(3)]
    np.testing.assert_array_equal(np.array(dts), g["dts"])
    np.testing.assert_array_equal(P.get_prim(), g["w"])
