"""Generates the golden fixtures in tests/golden/ from the DRAGON reference
itself (oracle/_ref: the reference's own sources compiled as a library,
driven through its Grid / Boundary / CFL API). Needs the reference sources in
this container; the fixtures it writes are committed so that the checks run
anywhere.

One fixture per configuration family of the hot path, each small enough for
the CPU oracle to reproduce in seconds:
  sod_1d_512        1D two-state problem, 512 cells, HLLC, minmod, Outflow,
                    CFL 0.3, advance to t = 0.2
  kh_2d_32          2D shear layer 32^2, HLLC, van Leer, CTU, periodic,
                    advance to t = 0.05
  ot_2d_24          2D MHD Orszag-Tang 24^2, HLLD, MC, CTU + CT, BETA_GATED,
                    periodic, advance to t = 0.02
  blast_3d_10       3D blast 10^3 (p 10 inside r < 0.1), exact solver, MC,
                    Outflow, three CFL steps
  kh_split_2d_32    the 2D shear layer through advance_split (Strang), t = 0.05
  blast_split_3d_12 3D blast 12^3, HLLC, van Leer, Reflective, advance_split
                    to t = 0.01 (all six sweep orders)

Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dragon_b200 import boundary, problems  # noqa: E402
from oracle import refgrid  # noqa: E402
from oracle.refgrid import bc_entries_from  # noqa: E402

RIEMANN_EXACT, RIEMANN_HLLC, RIEMANN_HLLX = 0, 2, 5
LIM_MINMOD, LIM_MC, LIM_VANLEER = 0, 1, 2


def sod():
    w0, dx = problems.sod_1d(512, ghosts=2)
    R = refgrid.RefGrid(dim=1, n=(512,), d=(dx,), ghosts=2, riemann=RIEMANN_HLLC, limiter=LIM_MINMOD)
    R.set_prim(w0)
    R.advance(0.2)
    return {"w0": w0, "w": R.get_prim(), "dx": dx, "t": 0.2}


def kh():
    w0, dx, dy = problems.kelvin_helmholtz_2d(32, ghosts=2, seed=1234)
    R = refgrid.RefGrid(dim=2, n=(32, 32), d=(dx, dy), ghosts=2, riemann=RIEMANN_HLLC, limiter=LIM_VANLEER)
    R.set_prim(w0)
    R.set_boundary(bc_entries_from(boundary.as_list(boundary.Periodic())))
    R.advance(0.05)
    return {"w0": w0, "w": R.get_prim(), "dx": dx, "dy": dy, "t": 0.05}


def ot():
    w0, B0, dx, dy = problems.orszag_tang_2d(24, ghosts=3)
    R = refgrid.RefGrid(dim=2, n=(24, 24), d=(dx, dy), ghosts=3, mhd=True, riemann=RIEMANN_HLLX, limiter=LIM_MC)
    R.set_prim(w0)
    R.set_faceB(B0)
    R.set_boundary(bc_entries_from(boundary.as_list(boundary.Periodic())))
    R.initialize_B_fields()
    w_init, B_init = R.get_prim(), R.get_faceB()
    R.advance(0.02)
    return {"w0": w0, "B0": B0, "w_init": w_init, "B_init": B_init, "w": R.get_prim(), "B": R.get_faceB(),
            "dx": dx, "dy": dy, "t": 0.02}


def blast():
    w0, d = problems.blast_3d(10, ghosts=2, p_in=10.0)
    R = refgrid.RefGrid(dim=3, n=(10, 10, 10), d=(d, d, d), ghosts=2, riemann=RIEMANN_EXACT, limiter=LIM_MC)
    R.set_prim(w0)
    dts = [R.step_cfl() for _ in range(3)]
    return {"w0": w0, "w": R.get_prim(), "d": d, "dts": np.array(dts)}


def kh_split():
    w0, dx, dy = problems.kelvin_helmholtz_2d(32, ghosts=2, seed=77)
    R = refgrid.RefGrid(dim=2, n=(32, 32), d=(dx, dy), ghosts=2, riemann=RIEMANN_HLLC, limiter=LIM_VANLEER)
    R.set_prim(w0)
    R.set_boundary(bc_entries_from(boundary.as_list(boundary.Periodic())))
    R.advance_split(0.05)
    return {"w0": w0, "w": R.get_prim(), "dx": dx, "dy": dy, "t": 0.05}


def blast_split():
    w0, d = problems.blast_3d(12, ghosts=2, p_in=10.0)
    R = refgrid.RefGrid(dim=3, n=(12, 12, 12), d=(d, d, d), ghosts=2, riemann=RIEMANN_HLLC, limiter=LIM_VANLEER)
    R.set_prim(w0)
    R.set_boundary(bc_entries_from(boundary.as_list(boundary.Reflective())))
    R.advance_split(0.01)
    return {"w0": w0, "w": R.get_prim(), "d": d, "t": 0.01}


def main():
    for name, fn in (("sod_1d_512", sod), ("kh_2d_32", kh), ("ot_2d_24", ot), ("blast_3d_10", blast),
                     ("kh_split_2d_32", kh_split), ("blast_split_3d_12", blast_split)):
        out = fn()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
