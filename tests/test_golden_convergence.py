"""The C restatement of the reference (oracle/dragon_oracle.c) reproduces the
reference's own accuracy-study norms at small sizes
(tests/golden/convergence.json, made by tests/golden/make_convergence.py):
the diagonal density wave (Examples/Diagonal) and the field loop
(Examples/LoopAdvection), run through the examples' main loop
(DRAGON/main/main.cpp:124-150)."""
import json
import os

import pytest

from conftest import ROOT
from dragon_b200 import boundary, problems
from oracle import port
from oracle.refgrid import bc_entries_from

with open(os.path.join(ROOT, "tests", "golden", "convergence.json")) as _f:
    GOLD = json.load(_f)

LIMITERS = {"minmod": 0, "mc": 1, "superbee": 3}
TOL = 1e-12


def main_loop(P, dt, final_time):
    t = 0.0
    while t < final_time:
        P.advance(dt)
        t += dt
    return t


def check(norms, ref):
    for v, r in zip(norms, ref):
        assert abs(v - r) <= TOL * abs(r), (norms, ref)


@pytest.mark.parametrize("case", ["2d_mc", "2d_minmod", "2d_superbee", "3d_mc"])
def test_diagonal(case):
    dim, lim = int(case[0]), case.split("_")[1]
    n = int(next(iter(GOLD["reference"]["diagonal"][case])))
    P = port.PortGrid(dim, (n,) * dim, (1.0 / n,) * dim, ghosts=2, riemann=2, limiter=LIMITERS[lim], cfl=1)
    w0, _ = problems.diagonal_advection(dim, n, ghosts=P.ghosts)
    P.set_prim(w0)
    P.set_boundary(bc_entries_from(boundary.as_list(boundary.Periodic())))
    t = main_loop(P, 0.05, 1.0)
    check(problems.diagonal_errors(P.get_prim(), n, t, P.ghosts), GOLD["reference"]["diagonal"][case][str(n)])


@pytest.mark.parametrize("case,n", [("2d_uniform", 32), ("2d_gaussian", 32), ("3d_uniform", 16)])
def test_field_loop(case, n):
    dim, gaussian = int(case[0]), case.endswith("gaussian")
    ns = (n, n // 2) if dim == 2 else (n, n // 2, n // 2)
    P = port.PortGrid(dim, ns, (2.0 / n,) * dim, ghosts=3, mhd=True, riemann=5, limiter=1, cfl=1, ct_energy=0)
    w, B, _ = problems.field_loop(dim, n, ghosts=P.ghosts, gaussian=gaussian)
    P.set_prim(w)
    P.set_faceB(B)
    P.set_boundary(bc_entries_from(boundary.as_list(boundary.Periodic())))
    P.initialize_B_fields()
    w0 = P.get_prim()
    main_loop(P, 0.1, 4.0)
    check(problems.loop_errors(P.get_prim(), w0, n, P.ghosts), GOLD["reference"]["loop"][case][str(n)])
