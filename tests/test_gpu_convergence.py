"""The reference's accuracy studies on the device path.

Examples/Diagonal and Examples/LoopAdvection publish L1 / L2 / max error
tables (Outputs/Validation_data.md) for a smooth density wave advected along
the diagonal (HLLC, 2D and 3D, three limiters) and for a weak field loop
advected across a periodic box (HLLD + CT). Each case here runs the example's
main loop (DRAGON/main/main.cpp:124-150: advance(dt), t += dt while t <
final_time) through dragon_b200.grid on the GPU, computes the example's norms
(problemComplete) and compares them:
  * with the published table to its 6 printed digits, for the rows the
    reference's own sources reproduce (tests/golden/convergence.json
    "reproduced"; the 2D uniform-loop and 3D diagonal tables are not
    among them);
  * with the reference's own output at small sizes (convergence.json
    "reference", made by tests/golden/make_convergence.py) to 1e-12
    relative, since the FP64 path is the reference's arithmetic.
The mixed-precision path runs the 2D MC wave at n = 512 too (7,800 steps):
its density field stays within TOL_MIXED_STATE relative L1 of the FP64 one,
and its error norm within TOL_MIXED_ERR of the FP64 norm (the FP32 flux
rounding, accumulated over the run, moves the L1 error by about 2 %).
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT, cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import problems  # noqa: E402

with open(os.path.join(ROOT, "tests", "golden", "convergence.json")) as _f:
    GOLD = json.load(_f)

LIMITERS = {"minmod": dg.LIMITER_MINMOD, "mc": dg.LIMITER_MC, "superbee": dg.LIMITER_SUPERBEE}
TOL_REF = 1e-12      # relative, against the reference's own output
TOL_MIXED_STATE = 1e-5  # relative L1 of the mixed density field against FP64
TOL_MIXED_ERR = 0.05    # relative change of the L1 error norm, mixed vs FP64
LOOP3D_MAX_N = 128      # the 256 rows take minutes each; they were run once


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def main_loop(G, dt, final_time):
    t = 0.0
    while t < final_time:
        G.advance(dt)
        t += dt
    return t


def run_diagonal(dim, n, limiter, precision=dg.PREC_FP64, keep=False):
    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=LIMITERS[limiter], cfl=dg.CFL_ADD, precision=precision)
    cls = dg.Grid2D if dim == 2 else dg.Grid3D
    G = cls(*([n] * dim), *([1.0 / n] * dim), ghosts=2, config=cfg)
    w0, _ = problems.diagonal_advection(dim, n, ghosts=G.ghosts)
    G.w[...] = w0
    G.boundary = dg.boundary.Periodic()
    t = main_loop(G, 0.05, 1.0)
    norms = problems.diagonal_errors(G.w, n, t, G.ghosts)
    return (norms, np.array(G.w)) if keep else norms


def run_loop(dim, n, gaussian):
    cfg = dg.Config(mhd=True, riemann=dg.RIEMANN_HLLX, limiter=dg.LIMITER_MC, cfl=dg.CFL_ADD,
                    ct_energy=dg.CT_CONSV_TOTAL_E)
    d = 2.0 / n
    if dim == 2:
        G = dg.Grid2D(n, n // 2, d, d, ghosts=3, config=cfg)
    else:
        G = dg.Grid3D(n, n // 2, n // 2, d, d, d, ghosts=3, config=cfg)
    w, B, _ = problems.field_loop(dim, n, ghosts=G.ghosts, gaussian=gaussian)
    G.w[...] = w
    G.B[...] = B
    G.boundary = dg.boundary.Periodic()
    G.initialize_B_fields()
    w0 = np.array(G.w)
    main_loop(G, 0.1, 4.0)
    return problems.loop_errors(G.w, w0, n, G.ghosts)


def six_digits(v, pub):
    """v agrees with pub as the reference prints it (std::cout, 6 significant digits)."""
    unit = 10.0 ** (math.floor(math.log10(abs(pub))) - 5)
    return abs(v - pub) <= 0.5 * unit * (1 + 1e-9)


def check_published(study, case, n, norms):
    pub = GOLD["published"][study][case][str(n)]
    print(f"{study} {case} n={n}: L1 {norms[0]:.6g} L2 {norms[1]:.6g} Linf {norms[2]:.6g}; published {pub}")
    for name, v, p in zip(("L1", "L2", "Linf"), norms, pub):
        assert six_digits(v, p), f"{study} {case} n={n} {name}: {v!r} vs published {p}"


def check_reference(study, case, n, norms):
    ref = GOLD["reference"][study][case][str(n)]
    for name, v, r in zip(("L1", "L2", "Linf"), norms, ref):
        assert abs(v - r) <= TOL_REF * abs(r), f"{study} {case} n={n} {name}: {v!r} vs reference {r!r}"


def published_cases(study, case):
    assert case in GOLD["reproduced"][study]
    return [int(n) for n in GOLD["published"][study][case]]


@pytest.mark.parametrize("limiter,n", [(lim, n) for lim in ("mc", "minmod", "superbee")
                                       for n in published_cases("diagonal", "2d_" + lim)])
def test_diagonal_2d_published(limiter, n):
    check_published("diagonal", "2d_" + limiter, n, run_diagonal(2, n, limiter))


@pytest.mark.parametrize("case,n", [(c, int(n)) for c, rows in GOLD["reference"]["diagonal"].items() for n in rows])
def test_diagonal_small_matches_reference(case, n):
    dim, limiter = int(case[0]), case.split("_")[1]
    check_reference("diagonal", case, n, run_diagonal(dim, n, limiter))


@pytest.mark.parametrize("n", published_cases("loop", "2d_gaussian"))
def test_loop_2d_gaussian_published(n):
    check_published("loop", "2d_gaussian", n, run_loop(2, n, True))


@pytest.mark.parametrize("case,n", [(c, n) for c in ("3d_uniform", "3d_gaussian")
                                    for n in published_cases("loop", c) if n <= LOOP3D_MAX_N])
def test_loop_3d_published(case, n):
    check_published("loop", case, n, run_loop(3, n, case.endswith("gaussian")))


@pytest.mark.parametrize("case,n", [(c, int(n)) for c, rows in GOLD["reference"]["loop"].items() for n in rows])
def test_loop_small_matches_reference(case, n):
    dim, shape = int(case[0]), case.split("_")[1]
    check_reference("loop", case, n, run_loop(dim, n, shape == "gaussian"))


def test_mixed_precision_keeps_the_error():
    n = 512
    fp64, w64 = run_diagonal(2, n, "mc", keep=True)
    mixed, wmx = run_diagonal(2, n, "mc", precision=dg.PREC_MIXED, keep=True)
    g = 2
    rho64 = w64[g:g + n, g:g + n, 0]
    rel = float(np.abs(wmx[g:g + n, g:g + n, 0] - rho64).sum() / np.abs(rho64).sum())
    print(f"diagonal 2d mc n={n}: FP64 {fp64}, mixed {mixed}, density rel L1 {rel:.3g}")
    assert rel <= TOL_MIXED_STATE
    assert abs(mixed[0] - fp64[0]) <= TOL_MIXED_ERR * fp64[0], (mixed, fp64)
