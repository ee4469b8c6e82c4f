"""GPU parity of the hydro path (1D sweep, 2D CTU) against the reference.

Every case runs the same seeded input through the device path (through the C
ABI, via dragon_b200.grid) and through the reference's own code
(oracle/_ref), and compares the padded arrays. Solvers without pow (HLLC, HLL,
HLLE, Roe) must agree bit for bit; paths through the exact solver differ only
by CUDA's pow vs glibc's pow (within 2 ulp), so they are held to 1e-12
relative L1 per field (the bar for the FP64 path).
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import problems  # noqa: E402

TOL_L1 = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


class _PortModule:
    """The C restatement with the reference handle's module interface."""

    def __init__(self):
        from oracle import port, refgrid
        self.RefGrid = port.PortGrid
        self.bc_entries_from = refgrid.bc_entries_from


def ref_mod():
    """The reference library when it was built, else the C restatement pinned to it."""
    from oracle import refgrid
    if refgrid.available("hydro"):
        return refgrid
    return _PortModule()


def make_pair(dim, n, d, w0, boundary, riemann=dg.RIEMANN_HLLX, limiter=dg.LIMITER_MC, cfl=dg.CFL_ADD, ghosts=2):
    refgrid = ref_mod()
    cfg = dg.Config(riemann=riemann, limiter=limiter, cfl=cfl)
    G = {1: dg.Grid1D, 2: dg.Grid2D, 3: dg.Grid3D}[dim](*n, *d, ghosts=ghosts, config=cfg)
    R = refgrid.RefGrid(dim, n, d, ghosts=ghosts, riemann=riemann, limiter=limiter, cfl=cfl)
    assert G.ghosts == R.ghosts
    G.w[...] = w0
    R.set_prim(w0)
    G.boundary = boundary
    R.set_boundary(refgrid.bc_entries_from(dg.boundary.as_list(boundary)))
    return G, R


def assert_same(a, b, exact=True, what=""):
    if exact:
        bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
        assert bad.size == 0, f"{what}: {len(bad)} mismatches, first at {bad[:3].tolist()}: " \
                              f"{a[tuple(bad[0])]} vs {b[tuple(bad[0])]}"
    else:
        l1 = problems.rel_l1(a, b)
        assert np.all(l1 <= TOL_L1), f"{what}: rel L1 per field {l1}"


def ref_advance_log(R, interval, tol=1e-14):
    """Grid::advance_unsplit (CFL.cpp:188-213) driven step by step through the
    reference's own boundary/CFL/step functions, logging the dt sequence."""
    dts = []
    while interval > tol:
        R.apply_boundary()
        t1 = min(interval, R.cfl_time())
        R.unsplit_step(t1)
        dts.append(t1)
        interval -= t1
    return dts


# ---------------------------------------------------------------------------
def test_sod_1d_to_t02_bitwise_and_dt_sequence():
    """The 1D Sod configuration: 512 cells, HLLC, minmod, outflow, CFL 0.3, t = 0.2."""
    w0, dx = problems.sod_1d(512, ghosts=2)
    G, R = make_pair(1, (512,), (dx,), w0, dg.Outflow(), riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MINMOD)
    dts = ref_advance_log(R, 0.2)
    res = G.advance(0.2)
    assert res.steps == len(dts)
    assert res.last_dt == dts[-1]
    assert res.retries == 0
    assert_same(G.w, R.get_prim(), exact=res.pivots_exact == 0, what="sod")
    # the logged loop is the reference's own advance(): same state
    R2 = ref_mod().RefGrid(1, (512,), (dx,), ghosts=2, riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_MINMOD)
    R2.set_prim(w0)
    R2.advance(0.2)
    assert_same(R2.get_prim(), R.get_prim(), what="ref advance vs logged loop")


@pytest.mark.parametrize("riemann", [dg.RIEMANN_HLLC, dg.RIEMANN_HLL, dg.RIEMANN_HLLE, dg.RIEMANN_ROE,
                                     dg.RIEMANN_EXACT])
@pytest.mark.parametrize("limiter", [0, 1, 2, 3, 4])
def test_1d_solvers_limiters(riemann, limiter):
    w0, dx = problems.sod_1d(200, ghosts=2, left=(1.0, 0.75, 1.0), right=(0.125, 0.0, 0.1))
    w0[2:-2, 3] = 0.3  # transverse velocity rides along
    G, R = make_pair(1, (200,), (dx,), w0, dg.Reflective("X-") + dg.Outflow.Gated("X+"), riemann=riemann,
                     limiter=limiter)
    for _ in range(25):
        R.step_cfl()
    G.advance_steps(25)
    exact = riemann != dg.RIEMANN_EXACT
    assert_same(G.w, R.get_prim(), exact=exact, what=f"1d s{riemann} l{limiter}")


def kh_pair(n, ny, riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_VANLEER, boundary=None, seed=1234):
    w0, dx, dy = problems.kelvin_helmholtz_2d(n, ghosts=2, seed=seed, ny=ny)
    return make_pair(2, (n, ny), (dx, dy), w0, boundary or dg.Periodic(), riemann=riemann, limiter=limiter)


def test_kh_2d_small_bitwise():
    """BASELINE 2D shear-layer setup at 64 x 64, 20 CFL steps."""
    G, R = kh_pair(64, 64)
    dts = [R.step_cfl() for _ in range(20)]
    res = G.advance_steps(20)
    assert res.steps == 20
    assert res.last_dt == dts[-1]
    assert_same(G.w, R.get_prim(), what="kh64")


def test_kh_2d_ragged_tiles_bitwise():
    """Extents that are not multiples of the 8 x 32 tile."""
    G, R = kh_pair(45, 77, boundary=dg.Periodic("X") + dg.Reflective("Y"))
    for _ in range(8):
        R.step_cfl()
    G.advance_steps(8)
    assert_same(G.w, R.get_prim(), what="kh45x77")


@pytest.mark.parametrize("riemann", [dg.RIEMANN_HLLC, dg.RIEMANN_HLL, dg.RIEMANN_HLLE, dg.RIEMANN_ROE,
                                     dg.RIEMANN_EXACT])
@pytest.mark.parametrize("limiter", [0, 1, 2, 3, 4])
def test_2d_solvers_limiters(riemann, limiter):
    G, R = kh_pair(24, 40, riemann=riemann, limiter=limiter,
                   boundary=dg.Outflow("X") + dg.Reflective("Y-") + dg.Outflow.Gated("Y+"))
    for _ in range(6):
        R.step_cfl()
    G.advance_steps(6)
    assert_same(G.w, R.get_prim(), exact=riemann != dg.RIEMANN_EXACT, what=f"2d s{riemann} l{limiter}")


def test_2d_advance_interval_matches_reference():
    G, R = kh_pair(32, 32)
    R.advance(0.05)
    res = G.advance(0.05)
    assert res.steps > 1
    assert_same(G.w, R.get_prim(), what="advance(0.05)")


def random_padded(shape, rng):
    w = np.zeros(shape)
    w[..., 0] = 10 ** rng.uniform(-1, 0.5, shape[:-1])
    w[..., 1] = 10 ** rng.uniform(-1, 0.5, shape[:-1])
    w[..., 2:5] = rng.uniform(-0.5, 0.5, shape[:-1] + (3,))
    return w


BC_CASES = [
    ("outflow", lambda: dg.Outflow()),
    ("outflow_nocorner", lambda: dg.Outflow("XY", False)),
    ("gated", lambda: dg.Outflow.Gated("XY")),
    ("reflective", lambda: dg.Reflective()),
    ("reflective_x_periodic_y", lambda: dg.Reflective("X") + dg.Periodic("YZ")),
    ("fixed_left", lambda: dg.Fixed([1.5, 0.7, 0.1, -0.2, 0.05], "X-") + dg.Outflow("X+Y", False)),
    ("periodic_nocorner", lambda: dg.Periodic("XY", False)),
    ("ignore_y", lambda: dg.Ignore("Y") + dg.Reflective("X", False)),
    ("mixed_order", lambda: dg.Periodic("X") + dg.Fixed([2, 1, 0, 0, 0], "Y+", False) + dg.Reflective("Y-")),
]


@pytest.mark.parametrize("name,make", BC_CASES)
def test_ghost_fill_and_cfl_bitwise(name, make):
    refgrid = ref_mod()
    rng = np.random.default_rng(abs(hash(name)) % 2 ** 32)
    nx, ny = 13, 9
    w0 = random_padded((nx + 4, ny + 4, 5), rng)
    G = dg.Grid2D(nx, ny, 0.1, 0.07, ghosts=2)
    R = refgrid.RefGrid(2, (nx, ny), (0.1, 0.07), ghosts=2)
    G.w[...] = w0
    R.set_prim(w0)
    b = make()
    G.boundary = b
    R.set_boundary(refgrid.bc_entries_from(dg.boundary.as_list(b)))
    G.apply_boundary()
    R.apply_boundary()
    assert_same(G.w, R.get_prim(), what=f"ghosts {name}")
    assert G.cfl_time() == R.cfl_time()
    # 1D variant of the same list
    w1 = random_padded((nx + 4, 5), rng)
    G1 = dg.Grid1D(nx, 0.1, ghosts=2)
    R1 = refgrid.RefGrid(1, (nx,), (0.1,), ghosts=2)
    G1.w[...] = w1
    R1.set_prim(w1)
    G1.boundary = b
    R1.set_boundary(refgrid.bc_entries_from(dg.boundary.as_list(b)))
    G1.apply_boundary()
    R1.apply_boundary()
    assert_same(G1.w, R1.get_prim(), what=f"ghosts1d {name}")
    assert G1.cfl_time() == R1.cfl_time()


def test_uniform_flow_unchanged_and_dt0_identity():
    """HydroGodunov_Tests.cpp:17-118,202-259: uniform states stay put; dt=0 is the identity."""
    n = 10
    w = np.zeros((n + 4, n + 4, 5))
    w[..., 0], w[..., 1], w[..., 2], w[..., 3], w[..., 4] = 1.0, 5.0, 1.0, 2.0, 3.0
    G = dg.Grid2D(n, n, 1.0, 1.0, ghosts=2)
    G.w[...] = w
    G.boundary = dg.Outflow()
    G.advance(1.0)
    assert np.allclose(G.interior(), w[2:-2, 2:-2], rtol=1e-15, atol=1e-18)
    rng = np.random.default_rng(0)
    w = random_padded((n + 4, n + 4, 5), rng)
    G.w[...] = w
    G.unsplit_step(0.0)
    ref = ref_mod().RefGrid(2, (n, n), (1.0, 1.0), ghosts=2)
    ref.set_prim(w)
    ref.unsplit_step(0.0)
    assert_same(G.w, ref.get_prim(), what="dt=0")


def test_periodic_conservation():
    """HydroGodunov_Tests.cpp:121-200: sums of conserved quantities hold to roundoff."""
    G, _ = kh_pair(48, 48)
    def totals(w):
        inner = w[2:-2, 2:-2]
        rho, p, v = inner[..., 0], inner[..., 1], inner[..., 2:5]
        E = p / (5.0 / 3.0 - 1.0) + 0.5 * rho * (v * v).sum(-1)
        return np.array([rho.sum(), (rho * v[..., 0]).sum(), (rho * v[..., 1]).sum(), E.sum()])
    t0 = totals(G.w)
    G.advance_steps(30)
    t1 = totals(G.w)
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.maximum(1, np.abs(t0)))


def test_failed_step_commits_nothing():
    """A step that would make an unphysical state raises and leaves the grid as
    it was (Unsplit.cpp:95-99 throws before the commit). The input is one the
    reference's own step rejects: a converging flow at Mach ~2000 with dt = 0.05
    (CFL number ~40)."""
    n = 16
    w = np.zeros((n + 4, n + 4, 5))
    w[..., 0], w[..., 1] = 1.0, 1e-3
    w[2:10, :, 2] = 50.0      # strong converging flow
    w[10:, :, 2] = -50.0
    G = dg.Grid2D(n, n, 1.0 / n, 1.0 / n, ghosts=2)
    G.w[...] = w
    G.boundary = dg.Outflow()
    G.apply_boundary()
    before = G.w.copy()
    R = ref_mod().RefGrid(2, (n, n), (1.0 / n, 1.0 / n), ghosts=2)
    R.set_prim(before)
    with pytest.raises(Exception):
        R.unsplit_step(0.05)
    assert_same(R.get_prim(), before, what="reference: no commit")
    with pytest.raises(dg.StepFailed) as exc:
        G.unsplit_step(0.05)
    assert exc.value.status.code == 3  # DRAGON_GPU_ESTEP
    assert_same(G.w, before, what="no commit")
    # the grid stays usable: a step the reference takes is taken bit for bit
    R.unsplit_step(1e-4)
    G.unsplit_step(1e-4)
    assert_same(G.w, R.get_prim(), what="step after the failure")


def test_retry_halving_matches_reference():
    """advance() halves dt after a failed step and retries (CFL.cpp:194-209)."""
    n = 32
    w0, dx = problems.sod_1d(n, ghosts=2, left=(1.0, 0.0, 1000.0), right=(1.0, 0.0, 0.01))
    G, R = make_pair(1, (n,), (dx,), w0, dg.Outflow(), riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_SUPERBEE)
    R.advance(0.02, False)
    res = G.advance(0.02, check_cfl=False)
    assert res.retries > 0, res
    assert_same(G.w, R.get_prim(), exact=res.pivots_exact == 0, what="forced dt")


def ref_step_with_retries(R, tol=1e-14):
    """One CFL step of Grid::advance_unsplit (CFL.cpp:188-209) through the
    reference's own functions: ghost fill, CFL dt, then the step, halving dt on
    the same ghosts until it succeeds. Returns (dt taken, retries)."""
    R.apply_boundary()
    t1 = R.cfl_time()
    retries = 0
    while True:
        try:
            R.unsplit_step(t1)
            return t1, retries
        except Exception:
            retries += 1
            t1 *= 0.5
            assert t1 >= tol


@pytest.mark.parametrize("nsteps", [1, 3])
def test_retry_on_last_step_of_budget(nsteps):
    """advance_steps(k) whose CFL steps fail and are retried, the last one
    included: with CFL_coeff = 2 every CFL-limited step of this shock tube is
    rejected once and taken at half the dt. The bookkeeping of a budget's last
    step then runs on the host after a retry."""
    n = 32
    w0, dx = problems.sod_1d(n, ghosts=2, left=(1.0, 0.0, 1000.0), right=(1.0, 0.0, 0.01))
    cfg = dg.Config(riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_SUPERBEE, cfl_coeff=2.0)
    G = dg.Grid1D(n, dx, ghosts=2, config=cfg)
    G.w[...] = w0
    G.boundary = dg.Outflow()
    # CFL_coeff is a compile-time constant of the reference (Config.h:67), so
    # the oracle here is its C restatement, which takes the coefficient at run
    # time and is pinned bit for bit to the reference (test_oracle_port.py)
    from oracle import port, refgrid
    R = port.PortGrid(1, (n,), (dx,), ghosts=2, riemann=dg.RIEMANN_HLLC, limiter=dg.LIMITER_SUPERBEE, cfl_coeff=2.0)
    R.set_prim(w0)
    R.set_boundary(refgrid.bc_entries_from(dg.boundary.as_list(dg.Outflow())))
    log = [ref_step_with_retries(R) for _ in range(nsteps)]
    assert log[-1][1] > 0, log  # the budget's last step was retried in the reference
    res = G.advance_steps(nsteps)
    assert res.steps == nsteps
    assert res.retries == sum(r for _, r in log), (res.retries, log)
    assert res.last_dt == log[-1][0]
    assert res.time_advanced == sum(t for t, _ in log)
    assert_same(G.w, R.get_prim(), exact=res.pivots_exact == 0, what="budget with retries")


@pytest.mark.parametrize("dim", [1, 2])
def test_pivot_to_exact_matches_reference(dim):
    """verify_and_fallback (Flux.cpp:77-97): with the Roe solver this two-state
    problem gives face fluxes that would empty a neighbouring cell, so faces
    pivot to the exact solver (counted), and the state still follows the
    reference to 1e-12 (the exact solver's pow)."""
    n = 128
    w1, dx = problems.riemann_1d(n, (0.607, -0.867, 0.049), (4.686, 0.985, 0.014), ghosts=2)
    if dim == 1:
        G, R = make_pair(1, (n,), (dx,), w1, dg.Outflow(), riemann=dg.RIEMANN_ROE, limiter=dg.LIMITER_MINMOD)
    else:
        ny = 32
        w = np.repeat(w1[:, None, :], ny + 4, axis=1)
        rng = np.random.default_rng(3)
        w[2:-2, 2:-2, 3] = 0.01 * rng.uniform(-1.0, 1.0, (n, ny))
        G, R = make_pair(2, (n, ny), (dx, dx), w, dg.Outflow("X") + dg.Periodic("Y"), riemann=dg.RIEMANN_ROE,
                         limiter=dg.LIMITER_MINMOD)
    dts = ref_advance_log(R, 0.05)
    res = G.advance(0.05)
    assert res.pivots_exact > 0, res
    assert res.steps == len(dts) and res.retries == 0
    assert_same(G.w, R.get_prim(), exact=False, what=f"{dim}D pivot")


def test_launch_count_reports_native_kernels():
    G, _ = kh_pair(16, 16)
    before = G.launch_count()
    G.advance_steps(3)
    assert G.launch_count() - before >= 6
