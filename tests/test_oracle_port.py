"""Pins the C restatement (oracle/dragon_oracle.c) to the reference.

1. Golden vectors from the reference's own tests (exact Sod star state,
   Testing/Core/Riemann/Riemann_Exact_Tests.cpp:116-149; limiter and MUSCL
   known answers, Testing/Core/TVD_Tests.cpp:64-213) hold for the oracle.
2. Bit-for-bit agreement with the reference library (oracle/_ref) on
   random unit inputs, every boundary type, and whole steps / advance loops
   in 1D, 2D and 3D, hydro and MHD, every solver and limiter.
CPU only (no GPU)."""
import ctypes

import numpy as np
import pytest

from oracle import port
from oracle import refgrid

D = ctypes.POINTER(ctypes.c_double)


def P(a):
    return a.ctypes.data_as(D)


def need_ref(variant="hydro"):
    if not refgrid.available(variant):
        pytest.skip("reference library not built")


def approx(a, b, rel=1e-15, abs_=1e-18):
    """DRAGON_Test::approx (Testing/Core/FluidElement_Tests.cpp:83-85)."""
    return abs(a - b) <= abs_ + rel * max(abs(a), abs(b))


# --- golden vectors ---------------------------------------------------------
def test_exact_sod_golden():
    L = port.load(False)
    sl, sr = np.zeros(5), np.zeros(5)
    it = ctypes.c_int()
    L.ora_exact_star(P(np.array([1.0, 1.0, 0, 0, 0])), P(np.array([0.125, 0.1, 0, 0, 0])), -1.0, P(sl), P(sr),
                     ctypes.byref(it))
    assert approx(sl[1], 0.29394518766601785) and approx(sr[1], 0.29394518766601785)
    assert approx(sl[2], 0.8411948521688083) and approx(sr[2], 0.8411948521688083)
    assert approx(sl[0], 0.4796890587209175)
    assert approx(sr[0], 0.22980574931194703)


def test_limiter_golden():
    L = port.load(False)
    lim = L.ora_limiter
    assert lim(0, 2.0, 3.0) == 2.0 and lim(0, -2.0, -3.0) == -2.0 and lim(0, -2.0, 3.0) == 0.0
    assert lim(1, 1.0, 3.0) == 2.0 and lim(1, -1.0, -3.0) == -2.0 and lim(1, 1.0, -3.0) == 0.0
    assert approx(lim(2, 2.0, 4.0), 8.0 / 3.0) and lim(2, 2.0, -4.0) == 0.0
    assert lim(3, 1.0, 4.0) == 2.0 and lim(3, 4.0, 1.0) == 2.0 and lim(3, -1.0, -4.0) == -2.0
    assert approx(lim(4, 2.0, 4.0), 12.0 / 5.0) and lim(4, 2.0, -4.0) == 0.0


def test_muscl_golden():
    """Zero-dt reconstruction and the first-order fallback (TVD_Tests.cpp:173-231)."""
    L = port.load(False)
    L.ora_set_options(5, 0, 1, 2, 6, 1e-12, 0.3, 1e-14)
    wl, wc, wr = (np.array(v, dtype=float) for v in ([1, 4, 1, 2, 3], [2, 5, 2, 3, 4], [3, 6, 3, 4, 5]))
    oL, oR = np.zeros(5), np.zeros(5)
    L.ora_muscl(P(wl), P(wc), P(wr), 0.0, P(np.zeros(3)), P(oL), P(oR))
    assert np.allclose(oL, [1.5, 4.5, 1.5, 2.5, 3.5], rtol=1e-15) and np.allclose(oR, [2.5, 5.5, 2.5, 3.5, 4.5])
    L.ora_set_options(5, 3, 1, 2, 6, 1e-12, 0.3, 1e-14)
    wl, wc, wr = (np.array(v, dtype=float) for v in ([1, 1, 0, 0, 0], [1, 1, 0, 0, 0], [10, 1, 0, 0, 0]))
    L.ora_muscl(P(wl), P(wc), P(wr), 0.0, P(np.zeros(3)), P(oL), P(oR))
    assert np.array_equal(oL, wc) and np.array_equal(oR, wc)


# --- bitwise against the reference ------------------------------------------
def rand_state(rng, nf):
    w = np.zeros(nf)
    w[0] = 10 ** rng.uniform(-2, 1)
    w[1] = 10 ** rng.uniform(-2, 2)
    w[2:5] = rng.uniform(-2, 2, 3) * rng.choice([0.0, 0.1, 1.0, 4.0])
    if nf == 8:
        w[5:8] = rng.uniform(-1, 1, 3) * rng.choice([0.0, 0.05, 1.0, 5.0])
    return w


@pytest.mark.parametrize("mhd", [False, True])
def test_unit_functions_bitwise(mhd):
    need_ref("mhd" if mhd else "hydro")
    R = refgrid.load("mhd" if mhd else "hydro")
    O = port.load(mhd)
    nf = 8 if mhd else 5
    rng = np.random.default_rng(21)
    msg = ctypes.create_string_buffer(64)
    for it in range(1500):
        a, b, c = (rand_state(rng, nf) for _ in range(3))
        lim = it % 5
        dt = rng.uniform(0, 0.5)
        dB = rng.uniform(-0.2, 0.2, 3) if mhd else np.zeros(3)
        R.ref_config(5, lim, 1, 2, 1)
        O.ora_set_options(5, lim, 1, 2, 6, 1e-12, 0.3, 1e-14)
        o = [np.zeros(nf) for _ in range(4)]
        R.ref_muscl(P(a), P(b), P(c), dt, P(dB), P(o[0]), P(o[1]))
        O.ora_muscl(P(a), P(b), P(c), dt, P(dB), P(o[2]), P(o[3]))
        assert np.array_equal(o[0], o[2], equal_nan=True) and np.array_equal(o[1], o[3], equal_nan=True)
        for s in ([5, 1, 4] if mhd else [5, 1, 4, 6, 0]):
            ax = int(rng.integers(0, 3))
            R.ref_config(s, lim, 1, 2, 1)
            rc1 = R.ref_riemann_flux(-1, P(a), P(b), dt, ax, P(o[0]), msg, 64)
            rc2 = O.ora_riemann_flux(s, P(a), P(b), dt, ax, P(o[1]))
            assert rc1 == rc2
            if rc1 == 0:
                assert np.array_equal(o[0], o[1], equal_nan=True), (s, a, b)


def random_padded(shape, rng, nf):
    w = np.zeros(shape + (nf,))
    w[..., 0] = 10 ** rng.uniform(-0.5, 0.5, shape)
    w[..., 1] = 10 ** rng.uniform(-0.5, 0.5, shape)
    w[..., 2:5] = rng.uniform(-0.3, 0.3, shape + (3,))
    if nf == 8:
        w[..., 5:8] = rng.uniform(-0.5, 0.5, shape + (3,))
    return w


BCS = [
    [],
    [(0, 63, 0, None)],
    [(1, 63, 1, None)],
    [(3, 63, 1, None)],
    [(3, 3, 1, None), (4, 60, 1, None)],
    [(2, 1, 1, [1.5, 0.7, 0.1, -0.2, 0.05, 0.3, -0.1, 0.2]), (0, 2 | 12, 0, None)],
    [(4, 63, 0, None)],
    [(5, 12, 1, None), (3, 3, 0, None)],
    [(4, 3, 1, None), (2, 8, 0, [2, 1, 0, 0, 0, 0.1, 0.2, 0.3]), (3, 4 | 48, 1, None)],
]


@pytest.mark.parametrize("mhd", [False, True])
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bc", range(len(BCS)))
def test_boundaries_bitwise(mhd, dim, bc):
    need_ref("mhd" if mhd else "hydro")
    nf = 8 if mhd else 5
    n = {1: (9,), 2: (7, 6), 3: (5, 4, 6)}[dim]
    d = (0.1, 0.07, 0.05)[:dim]
    rng = np.random.default_rng(100 * dim + bc)
    R = refgrid.RefGrid(dim, n, d, ghosts=2, mhd=mhd)
    O = port.PortGrid(dim, n, d, ghosts=2, mhd=mhd)
    w = random_padded(R.shape[:-1], rng, nf)
    R.set_prim(w)
    O.set_prim(w)
    if mhd and dim >= 2:
        b = rng.uniform(-1, 1, R.bshape)
        R.set_faceB(b)
        O.set_faceB(b)
    R.set_boundary(BCS[bc])
    O.set_boundary(BCS[bc])
    R.apply_boundary()
    O.apply_boundary()
    assert np.array_equal(R.get_prim(), O.get_prim())
    if mhd and dim >= 2:
        assert np.array_equal(R.get_faceB(), O.get_faceB())
    assert R.cfl_time() == O.cfl_time()


def kh(n, ny, g=2, seed=5):
    from dragon_b200 import problems
    return problems.kelvin_helmholtz_2d(n, ghosts=g, seed=seed, ny=ny)


@pytest.mark.parametrize("riemann", [5, 1, 4, 6, 0])
@pytest.mark.parametrize("limiter", [0, 1, 2, 3, 4])
def test_hydro_2d_steps_bitwise(riemann, limiter):
    need_ref()
    w0, dx, dy = kh(14, 11)
    kw = dict(riemann=riemann, limiter=limiter)
    R = refgrid.RefGrid(2, (14, 11), (dx, dy), ghosts=2, **kw)
    O = port.PortGrid(2, (14, 11), (dx, dy), ghosts=2, **kw)
    for G in (R, O):
        G.set_prim(w0)
        G.set_boundary([(4, 3, 1, None), (3, 12, 1, None)])
        G.advance(0.02)
    assert np.array_equal(R.get_prim(), O.get_prim())


@pytest.mark.parametrize("riemann", [5, 0, 6])
def test_hydro_1d_and_3d_bitwise(riemann):
    need_ref()
    from dragon_b200 import problems
    w1, dx = problems.sod_1d(64, ghosts=2)
    R = refgrid.RefGrid(1, (64,), (dx,), ghosts=2, riemann=riemann, limiter=0)
    O = port.PortGrid(1, (64,), (dx,), ghosts=2, riemann=riemann, limiter=0)
    for G in (R, O):
        G.set_prim(w1)
        G.advance(0.05)
    assert np.array_equal(R.get_prim(), O.get_prim())

    w3, d3 = problems.blast_3d(10, ghosts=2)
    rng = np.random.default_rng(9)
    w3[..., 2:5] = rng.uniform(-0.2, 0.2, w3.shape[:-1] + (3,))
    w3[..., 0] = np.where(w3[..., 0] > 0, w3[..., 0], 1.0)
    w3[..., 1] = np.where(w3[..., 1] > 0, w3[..., 1], 0.1)
    R = refgrid.RefGrid(3, (10, 10, 10), (d3, d3, d3), ghosts=2, riemann=riemann, limiter=1)
    O = port.PortGrid(3, (10, 10, 10), (d3, d3, d3), ghosts=2, riemann=riemann, limiter=1)
    for G in (R, O):
        G.set_prim(w3)
        G.set_boundary([(3, 63, 1, None)])
        for _ in range(3):
            G.step_cfl()
    assert np.array_equal(R.get_prim(), O.get_prim())


@pytest.mark.parametrize("riemann", [5, 1, 4])
@pytest.mark.parametrize("ct", [0, 1, 2])
def test_mhd_2d_steps_bitwise(riemann, ct):
    variant = "mhd" if ct == 2 else "mhd_rt"
    need_ref(variant)
    from dragon_b200 import problems
    w0, B0, dx, dy = problems.orszag_tang_2d(16, ghosts=3)
    R = refgrid.RefGrid(2, (16, 16), (dx, dy), ghosts=3, mhd=True, ct_runtime=(ct != 2), riemann=riemann, limiter=1,
                        ct_energy=ct)
    O = port.PortGrid(2, (16, 16), (dx, dy), ghosts=3, mhd=True, riemann=riemann, limiter=1, ct_energy=ct)
    for G in (R, O):
        G.set_prim(w0)
        G.set_faceB(B0)
        G.set_boundary([(4, 63, 1, None)])
        G.initialize_B_fields()
        for _ in range(4):
            G.step_cfl()
    assert np.array_equal(R.get_prim(), O.get_prim())
    assert np.array_equal(R.get_faceB(), O.get_faceB())


def test_mhd_blast_2d_and_3d_bitwise():
    need_ref("mhd")
    from dragon_b200 import problems
    w0, B0, dx = problems.blast_2d_mhd(12, ghosts=3)
    R = refgrid.RefGrid(2, (12, 12), (dx, dx), ghosts=3, mhd=True, limiter=2)
    O = port.PortGrid(2, (12, 12), (dx, dx), ghosts=3, mhd=True, limiter=2)
    for G in (R, O):
        G.set_prim(w0)
        G.set_faceB(B0)
        G.set_boundary([(0, 63, 1, None)])
        G.initialize_B_fields()
        G.advance(0.01)
    assert np.array_equal(R.get_prim(), O.get_prim())
    assert np.array_equal(R.get_faceB(), O.get_faceB())

    n = 7
    rng = np.random.default_rng(4)
    R = refgrid.RefGrid(3, (n, n, n), (0.1, 0.1, 0.1), ghosts=3, mhd=True)
    O = port.PortGrid(3, (n, n, n), (0.1, 0.1, 0.1), ghosts=3, mhd=True)
    w = random_padded(R.shape[:-1], rng, 8)
    b = np.zeros(R.bshape)
    b[..., 0], b[..., 1], b[..., 2] = 0.3, -0.2, 0.1
    b += rng.uniform(-0.01, 0.01, b.shape)
    for G in (R, O):
        G.set_prim(w)
        G.set_faceB(b)
        G.set_boundary([(4, 63, 1, None)])
        G.initialize_B_fields()
        for _ in range(2):
            G.step_cfl()
    assert np.array_equal(R.get_prim(), O.get_prim())
    assert np.array_equal(R.get_faceB(), O.get_faceB())
