"""The device path's per-cell and per-face functions, compiled for the CPU
(tests/hostcheck), agree bit for bit with the reference's FluidElement, TVD
and Riemann code on random states. The CUDA kernels call these same functions;
this catches operand-order slips before any GPU run. The exact solver's pow
is glibc's on both sides here (on the GPU it is CUDA's, within 2 ulp)."""
import ctypes

import numpy as np
import pytest

from conftest import build_hostcheck

D = ctypes.POINTER(ctypes.c_double)


def P(a):
    return a.ctypes.data_as(D)


def libs(mhd):
    from oracle import refgrid
    variant = "mhd" if mhd else "hydro"
    if not refgrid.available(variant):
        pytest.skip("reference oracle not built")
    R = refgrid.load(variant)
    R.ref_prim_to_cons.argtypes = [D, D]
    R.ref_cons_to_prim.argtypes = [D, D]
    R.ref_prim_flux.argtypes = [D, D]
    H = ctypes.CDLL(build_hostcheck(variant))
    H.hc_limiter.restype = ctypes.c_double
    H.hc_limiter.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    H.hc_muscl.argtypes = [ctypes.c_int, D, D, D, ctypes.c_double, D, D, D]
    H.hc_riemann_flux.argtypes = [ctypes.c_int, D, D, ctypes.c_double, ctypes.c_int, D]
    H.hc_prim_to_cons.argtypes = [D, D]
    H.hc_cons_to_prim.argtypes = [D, D]
    H.hc_prim_flux.argtypes = [D, D]
    return R, H


def random_state(rng, mhd, nf):
    w = np.zeros(nf)
    w[0] = 10 ** rng.uniform(-2, 1)
    w[1] = 10 ** rng.uniform(-2, 2)
    w[2:5] = rng.uniform(-2, 2, 3) * rng.choice([0.0, 0.1, 1.0, 4.0])
    if mhd:
        w[5:8] = rng.uniform(-1, 1, 3) * rng.choice([0.0, 0.05, 1.0, 5.0])
        if rng.random() < 0.1:
            w[5] = 0.0
    return w


@pytest.mark.parametrize("mhd", [False, True])
def test_conversions_and_flux_bitwise(mhd):
    R, H = libs(mhd)
    nf = 8 if mhd else 5
    rng = np.random.default_rng(7)
    for _ in range(3000):
        a = random_state(rng, mhd, nf)
        o1, o2 = np.zeros(nf), np.zeros(nf)
        R.ref_prim_to_cons(P(a), P(o1))
        H.hc_prim_to_cons(P(a), P(o2))
        assert np.array_equal(o1, o2, equal_nan=True)
        u = o1.copy()
        R.ref_cons_to_prim(P(u), P(o1))
        H.hc_cons_to_prim(P(u), P(o2))
        assert np.array_equal(o1, o2, equal_nan=True)
        R.ref_prim_flux(P(a), P(o1))
        H.hc_prim_flux(P(a), P(o2))
        assert np.array_equal(o1, o2, equal_nan=True)


def test_limiters_bitwise():
    R, H = libs(False)
    rng = np.random.default_rng(3)
    out = ctypes.c_double()
    for _ in range(4000):
        a, b = rng.normal(size=2) * 10 ** rng.uniform(-3, 3, 2)
        if rng.random() < 0.1:
            b = a
        for k in range(5):
            R.ref_limiter(k, a, b, ctypes.byref(out))
            assert out.value == H.hc_limiter(k, a, b) or (np.isnan(out.value) and np.isnan(H.hc_limiter(k, a, b)))


@pytest.mark.parametrize("mhd", [False, True])
def test_muscl_bitwise(mhd):
    R, H = libs(mhd)
    nf = 8 if mhd else 5
    rng = np.random.default_rng(11)
    for it in range(3000):
        a, b, c = (random_state(rng, mhd, nf) for _ in range(3))
        lim = it % 5
        dB = rng.uniform(-0.2, 0.2, 3) if mhd else np.zeros(3)
        dt = rng.uniform(0, 0.4)
        R.ref_config(5, lim, 1, 2, 1)
        L1, R1, L2, R2 = (np.zeros(nf) for _ in range(4))
        R.ref_muscl(P(a), P(b), P(c), dt, P(dB), P(L1), P(R1))
        H.hc_muscl(lim, P(a), P(b), P(c), dt, P(dB), P(L2), P(R2))
        assert np.array_equal(L1, L2, equal_nan=True) and np.array_equal(R1, R2, equal_nan=True)


@pytest.mark.parametrize("mhd", [False, True])
def test_riemann_dispatch_bitwise(mhd):
    """Each solver through the flux_X/Y/Z dispatch, with the hydro
    verify-and-fallback pivot active (dt/dx > 0)."""
    R, H = libs(mhd)
    nf = 8 if mhd else 5
    rng = np.random.default_rng(5)
    solvers = [5, 1, 4] if mhd else [5, 1, 4, 6, 0]
    msg = ctypes.create_string_buffer(128)
    for it in range(2500):
        a, b = random_state(rng, mhd, nf), random_state(rng, mhd, nf)
        dt = rng.choice([0.0, rng.uniform(0, 0.3), rng.uniform(0, 5.0)])
        for s in solvers:
            ax = int(rng.integers(0, 3))
            R.ref_config(s, 1, 1, 2, 1)
            o1, o2 = np.zeros(nf), np.zeros(nf)
            rc1 = R.ref_riemann_flux(-1, P(a), P(b), dt, ax, P(o1), msg, 128)
            rc2 = H.hc_riemann_flux(s, P(a), P(b), dt, ax, P(o2))
            assert rc1 == rc2, (s, a, b, dt)
            if rc1 == 0:
                assert np.array_equal(o1, o2, equal_nan=True), (s, ax, a, b, o1, o2)
