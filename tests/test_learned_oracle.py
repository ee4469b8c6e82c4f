"""CPU checks of the learned star-pressure guess: the numpy oracle is pinned
(BF16 rounding against torch, backward against finite differences, the
vectorised Newton against the C oracle's exact solver), and the device guess
policy, compiled for the host, keeps the reference's fluxes: the mean guess is
bit-identical to the plain exact solver, other guesses converge to the same
star state, unusable learned guesses fall back and capped ones are rerun."""
import ctypes

import numpy as np
import pytest
import torch

from conftest import build_hostcheck
from oracle import mlp_oracle as mo
from oracle import port

_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def hc():
    L = ctypes.CDLL(build_hostcheck("hydro"))
    L.hc_analytic_guess.restype = ctypes.c_double
    L.hc_analytic_guess.argtypes = [_dp, _dp]
    L.hc_exact_flux_guess.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.POINTER(ctypes.c_int)]
    L.hc_riemann_flux.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


def prim(rho, u, p):
    return np.array([rho, p, u, 0.0, 0.0])


def random_pairs(n, seed, strong=True):
    """Face pairs (rhoL, vxL, pL, rhoR, vxR, pR) with converging flow (Newton branch)."""
    rng = np.random.default_rng(seed)
    rl = 10 ** rng.uniform(-1, 1, n)
    rr = 10 ** rng.uniform(-1, 1, n)
    span = 3 if strong else 0.3
    pl = 10 ** rng.uniform(-span, span, n)
    pr = 10 ** rng.uniform(-span, span, n)
    ul = rng.uniform(0, 2, n)
    ur = rng.uniform(-2, 0, n)
    return np.stack([rl, ul, pl, rr, ur, pr], axis=1)


def exact_guess_flux(hc, row, mode, cap, learned=None):
    l, r = prim(*row[:3]), prim(*row[3:6])
    out = np.zeros(5)
    st = (ctypes.c_int * 6)()
    lp = None if learned is None else _p(np.array(learned, dtype=np.float64))
    hc.hc_exact_flux_guess(_p(l), _p(r), mode, cap, lp, _p(out), st)
    return out, dict(zip(["iters", "calls", "trrs", "cap_hits", "rejects", "reruns"], list(st)))


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(5000).astype(np.float32) * 10 ** rng.uniform(-6, 6, 5000).astype(np.float32),
                        np.float32([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -0.0, 0.0, 65504.0])])
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(mo.bf16(x), ref)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = np.zeros(mo.PARAMS, dtype=np.float64)
    p[:mo.WEIGHTS] = rng.standard_normal(mo.WEIGHTS) * 0.3
    p[mo.OFF_XSTD:mo.OFF_TMEAN] = 1.0
    p[mo.OFF_TSTD] = 1.0
    x = rng.standard_normal((64, 6)).astype(np.float32)
    t = rng.standard_normal(64).astype(np.float32)
    _, g = mo.loss_and_grad(p, x, t, quantise=False)
    h = 1e-6
    for k in rng.choice(mo.WEIGHTS, 60, replace=False).tolist() + [mo.OFF_B3]:
        a, b = p.copy(), p.copy()
        a[k] += h
        b[k] -= h
        fd = (mo.loss_and_grad(a, x, t, quantise=False)[0] - mo.loss_and_grad(b, x, t, quantise=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_analytic_guess_matches_device_function(hc):
    rows = np.concatenate([random_pairs(400, 2), random_pairs(400, 3, strong=False)])
    got = np.array([hc.hc_analytic_guess(_p(prim(*r[:3])), _p(prim(*r[3:6]))) for r in rows])
    np.testing.assert_allclose(got, mo.analytic_guess(rows), rtol=1e-13)


def test_vectorised_newton_matches_c_oracle():
    """The oracle's exact solver logs (p*, iterations) of a seeded 3D blast;
    the vectorised restatement reproduces both from the mean guess, cap 6."""
    from dragon_b200 import problems
    n = 10
    w, d = problems.blast_3d(n, ghosts=2, p_in=100.0)
    P = port.PortGrid(dim=3, n=(n, n, n), d=(d, d, d), ghosts=2, riemann=0, limiter=1, exact_max_iters=6)
    P.set_prim(w)
    with port.ExactLog(1 << 18) as log:
        for _ in range(3):
            P.step_cfl()
    rows = log.rows
    assert len(rows) > 1000
    ps, it = mo.newton(rows, (rows[:, 2] + rows[:, 5]) / 2, cap=6)
    np.testing.assert_allclose(ps, rows[:, 6], rtol=1e-14)
    np.testing.assert_array_equal(it, np.abs(rows[:, 7]))
    assert np.all((rows[:, 7] < 0) == (it == 6)) or np.all(rows[:, 7][it < 6] > 0)


def test_mean_guess_is_the_plain_exact_solver(hc):
    for row in random_pairs(50, 4):
        l, r = prim(*row[:3]), prim(*row[3:6])
        ref = np.zeros(5)
        hc.hc_riemann_flux(0, _p(l), _p(r), 0.0, 0, _p(ref))
        got, st = exact_guess_flux(hc, row, 0, 6)
        np.testing.assert_array_equal(got, ref)


def test_guesses_converge_to_the_same_flux(hc):
    """With the cap lifted every guess reaches the tolerance; fluxes agree to
    roundoff and the analytic guess needs fewer iterations on strong shocks."""
    it_mean = it_an = 0
    for row in random_pairs(200, 5):
        f0, s0 = exact_guess_flux(hc, row, 0, 64)
        f1, s1 = exact_guess_flux(hc, row, 1, 64)
        assert s0["cap_hits"] == 0 and s1["cap_hits"] == 0
        np.testing.assert_allclose(f1, f0, rtol=1e-11, atol=1e-13 * np.abs(f0).max())
        it_mean += s0["iters"]
        it_an += s1["iters"]
    assert it_an < 0.9 * it_mean, (it_an, it_mean)


def test_unusable_learned_guess_falls_back(hc):
    row = random_pairs(1, 6)[0]
    a = mo.analytic_guess(row[None])[0]
    f_an, _ = exact_guess_flux(hc, row, 1, 64)
    for bad in (np.nan, -1.0, 0.0, np.inf):
        f, st = exact_guess_flux(hc, row, 2, 64, learned=[bad, a])
        assert st["rejects"] == 1 and st["reruns"] == 0
        np.testing.assert_array_equal(f, f_an)


def test_capped_learned_start_is_rerun_from_the_analytic_guess(hc):
    """A learned start so far off that Newton hits the cap is judged: the
    solve reruns from the analytic guess, which converges."""
    row = np.array([1.0, 1.0, 1000.0, 1.0, -1.0, 0.01])
    a = mo.analytic_guess(row[None])[0]
    f_an, s_an = exact_guess_flux(hc, row, 1, 8)
    assert s_an["cap_hits"] == 0
    f, st = exact_guess_flux(hc, row, 2, 8, learned=[a * 1e-12, a])
    assert st["reruns"] == 1 and st["cap_hits"] == 1
    np.testing.assert_array_equal(f, f_an)


def test_oracle_learned_guess_gate():
    """Predictions inside the gate keep the analytic guess exactly."""
    rng = np.random.default_rng(7)
    p = np.zeros(mo.PARAMS, dtype=np.float32)
    p[:mo.WEIGHTS] = rng.standard_normal(mo.WEIGHTS).astype(np.float32) * 0.1
    p[mo.OFF_XSTD:mo.OFF_TMEAN] = 1.0
    p[mo.OFF_TSTD] = 1.0
    rows = random_pairs(300, 8)
    y, _ = mo.forward(p, mo.features(rows))
    p[mo.OFF_GATE] = np.float32(np.median(np.abs(y)))
    g, a, y2 = mo.guess(p, rows)
    inside = np.abs(y2) <= p[mo.OFF_GATE]
    assert inside.any() and (~inside).any()
    np.testing.assert_array_equal(g[inside], a[inside])
    np.testing.assert_allclose(g[~inside], a[~inside] * np.exp(y2[~inside]), rtol=1e-12)
