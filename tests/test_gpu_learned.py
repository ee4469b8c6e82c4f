"""GPU checks of the learned star-pressure guess: the Newton sample log
against the oracle's, the training gradient and the tensor-core inference
against the numpy oracle, the fallback and gate paths bit for bit against the
analytic guess, and what a trained network gains over the method without it
(Newton iterations per solve on a 3D blast, with identical converged states)."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

import dragon_b200 as dg  # noqa: E402
from dragon_b200 import learned, problems  # noqa: E402
from oracle import mlp_oracle as mo  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not cuda_ok():
        pytest.fail("CUDA device required for -m gpu tests")


def blast_pair(n, p_in, steps, cap=6):
    """The same 3D blast on the GPU (mean guess) and the oracle, with both logs."""
    from oracle import port
    w, d = problems.blast_3d(n, ghosts=2, p_in=p_in)
    G = dg.Grid3D(n, n, n, d, d, d, ghosts=2,
                  config=dg.Config(riemann=dg.RIEMANN_EXACT, limiter=dg.LIMITER_MC, exact_max_iters=cap))
    G.w[...] = w
    G.newton_log(1 << 20, 1)
    G.advance_steps(steps)
    P = port.PortGrid(dim=3, n=(n, n, n), d=(d, d, d), ghosts=2, riemann=0, limiter=1, exact_max_iters=cap)
    P.set_prim(w)
    with port.ExactLog(1 << 20) as log:
        for _ in range(steps):
            P.step_cfl()
    return G, log.rows


def test_newton_log_matches_oracle():
    """Same solves logged (order differs: the device log is filled by atomics):
    equal counts, equal per-column value sets to roundoff, equal iteration
    histograms."""
    G, ref = blast_pair(16, 100.0, 1)
    got = G.newton_log_rows()
    conv = ref[mo.loggable(ref)]
    assert len(got) == len(conv) > 200
    st = G.newton_stats()
    assert st["log_seen"] == len(got) == st["log_stored"]
    for c in range(7):
        np.testing.assert_allclose(np.sort(got[:, c]), np.sort(conv[:, c]), rtol=1e-12, atol=1e-300)
    h_got = np.bincount(got[:, 7].astype(int), minlength=8)
    h_ref = np.bincount(conv[:, 7].astype(int), minlength=8)
    assert np.abs(h_got - h_ref).sum() <= max(2, len(got) // 1000), (h_got, h_ref)


def trained_network(seed=3, runs=3, n=40, steps=12):
    net = learned.Network(seed=seed)
    info = learned.collect_blast_samples(net, runs=runs, n=n, steps=steps, seed=seed, stride=1, capacity=1 << 21)
    assert info["samples"] > 10000
    fit = learned.fit(net, steps=2000, batch=4096, lr=3e-3)
    return net, fit


@pytest.fixture(scope="module")
def net_and_fit():
    return trained_network()


def test_features_and_targets_match_oracle():
    _, rows = blast_pair(10, 300.0, 2)
    rows = rows[mo.loggable(rows)]
    net = learned.Network(seed=1)
    net.add_samples(rows)
    x, t = net.features(0, len(rows))
    np.testing.assert_allclose(x, mo.features(rows), rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(t, mo.targets(rows), rtol=1e-5, atol=1e-6)


def test_gradient_matches_oracle(net_and_fit):
    net, _ = net_and_fit
    n = 3000
    g, loss = net.gradient(0, n)
    x, t = net.features(0, n)
    loss_o, g_o = mo.loss_and_grad(net.params, x, t)
    assert abs(loss - loss_o) <= 1e-4 * abs(loss_o) + 1e-7
    scale = np.abs(g_o).max()
    np.testing.assert_allclose(g, g_o, rtol=2e-3, atol=2e-3 * scale)


def test_untrained_gradient_matches_oracle():
    """Same check at the random initialisation (large gradients, every unit active)."""
    _, rows = blast_pair(10, 1000.0, 2)
    rows = rows[mo.loggable(rows)]
    net = learned.Network(seed=9)
    net.add_samples(rows)
    net.fit_normalisation()
    n = min(len(rows), 2048)
    g, loss = net.gradient(0, n)
    x, t = net.features(0, n)
    loss_o, g_o = mo.loss_and_grad(net.params, x, t)
    assert abs(loss - loss_o) <= 1e-4 * abs(loss_o)
    np.testing.assert_allclose(g, g_o, rtol=2e-3, atol=2e-3 * np.abs(g_o).max())


def test_tensor_core_inference_matches_oracle(net_and_fit):
    net, _ = net_and_fit
    rng = np.random.default_rng(5)
    n = 5000
    pairs = np.stack([10 ** rng.uniform(-1, 1, n), rng.uniform(0, 1, n), 10 ** rng.uniform(-2, 2, n),
                      10 ** rng.uniform(-1, 1, n), rng.uniform(-1, 0, n), 10 ** rng.uniform(-2, 2, n)], axis=1)
    g, a, y = net.guess(pairs)
    p = net.params
    y_o, _ = mo.forward(p, mo.features(pairs))
    np.testing.assert_allclose(a, mo.analytic_guess(pairs), rtol=1e-13)
    err = np.abs(y - y_o)
    assert np.quantile(err, 0.99) <= 1e-3 * (1 + np.abs(y_o).max()), np.quantile(err, [0.5, 0.99, 1.0])
    assert err.max() <= 3e-2 * (1 + np.abs(y_o).max())
    r = y.astype(np.float64) * p[mo.OFF_TSTD] + p[mo.OFF_TMEAN]
    expect = np.where(np.abs(r) <= p[mo.OFF_GATE], a, a * np.exp(r))
    np.testing.assert_allclose(g, expect, rtol=1e-6)


def run_blast(n, p_in, steps, guess, cap, net=None):
    w, d = problems.blast_3d(n, ghosts=2, p_in=p_in)
    G = dg.Grid3D(n, n, n, d, d, d, ghosts=2,
                  config=dg.Config(riemann=dg.RIEMANN_EXACT, limiter=dg.LIMITER_MC, exact_max_iters=cap,
                                   exact_guess=guess))
    G.w[...] = w
    if net is not None:
        G.set_network(net)
    G.advance_steps(steps)
    return G.w.copy(), G.newton_stats()


def test_learned_guess_cuts_iterations_with_identical_states(net_and_fit):
    """On an unseen blast (other inner pressure and size), cap lifted for every
    guess: the learned start needs fewer Newton iterations per solve than the
    reference's mean guess, no more than the analytic guess, and every state
    agrees with the mean-guess run to roundoff."""
    net, _ = net_and_fit
    n, p_in, steps, cap = 36, 2000.0, 8, 64
    w_mean, s_mean = run_blast(n, p_in, steps, dg.GUESS_MEAN, cap)
    w_an, s_an = run_blast(n, p_in, steps, dg.GUESS_ANALYTIC, cap)
    w_l, s_l = run_blast(n, p_in, steps, dg.GUESS_LEARNED, cap, net)
    ipc = {k: s["newton_iters"] / s["exact_calls"] for k, s in (("mean", s_mean), ("analytic", s_an), ("learned", s_l))}
    assert s_mean["cap_hits"] == s_an["cap_hits"] == s_l["cap_hits"] == 0
    assert s_l["exact_calls"] == s_mean["exact_calls"] == s_an["exact_calls"]
    assert ipc["learned"] < 0.85 * ipc["mean"], ipc
    assert ipc["learned"] <= 1.02 * ipc["analytic"], ipc
    g = 2
    for w in (w_an, w_l):
        l1 = problems.rel_l1(w[g:-g, g:-g, g:-g], w_mean[g:-g, g:-g, g:-g])
        assert np.all(l1 <= 1e-12), l1


def test_unusable_network_falls_back_to_analytic():
    net = learned.Network(seed=4)
    p = net.params
    p[mo.OFF_B3] = np.nan
    net.params = p
    n, p_in, steps, cap = 16, 500.0, 3, 64
    w_an, s_an = run_blast(n, p_in, steps, dg.GUESS_ANALYTIC, cap)
    w_l, s_l = run_blast(n, p_in, steps, dg.GUESS_LEARNED, cap, net)
    assert s_l["guess_rejects"] == s_l["exact_calls"] > 0
    np.testing.assert_array_equal(w_l, w_an)
    assert s_l["newton_iters"] == s_an["newton_iters"]


def test_wide_gate_is_the_analytic_guess(net_and_fit):
    net, _ = net_and_fit
    keep = net.gate
    try:
        net.gate = 1e9
        n, p_in, steps, cap = 16, 500.0, 3, 64
        w_an, s_an = run_blast(n, p_in, steps, dg.GUESS_ANALYTIC, cap)
        w_l, s_l = run_blast(n, p_in, steps, dg.GUESS_LEARNED, cap, net)
        np.testing.assert_array_equal(w_l, w_an)
        assert s_l["newton_iters"] == s_an["newton_iters"] and s_l["guess_rejects"] == 0
    finally:
        net.gate = keep


def test_learned_needs_a_network_and_a_3d_grid():
    with pytest.raises(dg.grid._lib.DragonGPUError):
        dg.Grid2D(8, 8, 0.1, 0.1, config=dg.Config(riemann=dg.RIEMANN_EXACT, exact_guess=dg.GUESS_LEARNED))
    w, d = problems.blast_3d(8, ghosts=2, p_in=10.0)
    G = dg.Grid3D(8, 8, 8, d, d, d, config=dg.Config(riemann=dg.RIEMANN_EXACT, exact_guess=dg.GUESS_LEARNED))
    G.w[...] = w
    with pytest.raises(dg.grid._lib.DragonGPUError):
        G.advance_steps(1)


@pytest.mark.parametrize("err_exp,max_iters_per_solve", [(0, 1.0), (6, 2.0)])
def test_perfect_guess_arm_is_the_iteration_floor(err_exp, max_iters_per_solve):
    """The measurement arm GUESS_PERFECT starts Newton from the converged star
    pressure of an uncounted first solve (or from the mean guess where that
    needs no more iterations): every counted solve then converges in one
    iteration (at most two when the start carries a 1e-6 relative error), and
    the states equal the reference mean-guess solve's to 1e-12."""
    n, steps = 32, 4
    out = {}
    for name, guess, e in (("mean", dg.GUESS_MEAN, 0), ("perfect", dg.GUESS_PERFECT, err_exp)):
        w, d = problems.blast_3d(n, ghosts=2, p_in=100.0)
        G = dg.Grid3D(n, n, n, d, d, d, ghosts=2, config=dg.Config(
            riemann=dg.RIEMANN_EXACT, limiter=dg.LIMITER_MC, exact_max_iters=64, exact_guess=guess,
            perfect_guess_err_exp=e))
        G.w[...] = w
        G.advance_steps(steps)
        out[name] = (G.w.copy(), G.newton_stats())
        G.close()
    st = out["perfect"][1]
    assert st["exact_calls"] > 1000 and st["cap_hits"] == 0
    assert st["newton_iters"] <= max_iters_per_solve * st["exact_calls"]
    assert out["mean"][1]["newton_iters"] > 1.5 * st["exact_calls"]
    l1 = problems.rel_l1(out["perfect"][0], out["mean"][0])
    assert np.all(l1 <= 1e-12), l1
