"""Learned star-pressure guess for the exact Riemann solver (include/dragon_learned.h).

The reference starts the exact solver's Newton iteration from (pL + pR) / 2
(DRAGON/Hydro/Riemann/Exact.cpp:47; the guess is already a parameter of
Riemann::exact, Riemann.hpp:54). Here a 6 -> 32 -> 32 -> 1 network, trained on
the GPU by the library's own forward / backward kernels on converged solves
logged by the plain solver, predicts ln(p* / p_analytic); grids configured
with exact_guess = GUESS_LEARNED start Newton from it, keep the analytic guess
as fallback and judge, and still iterate to ExactRiemann_Tolerance.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .grid import GUESS_MEAN, LIMITER_MC, RIEMANN_EXACT, Config, Grid3D

PARAMS = 1328
WEIGHTS = 1313
INPUTS, HIDDEN = 6, 32
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 0, 192, 224, 1248, 1280, 1312
OFF_XMEAN, OFF_XSTD, OFF_TMEAN, OFF_TSTD, OFF_GATE = 1313, 1319, 1325, 1326, 1327

_fp = _lib.c_float_p
_dp = _lib.c_double_p


class Network:
    """A dragon_mlp handle: parameters, training set and optimiser state on the GPU."""

    def __init__(self, seed: int = 0):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.dragon_gpu_mlp_create(int(seed), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dragon_gpu_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters --------------------------------------------------------
    @property
    def params(self) -> np.ndarray:
        p = np.zeros(PARAMS, dtype=np.float32)
        _lib.check(self._lib.dragon_gpu_mlp_save(self._h, p.ctypes.data_as(_fp), PARAMS))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (PARAMS,):
            raise ValueError(f"expected {PARAMS} parameters")
        _lib.check(self._lib.dragon_gpu_mlp_load(self._h, p.ctypes.data_as(_fp), PARAMS))

    @property
    def gate(self) -> float:
        return float(self.params[OFF_GATE])

    @gate.setter
    def gate(self, g: float) -> None:
        _lib.check(self._lib.dragon_gpu_mlp_set_gate(self._h, float(g)))

    # -- training set ------------------------------------------------------
    def add_samples(self, rows: np.ndarray) -> None:
        """Appends log rows (n x 8: rhoL, vxL, pL, rhoR, vxR, pR, p*, iterations)."""
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        if rows.ndim != 2 or rows.shape[1] != 8:
            raise ValueError("rows must be n x 8")
        _lib.check(self._lib.dragon_gpu_mlp_add_samples(self._h, rows.ctypes.data, rows.shape[0], 0))

    def add_samples_from_grid(self, grid) -> int:
        """Appends a grid's stored Newton log straight from device memory; returns the count."""
        rows_p = ctypes.c_void_p()
        n = ctypes.c_longlong()
        _lib.check(self._lib.dragon_gpu_newton_log_device(grid._h, ctypes.byref(rows_p), ctypes.byref(n)))
        if n.value:
            _lib.check(self._lib.dragon_gpu_mlp_add_samples(self._h, rows_p, n.value, 1))
        return n.value

    @property
    def sample_count(self) -> int:
        return int(self._lib.dragon_gpu_mlp_sample_count(self._h))

    def clear_samples(self) -> None:
        _lib.check(self._lib.dragon_gpu_mlp_clear_samples(self._h))

    def fit_normalisation(self) -> None:
        _lib.check(self._lib.dragon_gpu_mlp_fit_normalisation(self._h))

    def features(self, first: int, n: int):
        x = np.zeros((n, INPUTS), dtype=np.float32)
        t = np.zeros(n, dtype=np.float32)
        _lib.check(self._lib.dragon_gpu_mlp_features(self._h, first, n, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp)))
        return x, t

    # -- training ----------------------------------------------------------
    def gradient(self, first: int, n: int):
        """(gradient of the WEIGHTS weights, loss) over samples [first, first + n)."""
        g = np.zeros(WEIGHTS, dtype=np.float32)
        loss = ctypes.c_float()
        _lib.check(self._lib.dragon_gpu_mlp_gradient(self._h, first, n, g.ctypes.data_as(_fp), ctypes.byref(loss)))
        return g, float(loss.value)

    def train(self, steps: int, batch: int = 8192, lr: float = 1e-3) -> float:
        loss = ctypes.c_float()
        _lib.check(self._lib.dragon_gpu_mlp_train(self._h, int(steps), int(batch), float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def evaluate(self, first: int, n: int) -> float:
        """RMS error of the predicted ln(p* / p_analytic) over samples [first, first + n)."""
        r = ctypes.c_float()
        _lib.check(self._lib.dragon_gpu_mlp_evaluate(self._h, first, n, ctypes.byref(r)))
        return float(r.value)

    # -- inference ---------------------------------------------------------
    def guess(self, pairs: np.ndarray):
        """Tensor-core inference on faces (n x 6: rhoL, vxL, pL, rhoR, vxR, pR):
        (learned guess, analytic guess, raw network output)."""
        pairs = np.ascontiguousarray(pairs, dtype=np.float64)
        n = pairs.shape[0]
        g = np.zeros(n)
        a = np.zeros(n)
        y = np.zeros(n, dtype=np.float32)
        _lib.check(self._lib.dragon_gpu_mlp_guess(self._h, pairs.ctypes.data_as(_dp), n, g.ctypes.data_as(_dp),
                                                  a.ctypes.data_as(_dp), y.ctypes.data_as(_fp)))
        return g, a, y


def blast_grid(n: int, p_in: float, config: Config, ghosts: int = 2):
    """The 3D blast on [-0.5, 0.5]^3: rho = 1, p = 0.1 outside, p_in inside r < 0.1, v = 0, Outflow."""
    from .problems import blast_3d
    w, d = blast_3d(n, ghosts=ghosts, p_in=p_in)
    G = Grid3D(n, n, n, d, d, d, ghosts=ghosts, config=config)
    G.w[...] = w
    return G


def collect_blast_samples(net: Network, runs: int = 8, n: int = 128, steps: int = 20, seed: int = 2024,
                          p_range=(10.0, 1e4), stride: int = 32, capacity: int = 1 << 21) -> dict:
    """Seeded 3D blast runs with the plain solver (mean guess, reference cap);
    every stride-th converged Newton solve goes into net's training set.
    Inner pressures are log-uniform in p_range. A run whose log filled up
    (capacity rows before its last step) kept only its early solves; the
    result counts such runs in "saturated_runs"."""
    rng = np.random.default_rng(seed)
    cfg = Config(riemann=RIEMANN_EXACT, limiter=LIMITER_MC, exact_guess=GUESS_MEAN)
    p_ins = np.exp(rng.uniform(np.log(p_range[0]), np.log(p_range[1]), runs))
    added = saturated = solves = 0
    for p_in in p_ins:
        G = blast_grid(n, float(p_in), cfg)
        G.newton_log(capacity, stride)
        G.advance_steps(steps)
        solves += G.newton_stats()["exact_calls"]
        got = net.add_samples_from_grid(G)
        saturated += got >= capacity
        added += got
        G.close()
    return {"runs": runs, "n": n, "steps": steps, "p_in": p_ins.tolist(), "samples": added, "stride": stride,
            "solves": solves, "saturated_runs": int(saturated)}


def c4_training_set(net: Network, runs: int = 6, seed: int = 2024) -> dict:
    """The training recipe of the 3D blast configuration: seeded 128^3 blasts
    (MC, outflow, exact solver with the reference's mean guess and cap) with the
    inner pressure log-uniform in [10, 1e4], 16 steps each, every second
    converged solve logged (~1e7 samples over six runs; the log holds 2^23
    rows per run, more than the ~8e6 the strongest blasts log)."""
    return collect_blast_samples(net, runs=runs, n=128, steps=16, seed=seed, p_range=(10.0, 1e4), stride=2,
                                 capacity=1 << 23)


def fit(net: Network, steps: int = 6000, batch: int = 8192, lr: float = 3e-3, gate_factor: float = 1.0) -> dict:
    """Normalises, trains with a stepped learning rate, and sets the gate to
    gate_factor x the RMS error of the predicted ln(p* / p_analytic) over the
    training set."""
    net.fit_normalisation()
    n = net.sample_count
    losses = []
    for frac, scale in ((0.5, 1.0), (0.3, 0.3), (0.2, 0.1)):
        losses.append(net.train(max(1, int(steps * frac)), batch, lr * scale))
    rmse = net.evaluate(0, n)
    net.gate = gate_factor * rmse
    return {"samples": n, "losses": losses, "rmse_log": rmse, "gate": net.gate}
