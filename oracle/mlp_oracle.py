"""CPU oracle of the learned star-pressure guess (numpy).

TEST INFRASTRUCTURE ONLY: the checker for the library's training and
inference kernels (dragon_b200/csrc/learned.cu, mlp.cuh). Only tests/ may
use it.

Restated here:
  * the face features and the network target ln(p* / p_analytic);
  * the adaptive analytic star-pressure guess (Toro, Riemann Solvers and
    Numerical Methods for Fluid Dynamics, 3rd ed., sec. 9.5.1, Q = 2) that the
    exact solver (DRAGON/Hydro/Riemann/Exact.cpp:47-84) is seeded with;
  * the 6 -> 32 -> 32 -> 1 ReLU network with BF16 rounding of the inputs,
    weights and hidden activations, its mean-square loss and the gradient
    with each rounding taken as the identity (straight-through), in float64;
  * the Newton iteration of Riemann::exact_StarP (Exact.cpp:71-84) vectorised,
    to count iterations from any guess.
The parameter layout is the one include/dragon_learned.h documents.
"""
from __future__ import annotations

import numpy as np

GAMMA = 5.0 / 3.0
IN, H = 6, 32
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 0, 192, 224, 1248, 1280, 1312
OFF_XMEAN, OFF_XSTD, OFF_TMEAN, OFF_TSTD, OFF_GATE = 1313, 1319, 1325, 1326, 1327
WEIGHTS, PARAMS = 1313, 1328


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def features(rows: np.ndarray) -> np.ndarray:
    """Face features from rows (rhoL, vxL, pL, rhoR, vxR, pR, ...), float32 like the device."""
    f = np.float32
    rl, ul, pl = rows[:, 0].astype(f), rows[:, 1], rows[:, 2].astype(f)
    rr, ur, pr = rows[:, 3].astype(f), rows[:, 4], rows[:, 5].astype(f)
    lr = np.log(rl / rr)
    lp = np.log(pl / pr)
    rbar = np.sqrt(rl) * np.sqrt(rr)
    pbar = np.sqrt(pl) * np.sqrt(pr)
    cbar = np.sqrt(f(GAMMA) * pbar / rbar)
    du = (ur - ul).astype(f) / cbar
    h = f(0.5)
    return np.stack([h * lr, h * lp, -h * du, -h * lr, -h * lp, h * du], axis=1).astype(f)


def analytic_guess(rows: np.ndarray) -> np.ndarray:
    """Adaptive PVRS / two-rarefaction / two-shock guess; the mean where unusable."""
    g = GAMMA
    rl, ul, pl, rr, ur, pr = (rows[:, i] for i in range(6))
    al, ar = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    du = ur - ul
    mean = (pl + pr) / 2
    ppv = np.maximum(0.0, mean - 0.125 * du * (rl + rr) * (al + ar))
    pmin, pmax = np.minimum(pl, pr), np.maximum(pl, pr)
    z = (g - 1) / (2 * g)
    with np.errstate(invalid="ignore", divide="ignore"):
        ptr = ((al + ar - (g - 1) / 2 * du) / (al / pl ** z + ar / pr ** z)) ** (2 * g / (g - 1))
        gl = np.sqrt(2 / (g + 1) / rl / (ppv + (g - 1) / (g + 1) * pl))
        gr = np.sqrt(2 / (g + 1) / rr / (ppv + (g - 1) / (g + 1) * pr))
        pts = (gl * pl + gr * pr - du) / (gl + gr)
    out = np.where((pmax / pmin <= 2) & (pmin <= ppv) & (ppv <= pmax), ppv, np.where(ppv < pmin, ptr, pts))
    return np.where((out > 0) & np.isfinite(out), out, mean)


def loggable(rows: np.ndarray) -> np.ndarray:
    """Rows of the C oracle's exact-solver log that the device log keeps:
    converged, positive finite p*, positive finite densities and pressures,
    finite velocities."""
    with np.errstate(invalid="ignore"):
        ok = (rows[:, 7] > 0) & np.isfinite(rows[:, :7]).all(axis=1) & (rows[:, 6] > 0)
        return ok & (rows[:, 0] > 0) & (rows[:, 2] > 0) & (rows[:, 3] > 0) & (rows[:, 5] > 0)


def targets(rows: np.ndarray) -> np.ndarray:
    return np.log(rows[:, 6] / analytic_guess(rows)).astype(np.float32)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p: np.ndarray, x: np.ndarray, quantise: bool = True):
    """Network output (normalised target units) for raw features x; returns
    (y, cache). quantise=False drops the BF16 rounding (for finite differences)."""
    if quantise:
        p = np.asarray(p, dtype=np.float32)
        q = bf16
    else:
        p = np.asarray(p, dtype=np.float64)
        q = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    W1, b1, W2, b2, W3, b3 = unpack(p)
    mean, std = p[OFF_XMEAN:OFF_XSTD], p[OFF_XSTD:OFF_TMEAN]
    xn = (x - mean) / std
    xq = q(xn.astype(np.float32) if quantise else xn).astype(np.float64)
    W1q, W2q, W3q = (q(w).astype(np.float64) for w in (W1, W2, W3))
    z1 = xq @ W1q.T + b1
    h1 = q(np.maximum(z1, 0).astype(np.float32) if quantise else np.maximum(z1, 0)).astype(np.float64)
    z2 = h1 @ W2q.T + b2
    h2 = q(np.maximum(z2, 0).astype(np.float32) if quantise else np.maximum(z2, 0)).astype(np.float64)
    y = h2 @ W3q + float(b3)
    return y, (xq, z1, h1, z2, h2, W2q, W3q)


def loss_and_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, quantise: bool = True):
    """0.5 mean((y - t_n)^2) and its gradient w.r.t. the WEIGHTS weights."""
    tn = (t.astype(np.float64) - p[OFF_TMEAN]) / p[OFF_TSTD]
    y, (xq, z1, h1, z2, h2, W2q, W3q) = forward(p, x, quantise)
    n = len(t)
    e = y - tn
    dy = e / n
    dz2 = (dy[:, None] * W3q[None, :]) * (z2 > 0)
    dz1 = (dz2 @ W2q) * (z1 > 0)
    g = np.zeros(WEIGHTS)
    g[OFF_W1:OFF_B1] = (dz1.T @ xq).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    return 0.5 * float(np.mean(e * e)), g


def guess(p: np.ndarray, rows: np.ndarray):
    """Learned guess as the solver uses it: the analytic guess unless the
    predicted |ln(p*/p_analytic)| exceeds the gate."""
    y, _ = forward(p, features(rows))
    r = y * p[OFF_TSTD] + p[OFF_TMEAN]
    a = analytic_guess(rows)
    return np.where(np.abs(r) <= p[OFF_GATE], a, a * np.exp(r)), a, y


def _f(p, rho, p0):
    g = GAMMA
    A, B = 2 / ((g + 1) * rho), (g - 1) / (g + 1) * p0
    a = np.sqrt(g * p0 / rho)
    with np.errstate(invalid="ignore"):
        ra = 2 / (g - 1) * a * ((p / p0) ** ((g - 1) / (2 * g)) - 1)
        sh = (p - p0) * np.sqrt(A / (B + p))
    return np.where(p > p0, sh, ra)


def _df(p, rho, p0):
    g = GAMMA
    A, B = 2 / ((g + 1) * rho), (g - 1) / (g + 1) * p0
    a = np.sqrt(g * p0 / rho)
    with np.errstate(invalid="ignore"):
        ra = (p / p0) ** (-(g + 1) / (2 * g)) / (rho * a)
        sh = np.sqrt(A / (p + B)) * (1 - (p - p0) / (2 * (B + p)))
    return np.where(p > p0, sh, ra)


def newton(rows: np.ndarray, p0: np.ndarray, cap: int = 64, tol: float = 1e-12):
    """Star pressure and iteration count of exact_StarP from guesses p0."""
    rl, ul, pl, rr, ur, pr = (rows[:, i] for i in range(6))
    p = np.array(p0, dtype=np.float64)
    n = np.zeros(len(p), dtype=np.int64)
    act = np.ones(len(p), dtype=bool)
    for _ in range(cap):
        fp = _f(p, rl, pl) + _f(p, rr, pr) + ur - ul
        d = np.minimum(fp / (_df(p, rl, pl) + _df(p, rr, pr)), 0.8 * p)
        pn = p - d
        cha = np.abs(d / (pn + d / 2))
        p = np.where(act, pn, p)
        n += act
        act &= cha > tol
        if not act.any():
            break
    return p, n
