"""dragon_b200: B200-native unsplit Godunov update for DRAGON grids.

The host-side mirror of DRAGON's Grid / Boundary API over the C ABI declared
in include/dragon_gpu.h (library: dragon_b200/libdragon_gpu.so).
"""
from .boundary import (X, Y, Z, BoundaryList, DeviceGhostFill, Fixed, GhostFill, Ignore, Outflow, Periodic, Reflective,
                       X_negative, X_positive, Y_negative, Y_positive, Z_negative, Z_positive, face_mask)
from .grid import (CFL_ADD, CFL_MAX, CT_CONSV_BETA_GATED, CT_CONSV_THERMAL, CT_CONSV_TOTAL_E, GUESS_ANALYTIC,
                   GUESS_LEARNED, GUESS_MEAN, GUESS_PERFECT, LIMITER_MC,
                   LIMITER_MINMOD, LIMITER_SUPERBEE, LIMITER_VANALBADA, LIMITER_VANLEER, PREC_FP64, PREC_MIXED,
                   RIEMANN_EXACT, RIEMANN_HLL, RIEMANN_HLLC, RIEMANN_HLLD, RIEMANN_HLLE, RIEMANN_HLLX, RIEMANN_ROE,
                   AdvanceResult, Config, Grid1D, Grid2D, Grid3D, StepFailed)
from . import hoard  # noqa: E402  (DRAGONHOARD: output and restart from device buffers)

__all__ = [n for n in dir() if not n.startswith("_")]
