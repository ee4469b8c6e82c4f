"""The C-ABI library loads and exports every symbol include/dragon_gpu.h,
include/dragon_learned.h and include/dragon_batch.h declare (no compute
calls: this runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("dragon_gpu.h", "dragon_learned.h", "dragon_batch.h")]


def declared_symbols():
    txt = "".join(open(h).read() for h in HEADERS)
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dragon_gpu_\w+)\s*\(", txt)))


def test_header_declares_api():
    syms = declared_symbols()
    for must in ("dragon_gpu_grid_create", "dragon_gpu_advance", "dragon_gpu_unsplit_step", "dragon_gpu_cfl_time",
                 "dragon_gpu_set_boundary", "dragon_gpu_upload_prim", "dragon_gpu_download_prim",
                 "dragon_gpu_mlp_train", "dragon_gpu_mlp_gradient", "dragon_gpu_newton_log_enable",
                 "dragon_gpu_batch_create", "dragon_gpu_batch_advance_steps", "dragon_gpu_batch_autotune"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from dragon_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    from dragon_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_user_ghostfill_detection():
    import dragon_b200 as dg

    class Jet(dg.GhostFill):
        def apply(self, grid):
            pass

    assert Jet("X-").is_custom and not dg.Outflow().is_custom and not dg.Periodic("Y").is_custom
    assert (dg.Periodic("Y") + Jet("X-")).has_custom()
    assert not (dg.Periodic("Y") + dg.Reflective("X")).has_custom()
