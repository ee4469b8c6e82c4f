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


# ctypes mirrors of the header structs (dragon_b200/_lib.py) against the C
# compiler's layout of the structs themselves.
STRUCTS = [("DragonConfig", "dragon_config"), ("BCDesc", "dragon_bc_desc"), ("StepStatus", "dragon_step_status"),
           ("AdvanceStats", "dragon_advance_stats"), ("NewtonStats", "dragon_newton_stats"),
           ("BatchTuning", "dragon_batch_tuning"), ("BatchStats", "dragon_batch_stats")]


def test_ctypes_structs_match_the_c_layout(tmp_path):
    import subprocess

    from dragon_b200 import _lib
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dragon_gpu.h"', '#include "dragon_learned.h"',
             '#include "dragon_batch.h"', 'int main(void) {']
    for py, c in STRUCTS:
        lines.append(f'    printf("{c} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'    printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ['    return 0;', '}']
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for py, c in STRUCTS:
        cls = getattr(_lib, py)
        assert got[(c, "size")] == ctypes.sizeof(cls), c
        for name, _ in cls._fields_:
            assert got[(c, name)] == getattr(cls, name).offset, (c, name)
