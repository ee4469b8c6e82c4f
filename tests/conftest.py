import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HOSTCHECK = os.path.join(ROOT, "tests", "hostcheck")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the device path")


def build_hostcheck(variant: str) -> str:
    """Builds tests/hostcheck/libhostcheck_{hydro,mhd}.so (CPU build of the device math)."""
    out = os.path.join(HOSTCHECK, f"libhostcheck_{variant}.so")
    src = os.path.join(HOSTCHECK, "hostcheck.cpp")
    deps = [src] + [os.path.join(ROOT, "dragon_b200", "csrc", f)
                    for f in ("fluid.cuh", "recon.cuh", "riemann.cuh", "frame.cuh")]
    if not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", out, src]
        if variant == "mhd":
            cmd.insert(1, "-DHC_MHD")
        subprocess.run(cmd, check=True)
    return out


def build_oracle() -> None:
    """Builds the C restatement (and the reference libraries when the sources exist)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-j8"], check=True)


@pytest.fixture(scope="session")
def ref_hydro():
    from oracle import refgrid
    if not refgrid.available("hydro"):
        try:
            build_oracle()
        except Exception:
            pass
    if not refgrid.available("hydro"):
        pytest.skip("reference oracle library not built (needs the reference sources)")
    return refgrid


def cuda_ok() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
