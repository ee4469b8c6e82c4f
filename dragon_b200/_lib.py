"""ctypes binding of the C ABI in include/dragon_gpu.h.

The shared library is built in-tree (dragon_b200/libdragon_gpu.so) by
``dragon_b200.build.build()``. There is no CPU fallback: importing the binding
without the library, or calling into it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdragon_gpu.so")

c_double_p = ctypes.POINTER(ctypes.c_double)


class DragonConfig(ctypes.Structure):
    """dragon_config (include/dragon_gpu.h)."""

    _fields_ = [
        ("mhd", ctypes.c_int),
        ("riemann", ctypes.c_int),
        ("limiter", ctypes.c_int),
        ("cfl", ctypes.c_int),
        ("ct_energy", ctypes.c_int),
        ("exact_max_iters", ctypes.c_int),
        ("exact_tol", ctypes.c_double),
        ("cfl_coeff", ctypes.c_double),
        ("timestep_tol", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("exact_guess", ctypes.c_int),
        ("perfect_guess_err_exp", ctypes.c_int),
        ("reserved", ctypes.c_int * 5),
    ]


class BCDesc(ctypes.Structure):
    """dragon_bc_desc."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("faces", ctypes.c_int),
        ("corners", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("state", ctypes.c_double * 8),
    ]


class StepStatus(ctypes.Structure):
    """dragon_step_status."""

    _fields_ = [
        ("code", ctypes.c_int),
        ("stage", ctypes.c_int),
        ("cell", ctypes.c_longlong),
        ("dt", ctypes.c_double),
    ]


class AdvanceStats(ctypes.Structure):
    """dragon_advance_stats."""

    _fields_ = [
        ("steps", ctypes.c_int),
        ("retries", ctypes.c_int),
        ("last_dt", ctypes.c_double),
        ("time_advanced", ctypes.c_double),
        ("pivots_exact", ctypes.c_ulonglong),
        ("hlld_to_hlle", ctypes.c_ulonglong),
        ("newton_iters", ctypes.c_ulonglong),
        ("exact_calls", ctypes.c_ulonglong),
        ("trrs", ctypes.c_ulonglong),
        ("muscl_first_order", ctypes.c_ulonglong),
        ("failure", StepStatus),
    ]


class NewtonStats(ctypes.Structure):
    """dragon_newton_stats (include/dragon_learned.h)."""

    _fields_ = [(n, ctypes.c_ulonglong) for n in (
        "exact_calls", "newton_iters", "trrs", "cap_hits", "guess_rejects", "judge_reruns", "pivots_exact",
        "log_seen", "log_stored")]


c_float_p = ctypes.POINTER(ctypes.c_float)


class BatchTuning(ctypes.Structure):
    """dragon_batch_tuning (include/dragon_batch.h)."""

    _fields_ = [("tile_1d", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("order", ctypes.c_int),
                ("graph_steps", ctypes.c_int), ("mhd_tiles", ctypes.c_int), ("wave", ctypes.c_int)]


class BatchStats(ctypes.Structure):
    """dragon_batch_stats (include/dragon_batch.h)."""

    _fields_ = [("steps", ctypes.c_int), ("retries", ctypes.c_int), ("graph_replays", ctypes.c_int),
                ("work_items", ctypes.c_longlong), ("spin_timeouts", ctypes.c_ulonglong), ("replay_ms", ctypes.c_double)]

class HoardOpts(ctypes.Structure):
    """dragon_hoard_opts."""

    _fields_ = [("write_option", ctypes.c_int), ("redundant", ctypes.c_int), ("compression", ctypes.c_int),
                ("ghosts", ctypes.c_int), ("threads", ctypes.c_int), ("reserved", ctypes.c_int * 3)]


class H5Dataset(ctypes.Structure):
    """dragon_h5_dataset."""

    _fields_ = [("path", ctypes.c_char_p), ("rank", ctypes.c_int), ("dims", ctypes.c_longlong * 3),
                ("type", ctypes.c_int), ("data", ctypes.c_void_p)]


class H5Attr(ctypes.Structure):
    """dragon_h5_attr."""

    _fields_ = [("name", ctypes.c_char_p), ("type", ctypes.c_int), ("ivalue", ctypes.c_int),
                ("dvalue", ctypes.c_double)]


# Every symbol include/dragon_gpu.h, include/dragon_learned.h and
# include/dragon_batch.h declare, with its ctypes signature.
SIGNATURES = {
    "dragon_gpu_default_config": (None, [ctypes.POINTER(DragonConfig), ctypes.c_int]),
    "dragon_gpu_grid_create": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
         ctypes.c_double, ctypes.c_int, ctypes.POINTER(DragonConfig), ctypes.POINTER(ctypes.c_void_p)],
    ),
    "dragon_gpu_grid_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_grid_info": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    ),
    "dragon_gpu_prim_count": (ctypes.c_size_t, [ctypes.c_void_p]),
    "dragon_gpu_faceB_count": (ctypes.c_size_t, [ctypes.c_void_p]),
    "dragon_gpu_upload_prim": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "dragon_gpu_download_prim": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "dragon_gpu_upload_faceB": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "dragon_gpu_download_faceB": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "dragon_gpu_set_boundary": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BCDesc), ctypes.c_int]),
    "dragon_gpu_apply_boundary": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_boundary_entries": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_apply_boundary_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "dragon_gpu_initialize_B_fields": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_cfl_time": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "dragon_gpu_unsplit_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(StepStatus)]),
    "dragon_gpu_advance": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(AdvanceStats)]),
    "dragon_gpu_advance_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(AdvanceStats)]),
    "dragon_gpu_split_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(StepStatus)]),
    "dragon_gpu_advance_split": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(AdvanceStats)]),
    "dragon_gpu_advance_steps_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dragon_gpu_advance_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "dragon_gpu_halo_size": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "dragon_gpu_halo_pack": (
        ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_int] * 5 + [ctypes.c_void_p, ctypes.c_int]),
    "dragon_gpu_halo_unpack": (
        ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_int] * 5 + [ctypes.c_void_p, ctypes.c_int]),
    "dragon_gpu_step_rollback": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "dragon_gpu_device_state": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_longlong),
         ctypes.POINTER(ctypes.c_longlong)],
    ),
    "dragon_gpu_launch_count": (ctypes.c_ulonglong, [ctypes.c_void_p]),
    "dragon_gpu_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dragon_gpu_debug_set": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "dragon_gpu_user_fill_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "dragon_gpu_user_fill_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_user_fill_log": (ctypes.c_char_p, [ctypes.c_void_p]),
    "dragon_gpu_set_user_fill": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "dragon_gpu_profile_read": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                       ctypes.c_int]),
    "dragon_gpu_cfl_time_noalloc": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p,
         ctypes.c_longlong, ctypes.c_longlong, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
         ctypes.c_double, ctypes.c_void_p, c_double_p]),
    "dragon_gpu_last_error": (ctypes.c_char_p, []),
    # dragon_learned.h
    "dragon_gpu_newton_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(NewtonStats), ctypes.c_int]),
    "dragon_gpu_newton_log_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]),
    "dragon_gpu_newton_log_read": (
        ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    "dragon_gpu_newton_log_device": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_longlong)]),
    "dragon_gpu_mlp_create": (ctypes.c_int, [ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_void_p)]),
    "dragon_gpu_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_mlp_load": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "dragon_gpu_mlp_save": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "dragon_gpu_mlp_add_samples": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]),
    "dragon_gpu_mlp_sample_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "dragon_gpu_mlp_clear_samples": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_mlp_fit_normalisation": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_mlp_features": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, c_float_p, c_float_p]),
    "dragon_gpu_mlp_gradient": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, c_float_p, c_float_p]),
    "dragon_gpu_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, c_float_p]),
    "dragon_gpu_mlp_evaluate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, c_float_p]),
    "dragon_gpu_mlp_set_gate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "dragon_gpu_mlp_guess": (
        ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_longlong, c_double_p, c_double_p, c_float_p]),
    "dragon_gpu_grid_set_mlp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    # dragon_batch.h
    "dragon_gpu_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p)]),
    "dragon_gpu_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_batch_add_instance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "dragon_gpu_batch_size": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_batch_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchTuning)]),
    "dragon_gpu_batch_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchTuning)]),
    "dragon_gpu_batch_autotune": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(BatchTuning), ctypes.POINTER(ctypes.c_double)]),
    "dragon_gpu_batch_advance_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(BatchStats)]),
    "dragon_gpu_set_origin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "dragon_gpu_hoard_default_opts": (None, [ctypes.POINTER(HoardOpts)]),
    "dragon_gpu_hoard_write": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(HoardOpts)]),
    "dragon_gpu_hoard_write_async": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(HoardOpts)]),
    "dragon_gpu_hoard_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "dragon_gpu_hoard_load": (
        ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, c_double_p, ctypes.POINTER(ctypes.c_int)]),
    "dragon_hoard_write_host": (
        ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                       c_double_p, ctypes.c_double, ctypes.c_int, c_double_p, c_double_p, ctypes.POINTER(HoardOpts)]),
    "dragon_hoard_load_host": (
        ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                       c_double_p, c_double_p, c_double_p, ctypes.POINTER(ctypes.c_int), c_double_p]),
    "dragon_h5_write": (
        ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(H5Attr), ctypes.c_int, ctypes.POINTER(H5Dataset), ctypes.c_int,
                       ctypes.c_int, ctypes.c_int]),
    "dragon_h5_read_attr": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, c_double_p]),
    "dragon_h5_dataset_shape": (
        ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]),
    "dragon_h5_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, c_double_p, ctypes.c_longlong]),
}

_lib = None


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads the in-tree C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build the CUDA extension first (python -c 'import __graft_entry__ as g; g.build()')")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class DragonGPUError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != 0:
        msg = _lib.dragon_gpu_last_error().decode() if _lib is not None else "unknown"
        raise DragonGPUError(rc, msg)
