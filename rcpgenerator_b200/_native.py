"""ctypes binding of the engine's C ABI (include/rcpg.h).

The shared library is built in-tree (``make -C rcpgenerator_b200/csrc`` or
``__graft_entry__.build()``) as ``rcpgenerator_b200/librcpg_cuda.so``. There is
no CPU fallback: importing this module without the library raises, and every
compute entry point fails with ``RCPG_ECUDA`` when no CUDA device is present.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librcpg_cuda.so"

RCPG_OK = 0
RCPG_ERUNTIME = -1
RCPG_ECUDA = -2
RCPG_EINVAL = -22
RCPG_ENOSPC = -28

# Every symbol include/rcpg.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = (
    "rcpg_version",
    "rcpg_abi_version",
    "rcpg_device_count",
    "rcpg_default_options",
    "rcpg_run_packing",
    "rcpg_result_free",
    "rcpg_run_batch",
    "rcpg_run_batch_growth",
    "rcpg_batch_tuning",
    "rcpg_engine_create",
    "rcpg_engine_advance",
    "rcpg_engine_steps",
    "rcpg_engine_kernel_launches",
    "rcpg_engine_result",
    "rcpg_engine_destroy",
    "rcpg_engine_profile_pair_kernel",
    "rcpg_engine_profile_build_kernel",
    "rcpg_t_shell",
    "rcpg_pairs_full",
    "rcpg_pairs_full_noalloc",
    "rcpg_pairs_forces_scan",
    "rcpg_forces",
    "rcpg_mean_force",
    "rcpg_adam_step",
    "rcpg_refresh_check",
    "rcpg_scale_diameters_nd",
    "rcpg_initialize_particles",
    "rcpg_overlap_report",
    "rcpg_mlp_param_count",
    "rcpg_mlp_workspace_bytes",
    "rcpg_mlp_forward",
    "rcpg_mlp_train_step",
    "rcpg_mlp_to_bf16",
)

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i8p = C.POINTER(C.c_int8)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)


class PackingInput(C.Structure):
    _fields_ = [
        ("N", C.c_uint64),
        ("ndim", C.c_int32),
        ("positions", _dp),
        ("diameters", _dp),
        ("box", _dp),
        ("box_len", C.c_int32),
        ("walls", _i8p),
        ("walls_len", C.c_int32),
        ("neighbor_max", C.c_uint32),
        ("seed", C.c_uint32),
        ("fix_height", C.c_int32),
    ]


class RunOptions(C.Structure):
    _fields_ = [
        ("max_steps", C.c_uint64),
        ("has_mu_override", C.c_int32),
        ("mu_override", C.c_double),
        ("fix_diameter", C.c_int32),
        ("has_target_phi", C.c_int32),
        ("target_phi", C.c_double),
        ("reorder_interval", C.c_uint64),
        ("has_initial_phi_target", C.c_int32),
        ("initial_phi_target", C.c_double),
        ("exact", C.c_int32),
        ("device", C.c_int32),
        ("graph_steps", C.c_int32),
        ("pair_precision", C.c_int32),
        ("mixed_switch", C.c_double),
        ("growth_steps", C.c_uint64),
    ]


class Observation(C.Structure):
    _fields_ = [
        ("step", C.c_uint64),
        ("phi", C.c_double),
        ("force_magnitude", C.c_double),
        ("energy", C.c_double),
        ("max_min_dist", C.c_double),
    ]


OBSERVER = C.CFUNCTYPE(None, C.POINTER(Observation), _dp, C.c_void_p)


class Result(C.Structure):
    _fields_ = [
        ("N", C.c_uint64),
        ("ndim", C.c_int32),
        ("steps", C.c_uint64),
        ("phi", C.c_double),
        ("max_min_dist", C.c_double),
        ("force_magnitude", C.c_double),
        ("positions", _dp),
        ("diameters", _dp),
        ("box", _dp),
        ("walls", _i8p),
        ("phi_history", _dp),
        ("force_history", _dp),
        ("energy_history", _dp),
        ("max_overlap_history", _dp),
        ("mu_history", _dp),
        ("alpha_history", _dp),
        ("mu_flag_history", _i8p),
        ("particle_origin", _u64p),
        ("trace_len", C.c_uint64),
        ("trace_steps", _u64p),
        ("trace_positions", _dp),
        ("trace_diameters", _dp),
        ("trace_phi", _dp),
        ("trace_force", _dp),
        ("trace_energy", _dp),
        ("trace_max_min_dist", _dp),
        ("pair_builds", C.c_uint64),
        ("row_capacity", C.c_uint32),
        ("kernel_launches", C.c_uint64),
        ("fp64_switch_step", C.c_uint64),
        ("pair_energy_rel_error", C.c_double),
        ("pair_force_rel_error", C.c_double),
    ]


class Distribution(C.Structure):
    _fields_ = [
        ("type", C.c_char_p),
        ("d", C.c_double),
        ("mu", C.c_double),
        ("sigma", C.c_double),
        ("mu1", C.c_double),
        ("sigma1", C.c_double),
        ("mu2", C.c_double),
        ("sigma2", C.c_double),
        ("p", C.c_double),
        ("d1", C.c_double),
        ("d2", C.c_double),
        ("d_min", C.c_double),
        ("d_max", C.c_double),
        ("exponent", C.c_double),
        ("scale", C.c_double),
        ("shape", C.c_double),
        ("custom", _dp),
        ("custom_len", C.c_uint64),
    ]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"rcpgenerator_b200: CUDA library {LIB_PATH} is missing; build it with "
            "`make -C rcpgenerator_b200/csrc` (this engine has no CPU path)"
        )
    lib = C.CDLL(os.fspath(LIB_PATH), mode=C.RTLD_GLOBAL)
    vp, sz, cp = C.c_void_p, C.c_size_t, C.c_char_p
    sig = {
        "rcpg_version": (C.c_char_p, []),
        "rcpg_abi_version": (C.c_int32, []),
        "rcpg_device_count": (C.c_int32, []),
        "rcpg_default_options": (None, [C.POINTER(RunOptions)]),
        "rcpg_run_packing": (
            C.c_int32,
            [C.POINTER(PackingInput), C.POINTER(RunOptions), C.c_uint64, C.c_int32, C.c_uint64,
             OBSERVER, vp, C.POINTER(C.POINTER(Result)), cp, sz],
        ),
        "rcpg_result_free": (None, [C.POINTER(Result)]),
        "rcpg_batch_tuning": (
            C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), _dp, cp, sz]
        ),
        "rcpg_run_batch_growth": (
            C.c_int32,
            [C.POINTER(PackingInput), C.c_uint64, C.POINTER(RunOptions), _u64p, C.c_int32,
             C.POINTER(C.POINTER(Result)), C.POINTER(C.c_int32), cp, sz],
        ),
        "rcpg_run_batch": (
            C.c_int32,
            [C.POINTER(PackingInput), C.c_uint64, C.POINTER(RunOptions), C.c_int32,
             C.POINTER(C.POINTER(Result)), C.POINTER(C.c_int32), cp, sz],
        ),
        "rcpg_engine_create": (
            C.c_int32,
            [C.POINTER(PackingInput), C.POINTER(RunOptions), vp, C.POINTER(vp), cp, sz],
        ),
        "rcpg_engine_advance": (C.c_int32, [vp, C.c_uint64, C.POINTER(C.c_int32), cp, sz]),
        "rcpg_engine_steps": (C.c_uint64, [vp]),
        "rcpg_engine_kernel_launches": (C.c_uint64, [vp]),
        "rcpg_engine_result": (C.c_int32, [vp, C.POINTER(C.POINTER(Result)), cp, sz]),
        "rcpg_engine_destroy": (None, [vp]),
        "rcpg_engine_profile_build_kernel": (C.c_int32, [vp, C.c_uint32, _dp, _dp, cp, sz]),
        "rcpg_engine_profile_pair_kernel": (
            C.c_int32, [vp, C.c_uint32, _dp, _dp, _dp, cp, sz]
        ),
        "rcpg_t_shell": (C.c_double, [_dp, C.c_uint64]),
        "rcpg_pairs_full": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, _dp, _i8p, C.c_double, C.c_uint32, vp, vp, _u32p, vp,
             cp, sz],
        ),
        "rcpg_pairs_full_noalloc": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, _dp, _i8p, C.c_double, C.c_uint32, vp, vp, _u32p, vp,
             cp, sz],
        ),
        "rcpg_pairs_forces_scan": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, _dp, _i8p, C.c_double, C.c_double, C.c_int32, C.c_uint32,
             vp, vp, _u32p, vp, _dp, _i32p, vp, cp, sz],
        ),
        "rcpg_forces": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, _dp, _i8p, vp, vp, C.c_uint32, C.c_double, C.c_int32,
             vp, _dp, vp, cp, sz],
        ),
        "rcpg_mean_force": (C.c_int32, [C.c_uint64, C.c_int32, vp, _dp, vp, cp, sz]),
        "rcpg_adam_step": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, vp, vp, _dp, C.c_double, C.c_uint64, vp, cp, sz],
        ),
        "rcpg_refresh_check": (
            C.c_int32,
            [C.c_uint64, C.c_int32, vp, vp, vp, vp, vp, C.c_double, vp, _u64p, vp, cp, sz],
        ),
        "rcpg_scale_diameters_nd": (
            C.c_double, [_dp, C.c_uint64, C.c_double, _dp, C.c_int32, C.c_int32, _dp]
        ),
        "rcpg_initialize_particles": (
            C.c_int32,
            [C.c_double, C.c_uint64, C.c_int32, _dp, C.c_int32, _i8p, C.c_int32, C.c_int32,
             C.POINTER(Distribution), C.c_uint64, _dp, _dp, _dp, _i8p, _dp, _dp, cp, sz],
        ),
        "rcpg_overlap_report": (
            C.c_int32,
            [C.c_uint64, C.c_int32, _dp, _dp, _dp, _u64p, _u64p, C.c_uint64, _u32p, _dp, _dp, C.c_int32,
             cp, sz],
        ),
        "rcpg_mlp_param_count": (C.c_uint64, [_i32p, C.c_int32]),
        "rcpg_mlp_workspace_bytes": (C.c_uint64, [_i32p, C.c_int32, C.c_int32]),
        "rcpg_mlp_forward": (
            C.c_int32,
            [_i32p, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, C.c_uint64, vp, cp, sz],
        ),
        "rcpg_mlp_train_step": (
            C.c_int32,
            [_i32p, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp, C.c_float, C.c_int32,
             vp, vp, C.c_uint64, vp, cp, sz],
        ),
        "rcpg_mlp_to_bf16": (C.c_int32, [C.c_uint64, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class NativeError(RuntimeError):
    """Error returned by the C ABI; ``code`` is the RCPG_E* value."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def raise_for(code: int, err: C.Array) -> None:
    if code == RCPG_OK:
        return
    msg = err.value.decode(errors="replace") or f"rcpgenerator_b200 error {code}"
    if code == RCPG_EINVAL:
        raise ValueError(msg)
    if code == RCPG_ERUNTIME:
        raise RuntimeError(msg)
    raise NativeError(code, msg)


def errbuf() -> C.Array:
    return C.create_string_buffer(4096)
