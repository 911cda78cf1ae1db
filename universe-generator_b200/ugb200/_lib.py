"""ctypes binding of libug.so (the C ABI declared in include/ug.h).

The packer has no CPU fallback: importing this module on a machine without
the built library, or calling into it without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# UG_LIB=checked selects the index-guarded diagnostic build (libug_checked.so)
LIB_PATH = os.path.join(HERE, "libug_checked.so" if os.environ.get("UG_LIB") == "checked" else "libug.so")

UG_OK, UG_EINVAL, UG_ENOMEM, UG_ECAP, UG_ECUDA, UG_ETIMEDOUT, UG_ENOTSUP = range(7)
RNG_PHILOX, RNG_KNOT = 0, 1
ZGRID_REF, ZGRID_MID = 0, 1
EXCL_REF, EXCL_OPEN = 0, 1
GROUP_NONE, GROUP_SUBPATH, GROUP_UNIQUE = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1

EXPORTS = (
    "ug_version", "ug_last_error", "ug_struct_sizes", "ug_device_info", "ug_selftest_bounded_wait", "ug_batch_create", "ug_batch_run", "ug_batch_done",
    "ug_batch_stats", "ug_batch_accepted", "ug_batch_accepted_all", "ug_batch_positions", "ug_batch_params",
    "ug_batch_params_noalloc",
    "ug_batch_kernel_times", "ug_batch_reset_times", "ug_batch_counters", "ug_batch_mixed_error",
    "ug_batch_destroy", "ug_pack_create", "ug_pack_run", "ug_pack_stats", "ug_pack_destroy",
    "ug_frame_bake", "ug_batch_frames", "ug_state_bytes", "ug_batch_save_state", "ug_batch_restore",
    "ug_batch_probe", "ug_apparent_positions", "ug_apparent_positions_async",
)


class UniverseCfg(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("T", C.c_int32), ("terms", C.c_int32), ("rng", C.c_int32),
        ("zgrid", C.c_int32), ("excl", C.c_int32), ("cross1d", C.c_int32),
        ("pin_sin1", C.c_int32), ("group_mode", C.c_int32), ("round_size", C.c_int32),
        ("seed", C.c_uint64), ("attempts", C.c_int64), ("max_n", C.c_int64),
        ("sub_attempts", C.c_int64), ("accept_rate", C.c_double),
        ("sub_accept_rate", C.c_double), ("sub_fill_rate", C.c_double),
        ("euclid", C.c_int32), ("surv_cap", C.c_int32),
    ]


class RunOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("device", C.c_int32), ("rounds_per_sync", C.c_int32),
        ("use_graph", C.c_int32), ("kernel_timing", C.c_int32), ("force_hash", C.c_int32),
        ("stream", C.c_uint64), ("slot_hint", C.c_int64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_unique", C.c_int64), ("n_sub", C.c_int64),
        ("attempts", C.c_int64), ("phase1_end", C.c_int64), ("rounds", C.c_int64),
        ("gray", C.c_int64), ("evals", C.c_int64), ("evals_fp64", C.c_int64),
        ("state", C.c_int32), ("grid_kind", C.c_int32), ("filled", C.c_int64),
        ("visits", C.c_int64),
    ]


class KernelTimes(C.Structure):
    _fields_ = [("ms", C.c_double * 12), ("launches", C.c_int64 * 12),
                ("names", C.c_char_p * 12)]


class UgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ug error {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libug.so and declare its signatures (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run universe-generator_b200/ugb200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.ug_version.restype = C.c_int
    L.ug_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.ug_struct_sizes.argtypes = [vp, i32]
    L.ug_selftest_bounded_wait.argtypes = [i64, vp]
    L.ug_device_info.argtypes = [i32, C.c_char_p, C.c_size_t, vp]
    L.ug_batch_create.argtypes = [C.POINTER(UniverseCfg), i32, C.POINTER(RunOpts), C.POINTER(vp)]
    L.ug_batch_run.argtypes = [vp, i64]
    L.ug_batch_done.argtypes = [vp]
    L.ug_batch_reset.argtypes = [vp, vp]
    L.ug_batch_stats.argtypes = [vp, i32, C.POINTER(Stats)]
    L.ug_batch_accepted.argtypes = [vp, i32, vp, vp, i64, C.POINTER(i64)]
    L.ug_batch_accepted_all.argtypes = [vp, vp, vp, i64, vp]
    L.ug_batch_positions.argtypes = [vp, i32, vp, i64]
    L.ug_batch_params.argtypes = [vp, i32, vp, vp, vp, vp, i64]
    L.ug_batch_params_noalloc.argtypes = [vp, i32, vp, vp, vp, vp, i64]
    L.ug_batch_kernel_times.argtypes = [vp, C.POINTER(KernelTimes)]
    L.ug_batch_reset_times.argtypes = [vp]
    L.ug_batch_counters.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]
    L.ug_batch_mixed_error.argtypes = [vp, i32, i64, i64, C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.ug_batch_destroy.argtypes = [vp]
    L.ug_frame_bake.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp]
    L.ug_batch_frames.argtypes = [vp, i32, vp, vp]
    L.ug_state_bytes.argtypes = []
    L.ug_batch_save_state.argtypes = [vp, i32, vp]
    L.ug_batch_restore.argtypes = [vp, i32, i64, vp, vp, vp]
    L.ug_batch_probe.argtypes = [vp, i32, C.c_uint64, i64, i32, vp, vp]
    L.ug_apparent_positions.argtypes = [vp, i64, C.c_double, C.c_double, i32, i32, vp, vp, vp]
    L.ug_apparent_positions_async.argtypes = [vp, i64, C.c_double, C.c_double, i32, i32, vp, vp, vp, vp]
    for name in EXPORTS:
        f = getattr(L, name)
        if f.restype is None or name != "ug_last_error":
            f.restype = C.c_int
    L.ug_state_bytes.restype = i64
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().ug_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != UG_OK:
        raise UgError(rc, last_error())
