"""ctypes binding of libnbb.so (include/nbb.h).

The CUDA library is the only implementation: when it is missing or cannot
be loaded this module raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libnbb.so")

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_Z = C.c_size_t

# nbb_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_DOMAIN = 2
ERR_LOGIC = 3
ERR_CUDA = 4
ERR_DEVICE = 5
ERR_TIMEOUT = 6
ERR_OVERFLOW = 7
ERR_NO_DEVICE = 8

PRECISION_FP64 = 0
PRECISION_MIXED = 1


class Config(C.Structure):
    _fields_ = [("time_step", C.c_double), ("theta", C.c_double), ("softening", C.c_double),
                ("gravitational_constant", C.c_double), ("precision", C.c_int),
                ("group_size", C.c_int), ("use_graph", C.c_int), ("device", C.c_int),
                ("cache_depth", C.c_int)]


class StateView(C.Structure):
    _fields_ = [("count", C.c_size_t)] + [(f, _P) for f in (
        "mass", "x", "y", "z", "vx", "vy", "vz", "type", "ax", "ay", "az")]


class Stats(C.Structure):
    _fields_ = [("n_groups", C.c_int), ("n_octree_nodes", C.c_int), ("interactions", C.c_int64),
                ("mac_tests", C.c_int64), ("group_size", C.c_int), ("stack_overflow", C.c_int64),
                ("cache_depth", C.c_int)]


class TreeExport(C.Structure):
    _fields_ = [("box", C.c_double * 4)] + [(f, _P) for f in (
        "keys", "idx", "uniq", "gfirst", "gcount", "left", "right", "rfirst", "rlast", "plen",
        "rparent", "plan_level", "plan_count", "plan_offset")] + [("m_capacity", C.c_int)] + [
        (f, _P) for f in ("children", "oparent", "olevel", "oprefix", "ofirst", "ocount",
                          "child_count", "cx", "cy", "cz", "half", "mass", "comx", "comy",
                          "comz")] + [("n_groups", C.c_int), ("n_octree", C.c_int)]


class Diagnostics(C.Structure):
    _fields_ = [("mass", _D), ("center_of_mass", _D * 3), ("momentum", _D * 3), ("angular_momentum", _D * 3),
                ("kinetic_energy", _D), ("potential_energy", _D), ("total_energy", _D), ("potential", _I)]


POTENTIAL_NONE, POTENTIAL_TREE, POTENTIAL_DIRECT = 0, 1, 2


class OctreeView(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("n_particles", C.c_int)] + [(f, _P) for f in (
        "children", "parent", "first", "count", "mass", "comx", "comy", "comz", "cx", "cy", "cz",
        "half")]


# symbol -> (restype, argtypes); the exported surface of include/nbb.h
SIGNATURES = {
    "nbb_config_default": (None, [_P]),
    "nbb_sim_create": (_I, [_P, _Z] + [_P] * 8 + [_I, _P]),
    "nbb_ensemble_create": (_I, [_P, _I, _P, _P] + [_P] * 7 + [_I, _P]),
    "nbb_sim_initialize": (_I, [_P]),
    "nbb_sim_step": (_I, [_P]),
    "nbb_sim_run": (_I, [_P, C.c_uint64]),
    "nbb_sim_time": (_D, [_P]),
    "nbb_sim_step_number": (C.c_uint64, [_P]),
    "nbb_sim_state": (_I, [_P, _P]),
    "nbb_sim_upload": (_I, [_P] * 8),
    "nbb_sim_download": (_I, [_P] * 7),
    "nbb_sim_download_accel": (_I, [_P] * 4),
    "nbb_sim_step_host": (_I, [_P] * 14),
    "nbb_sim_set_stream": (_I, [_P, _P]),
    "nbb_sim_synchronize": (_I, [_P]),
    "nbb_sim_destroy": (_I, [_P]),
    "nbb_sim_stats": (_I, [_P, _P]),
    "nbb_sim_profile": (_I, [_P, _P, _P]),
    "nbb_sim_export": (_I, [_P, _P]),
    "nbb_accel": (_I, [_Z, _P, _P, _P, _P, _D, _D, _D, _I, _P, _P, _P, _I, _P, _P]),
    "nbb_accel_direct": (_I, [_Z, _P, _P, _P, _P, _I, _P, _D, _D, _P, _P, _P, _I]),
    "nbb_accel_octree": (_I, [_P] * 9 + [_D, _D, _D, _I, _I]),
    "nbb_kick_drift": (_I, [_P] * 9 + [_Z, _D, _P]),
    "nbb_kick": (_I, [_P] * 6 + [_Z, _D, _P]),
    "nbb_octree_from_keys": (_I, [_P, _I, _P]),
    "nbb_radix_tree": (_I, [_P, _I] + [_P] * 6),
    "nbb_measure_fma_tflops": (_I, [_I, _P]),
    "nbb_selftest_bounded_wait": (_I, []),
    "nbb_sim_diagnostics": (_I, [_P, _I, _P]),
    "nbb_frame_bytes": (_Z, [_P, _Z]),
    "nbb_sim_capture_frame": (_I, [_P, _Z, C.c_uint64, _P, _Z, _P, _I]),
    "nbb_sim_rollout": (_I, [_P, C.c_uint64, C.c_uint64]),
    "nbb_sim_backward": (_I, [_P] * 14 + [_I]),
    "nbb_frozen_rollout": (_I, [_P, _Z] + [_P] * 7 + [_Z] + [_P] * 7 + [C.c_uint64] + [_P] * 6 + [_I]),
    "nbb_direct_rollout_adjoint": (_I, [_P, _Z] + [_P] * 7 + [C.c_uint64] + [_P] * 6 + [_P] * 6 + [_P] * 7
                                   + [_I]),
    "nbb_last_error_message": (C.c_char_p, []),
    "nbb_last_error_code": (_I, []),
    "nbb_kernel_launch_count": (C.c_uint64, []),
}

_lib = None


def load() -> C.CDLL:
    """Load libnbb.so (built by ``make -C amsc-nbody_b200``); raises when it
    is absent -- there is no other implementation to fall back to."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libnbb.so not built: {LIB_PATH} (run make -C amsc-nbody_b200)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class NbbError(RuntimeError):
    """Base of the library's errors; ``status`` is the nbb_status value and
    ``code`` the stage/device code."""

    def __init__(self, status: int, message: str, code: int = 0):
        super().__init__(message)
        self.status = status
        self.code = code


class InvalidArgument(NbbError, ValueError):
    """std::invalid_argument in the reference."""


class DomainError(NbbError, ValueError):
    """std::domain_error in the reference (non-finite positions)."""


class LogicError(NbbError):
    """std::logic_error in the reference (call order / state)."""


class DeviceError(NbbError):
    """std::runtime_error from a device error code in the reference."""


class OverflowErrorNbb(NbbError, OverflowError):
    """std::overflow_error in the reference."""


class NoDevice(NbbError):
    """No usable CUDA device."""


_STATUS_CLASS = {
    ERR_INVALID_ARGUMENT: InvalidArgument,
    ERR_DOMAIN: DomainError,
    ERR_LOGIC: LogicError,
    ERR_CUDA: DeviceError,
    ERR_DEVICE: DeviceError,
    ERR_TIMEOUT: DeviceError,
    ERR_OVERFLOW: OverflowErrorNbb,
    ERR_NO_DEVICE: NoDevice,
}


def check(status: int) -> None:
    if status == OK:
        return
    lib = load()
    msg = lib.nbb_last_error_message().decode(errors="replace")
    code = lib.nbb_last_error_code()
    raise _STATUS_CLASS.get(status, NbbError)(status, msg, code)


def ptr(a):
    """Host numpy array or torch tensor -> void pointer (None stays NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(_P)
