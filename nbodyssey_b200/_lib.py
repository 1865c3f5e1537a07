"""ctypes binding of libnbody_b200.so (the C ABI in include/nbody_b200.h).

The library is built in-tree by ``__graft_entry__.build()`` (nvcc, sm_100a).
There is no fallback: if the shared object is missing or fails to load, every
entry point raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnbody_b200.so")

NB_OK = 0
NB_ERR_INVALID = 1
NB_ERR_CUDA = 2
NB_ERR_DEVICE = 3
NB_ERR_NOMEM = 4
NB_ERR_IO = 5
NB_ERR_STATE = 6
NB_ERR_NOTFOUND = 7

NB_FORCE_NAIVE = 0
NB_FORCE_BH = 1
NB_FORCE_AUTO = 2
NB_AUTO_CROSSOVER = 20000
NB_TRAVERSE_THREAD = 0
NB_TRAVERSE_WARP = 1
NB_PHASES = 8
NB_STATE_TRAILER = 1
NB_STATE_ACC = 2
NB_STATE_LO = 4
PHASE_NAMES = ("prep", "morton", "sort", "build", "com", "walk", "energy", "other")


class NativeLibraryError(RuntimeError):
    """libnbody_b200.so is missing or could not be loaded."""


class NbError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__("nbody_b200 error %d: %s" % (code, msg))
        self.code = code


class nb_params(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("eps", ctypes.c_float),
                ("G", ctypes.c_float), ("theta", ctypes.c_float),
                ("force", ctypes.c_int32), ("traverse", ctypes.c_int32),
                ("key_bits", ctypes.c_int32), ("compensated", ctypes.c_int32),
                ("walk_kernel", ctypes.c_int32)]


NB_TUNE_VERSION = 2
NB_TUNE_BUCKETS = 16
NB_TUNE_THETAS = 3


class nb_tune_table(ctypes.Structure):
    _fields_ = [("version", ctypes.c_int32), ("sms", ctypes.c_int32),
                ("device", ctypes.c_char * 64),
                ("ap_threads", ctypes.c_int32 * NB_TUNE_BUCKETS),
                ("ap_k", ctypes.c_int32 * NB_TUNE_BUCKETS),
                ("ap_ctas", ctypes.c_int32 * NB_TUNE_BUCKETS),
                ("walk_warps", ctypes.c_int32),
                ("crossover", (ctypes.c_int32 * 2) * NB_TUNE_THETAS),
                ("crossover_batch", ctypes.c_int32 * NB_TUNE_THETAS)]


class nb_run_stats(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("force_ms", ctypes.c_double),
                ("force_calls", ctypes.c_long), ("frames", ctypes.c_int),
                ("e0", ctypes.c_double), ("e_final", ctypes.c_double),
                ("rel_final", ctypes.c_double),
                ("phase_ms", ctypes.c_double * NB_PHASES)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_S = ctypes.c_char_p
_SZ = ctypes.c_size_t
_PP = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes)
SIGNATURES = {
    "nb_params_default": (None, [ctypes.POINTER(nb_params)]),
    "nb_last_error": (_S, []),
    "nb_version": (_I, []),
    "nb_device_count": (_I, [ctypes.POINTER(_I)]),
    "nb_set_device": (_I, [_I]),
    "nb_alloc_pinned": (_I, [_SZ, _PP]),
    "nb_free_pinned": (_I, [_P]),
    "nb_measure_fp32_peak": (_I, [ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "nb_flush_l2": (_I, [_P, _SZ]),
    "nb_autotune": (_I, [_S, ctypes.POINTER(nb_tune_table)]),
    "nb_tune_get": (_I, [ctypes.POINTER(nb_tune_table)]),
    "nb_tune_set": (_I, [ctypes.POINTER(nb_tune_table)]),
    "nb_tune_defaults": (_I, [ctypes.POINTER(nb_tune_table)]),
    "nb_tune_load": (_I, [_S]),
    "nb_tune_save": (_I, [_S]),
    "nb_sim_create": (_I, [_I, _P, _P, ctypes.POINTER(nb_params), _PP]),
    "nb_sim_destroy": (_I, [_P]),
    "nb_sim_n": (_I, [_P, ctypes.POINTER(_I)]),
    "nb_set_params": (_I, [_P, ctypes.POINTER(nb_params)]),
    "nb_get_params": (_I, [_P, ctypes.POINTER(nb_params)]),
    "nb_set_state": (_I, [_P, _P, _P]),
    "nb_get_positions": (_I, [_P, _P]),
    "nb_get_velocities": (_I, [_P, _P]),
    "nb_get_position_lo": (_I, [_P, _P]),
    "nb_get_accelerations": (_I, [_P, _P]),
    "nb_set_state_acc": (_I, [_P, _P, _P, _P]),
    "nb_step_host": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "nb_step_host_state": (_I, [_P, _P, _P, _P, _P]),
    "nb_compute_forces": (_I, [_P, _P]),
    "nb_step": (_I, [_P, _I]),
    "nb_sync": (_I, [_P]),
    "nb_energy": (_I, [_P, _P, _P]),
    "nb_set_timing": (_I, [_P, _I]),
    "nb_force_timing": (_I, [_P, ctypes.POINTER(_D), ctypes.POINTER(ctypes.c_long)]),
    "nb_reset_timing": (_I, [_P]),
    "nb_phase_times": (_I, [_P, _P, ctypes.POINTER(ctypes.c_long)]),
    "nb_record": (_I, [_P, _I]),
    "nb_elapsed_ms": (_I, [_P, _I, _I, ctypes.POINTER(_D)]),
    "nb_set_graphs": (_I, [_P, _I]),
    "nb_debug_lbvh": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "nb_debug_forces": (_I, [_P, _P, _P]),
    "nb_debug_pairs": (_I, [_P, _P]),
    "nb_compare_forces": (_I, [_P, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "nb_workspace_create": (_I, [_PP]),
    "nb_workspace_destroy": (_I, [_P]),
    "nb_compute_forces_dev": (_I, [_P, _I, _P, _P, ctypes.POINTER(nb_params), _P]),
    "nb_leapfrog_step_dev": (_I, [_P, _I, _P, _P, _P, ctypes.POINTER(nb_params), _P]),
    "nb_total_energy_dev": (_I, [_P, _I, _P, _P, ctypes.POINTER(nb_params), _P, _P]),
    "nb_compute_forces_naive_static": (_I, [_I, _P, _P, _F, _F, _P]),
    "nb_compute_forces_naive_static_status": (_I, [ctypes.POINTER(ctypes.c_uint), _P]),
    "nb_forces_range_dev": (_I, [_P, _I, _P, _P, _P, _P, _P, ctypes.POINTER(nb_params),
                                 _I, _I, _P]),
    "nb_forces_gather_dev": (_I, [_P, _I, _P, _P, _P, ctypes.POINTER(nb_params), _P]),
    "nb_ensemble_create": (_I, [_I, _P, _P, _P, _P, _PP]),
    "nb_ensemble_destroy": (_I, [_P]),
    "nb_ensemble_size": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong)]),
    "nb_ensemble_step": (_I, [_P, _I]),
    "nb_ensemble_sync": (_I, [_P]),
    "nb_ensemble_set_graphs": (_I, [_P, _I]),
    "nb_ensemble_get_state": (_I, [_P, _I, _P, _P]),
    "nb_ensemble_get_accelerations": (_I, [_P, _I, _P]),
    "nb_ensemble_energy": (_I, [_P, _P]),
    "nb_ensemble_force": (_I, [_P, _I, ctypes.POINTER(_I)]),
    "nb_ensemble_kernels_per_step": (_I, [_P, ctypes.POINTER(_I)]),
    "nb_ensemble_record": (_I, [_P, _I]),
    "nb_ensemble_elapsed_ms": (_I, [_P, _I, _I, ctypes.POINTER(_D)]),
    "nb_server_create": (_I, [_SZ, _I, _PP]),
    "nb_server_destroy": (_I, [_P]),
    "nb_server_submit": (_I, [_P, _I, _P, _P, ctypes.POINTER(nb_params), _I, _I, _S,
                              ctypes.POINTER(ctypes.c_longlong)]),
    "nb_server_poll": (_I, [_P, ctypes.c_longlong, ctypes.POINTER(_I),
                            ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "nb_server_wait": (_I, [_P, ctypes.c_longlong, _D]),
    "nb_server_result": (_I, [_P, ctypes.c_longlong, _P, _P, _I]),
    "nb_server_get_stats": (_I, [_P, _P]),
    "nb_server_force": (_I, [_P, ctypes.c_longlong, ctypes.POINTER(_I)]),
    "nb_read_ic": (_I, [_S, ctypes.POINTER(_I), _P, _P]),
    "nb_write_ic": (_I, [_S, _I, _P, _P]),
    "nb_write_frame": (_I, [_S, _I, _I, _P]),
    "nb_write_state_file": (_I, [_S, _I, _P, _P, _P, _P, ctypes.POINTER(nb_params)]),
    "nb_read_state_file": (_I, [_S, ctypes.POINTER(_I), _P, _P, _P, _P,
                                ctypes.POINTER(nb_params), ctypes.POINTER(_I)]),
    "nb_save_state": (_I, [_P, _S]),
    "nb_load_state": (_I, [_P, _S]),
    "nb_format_energy_row": (_I, [_P, _SZ, _I, _F, _D, _D, _D, _D]),
    "nb_run": (_I, [_P, _I, _I, _S, _S, _I, ctypes.POINTER(nb_run_stats)]),
}

_lib = None


def load():
    """Loads the native library (once).  Raises NativeLibraryError."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryError(
            "%s is missing: build it with `python -c 'import __graft_entry__ as g; "
            "g.build()'` (nvcc, sm_100a)" % LIB_PATH)
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise NativeLibraryError("cannot load %s: %s" % (LIB_PATH, e)) from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    """Raises NbError for a non-zero status, with the library's message."""
    if rc != NB_OK:
        msg = load().nb_last_error()
        raise NbError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    """Data pointer of a numpy array (or None)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)
