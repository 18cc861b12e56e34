"""ctypes bindings of the C ABI in include/pme_recip.h and include/pme_direct.h (libpme_b200.so).

The shared library is built in-tree by gpu_recip_b200/build.py.  There is no fallback: if the
library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libpme_b200.so")

PME_OK = 0
PME_EINVAL = -1
PME_EUNSUPPORTED = -2
PME_ECUDA = -3
PME_ETIMEOUT = -4
PME_ENOMEM = -5
PME_ESTATE = -6

PME_FFT_COLUMN, PME_FFT_SLAB, PME_FFT_BOX = 0, 1, 2
PME_FORCE_F32_SOA, PME_FORCE_F32X3, PME_FORCE_I64_SOA_ACCUM = 0, 1, 2
PME_EV_RECIP, PME_EV_SELF, PME_EV_VIRIAL, PME_EV_COUNT = 0, 1, 2, 11
PME_VDW_NONE, PME_VDW_VSH = 0, 1
PME_ELEC_NONE, PME_ELEC_EWALD = 0, 101

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)

# name -> argtypes; every function returns int unless listed in _RESTYPES
SIGNATURES = {
    "pme_create": [_I, _I, _I, _I, _I, _I, _I, _P, ctypes.POINTER(_P)],
    "pme_destroy": [_P],
    "pme_set_stream": [_P, _P],
    "pme_get_stream": [_P, ctypes.POINTER(_P)],
    "pme_recip_loop_run": [_P, _D, _P, ctypes.POINTER(ctypes.c_longlong)],
    "pme_set_order": [_P, _I],
    "pme_get_nfft": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "pme_get_order": [_P, ctypes.POINTER(_I)],
    "pme_print_info": [_P],
    "pme_spread_charge": [_P, _P, _I, _DP],
    "pme_r2c_fft": [_P],
    "pme_scalar_sum": [_P, _DP, _D, _I, _I],
    "pme_c2r_fft": [_P],
    "pme_gather_force": [_P, _P, _I, _DP, _I, _I, _P],
    "pme_calc_self_energy": [_P, _P, _I, _D],
    "pme_clear_energy_virial": [_P],
    "pme_get_energy_virial": [_P, _DP, _DP, _DP],
    "pme_copy_energy_virial_async": [_P, _P],
    "pme_energy_virial_device_ptr": [_P, ctypes.POINTER(_P)],
    "pme_set_energy_virial_mirror": [_P, _P],
    "pme_eval_ortho": [_P, _D, _D, _D, _P, _I, _D, _I, _I, _I, _P, _I],
    "pme_eval": [_P, _DP, _P, _I, _D, _I, _I, _I, _P, _I],
    "pme_eval_host": [_P, _DP, _P, _I, _D, _I, _I, _I, _P, _I],
    "pme_copy_charge_grid_fixed": [_P, _P],
    "pme_copy_charge_grid": [_P, _P],
    "pme_copy_fft_grid": [_P, _P],
    "pme_copy_solved_grid": [_P, _P],
    "pme_load_charge_grid": [_P, _P],
    "pme_get_status": [_P, ctypes.POINTER(_I)],
    "pme_set_barrier_spin_limit": [_P, ctypes.c_uint],
    "pme_reserve_atoms": [_P, _I],
    "pme_set_fault_injection": [_P, _I],
    "pme_set_fft_schedule": [_P, _I],
    "pme_set_x_gather_fusion": [_P, _I],
    "pme_batch_create": [_P, _I, _P, ctypes.POINTER(_P)],
    "pme_batch_destroy": [_P],
    "pme_batch_set_stream": [_P, _P],
    "pme_batch_set_system": [_P, _I, _DP, _P, _P],
    "pme_batch_commit": [_P],
    "pme_batch_eval": [_P],
    "pme_batch_clear_energy_virial": [_P],
    "pme_batch_get_energy_virial": [_P, _DP],
    "pme_batch_info": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_size_t)],
    "pme_system_device_bytes": [_I, _I, _I],
    "pme_set_trace": [_P, _P, _I],
    "pme_spread_charge_noalloc": [_P, _I, _DP, _I, _I, _I, _I, _P, _P],
    "pme_force_convert": [_P, _I, _I, _P, _I, _I, _P],
    "pme_force_convert_add": [_P, _I, _I, _P, _I, _I, _P],
    "pme_batch_set_trace": [_P, _P, _I],
    "pme_autotune": [_P, _P, _I, _D, _D, _D, _D, _I, _P],
    "pme_get_tune_config": [_P, _P],
    "pme_set_tune_config": [_P, _P],
    "pme_tune_cache_clear": [],
    "pme_batch_autotune": [_P, _I, _P],
    "pme_server_create": [ctypes.c_size_t, _I, _P, ctypes.POINTER(_P)],
    "pme_server_destroy": [_P],
    "pme_request_device_bytes": [_P],
    "pme_server_submit": [_P, _P, ctypes.POINTER(ctypes.c_longlong)],
    "pme_server_wait": [_P, ctypes.c_longlong, _D, _DP],
    "pme_server_get_stats": [_P, _P],
    "pme_direct_create": [_P, ctypes.POINTER(_P)],
    "pme_direct_destroy": [_P],
    "pme_direct_set_stream": [_P, _P],
    "pme_direct_setup": [_P, _D, _D, _D, _D, _D, _D, _D, _I, _I],
    "pme_direct_set_box_size": [_P, _D, _D, _D],
    "pme_direct_set_vdwparam": [_P, _I, _P],
    "pme_direct_set_vdwparam14": [_P, _I, _P],
    "pme_direct_set_vdwtype": [_P, _I, _P],
    "pme_direct_set_exclusions": [_P, _I, _P, _P, _P],
    "pme_direct_set_14_list": [_P, _I, _I, _P, _P],
    "pme_direct_calc_force": [_P, _P, _I, _I, _I, _I, _P],
    "pme_direct_calc_14_force": [_P, _P, _I, _I, _I, _P],
    "pme_direct_clear_energy_virial": [_P],
    "pme_direct_get_energy_virial": [_P, _DP, _DP, _DP, _DP],
    "pme_last_error_string": [],
    "pme_status_string": [_I],
    "pme_version": [],
}
_RESTYPES = {"pme_last_error_string": ctypes.c_char_p, "pme_status_string": ctypes.c_char_p,
             "pme_system_device_bytes": ctypes.c_size_t, "pme_request_device_bytes": ctypes.c_size_t}

PME_INJECT_NONE, PME_INJECT_SKIP_BARRIER = 0, 1
PME_SCHED_AUTO, PME_SCHED_PLANES, PME_SCHED_PASSES, PME_SCHED_CLUSTER = 0, 1, 2, 3
PME_XGATHER_AUTO, PME_XGATHER_OFF = 0, 1
PME_REAL_F32, PME_REAL_F64 = 0, 1


class SystemDesc(ctypes.Structure):
    """pme_system_desc of include/pme_recip.h."""
    _fields_ = [("nfftx", _I), ("nffty", _I), ("nfftz", _I), ("order", _I), ("natom", _I),
                ("box", ctypes.c_double * 3), ("kappa", ctypes.c_double), ("xyzq", _P),
                ("force", _P), ("force_kind", _I), ("stride", _I), ("calc_energy", _I),
                ("calc_virial", _I)]


class RecipHeader(ctypes.Structure):
    """pme_recip_header of include/pme_recip.h."""
    _fields_ = [("inv_boxx", ctypes.c_double), ("inv_boxy", ctypes.c_double), ("inv_boxz", ctypes.c_double),
                ("ncoord", _I), ("calc_energy", _I), ("calc_virial", _I)]


RECV_HEADER = ctypes.CFUNCTYPE(_I, _P, ctypes.POINTER(RecipHeader))
RECV_COORD = ctypes.CFUNCTYPE(_I, _P, _I, _P, ctypes.POINTER(_P))
SEND_FORCE = ctypes.CFUNCTYPE(_I, _P, _I, _P, ctypes.POINTER(ctypes.c_double))


class RecipComm(ctypes.Structure):
    """pme_recip_comm of include/pme_recip.h."""
    _fields_ = [("user", _P), ("recv_header", RECV_HEADER), ("recv_coord", RECV_COORD),
                ("send_force", SEND_FORCE)]


class TuneConfig(ctypes.Structure):
    """pme_tune_config of include/pme_recip.h."""
    _fields_ = [("schedule", _I), ("x_lines", _I), ("y_lines", _I), ("z_columns", _I),
                ("grid_ctas", _I), ("us_per_eval", ctypes.c_float), ("candidates", _I)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(ctypes.Structure):
    """pme_request of include/pme_recip.h."""
    _fields_ = [("nfftx", _I), ("nffty", _I), ("nfftz", _I), ("order", _I), ("natom", _I),
                ("box", ctypes.c_double * 3), ("kappa", ctypes.c_double), ("xyzq", _P),
                ("n_evals", _I), ("sigma", ctypes.c_float), ("seed", ctypes.c_ulonglong),
                ("calc_energy", _I), ("calc_virial", _I), ("ev_out", _P), ("force_out", _P)]


class ServerStats(ctypes.Structure):
    """pme_server_stats of include/pme_recip.h."""
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("evals", ctypes.c_longlong), ("steps", ctypes.c_longlong),
                ("active", ctypes.c_longlong), ("pending", ctypes.c_longlong),
                ("arena_bytes", ctypes.c_size_t), ("arena_used", ctypes.c_size_t),
                ("seconds", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


class PMEError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {status_name(status)} ({status}): {msg}")
        self.status = status


def load(path: str | None = None):
    """Load libpme_b200.so (raises if it is absent: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"CUDA library {p} is missing; build it with python -m gpu_recip_b200.build")
    lib = ctypes.CDLL(p)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _RESTYPES.get(name, _I)
    _lib = lib
    return lib


def status_name(status: int) -> str:
    try:
        return load().pme_status_string(status).decode()
    except Exception:  # library not loadable while formatting an error
        return str(status)


def check(status: int, where: str) -> None:
    if status != PME_OK:
        msg = load().pme_last_error_string().decode(errors="replace")
        raise PMEError(status, where, msg)


def dbl9(values) -> ctypes.Array:
    arr = (ctypes.c_double * 9)(*[float(v) for v in values])
    return arr


def exported_symbols():
    return list(SIGNATURES)
