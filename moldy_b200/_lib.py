"""ctypes binding of ``libmoldy_gpu.so`` (the C ABI in ``include/moldy_gpu.h``).

There is no CPU fallback: if the library is missing or cannot be loaded this
module raises, and every compute call goes to the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmoldy_gpu.so")

MOLDY_OK = 0
ERRORS = {
    1: "MOLDY_ERR_INVALID",
    2: "MOLDY_ERR_NEIGHBOUR_OVERFLOW",
    3: "MOLDY_ERR_SINGULAR_BOX",
    4: "MOLDY_ERR_CUDA",
    5: "MOLDY_ERR_ORDER",
    6: "MOLDY_ERR_CAPACITY",
    7: "MOLDY_ERR_UNSUPPORTED",
    8: "MOLDY_ERR_NO_DEVICE",
}
PREC_FP64 = 0
PREC_MIXED = 1


class MoldyError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("rnear", ctypes.c_double), ("deltat", ctypes.c_double),
                ("press", ctypes.c_double), ("bdel2", ctypes.c_double),
                ("nm", ctypes.c_int32), ("nnbrs", ctypes.c_int32), ("ivol", ctypes.c_int32),
                ("ntcm", ctypes.c_int32), ("ntc", ctypes.c_int32),
                ("nlcx", ctypes.c_int32), ("nlcy", ctypes.c_int32), ("nlcz", ctypes.c_int32),
                ("atomstress", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("device", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_M9 = ctypes.c_double * 9


class ForceOut(ctypes.Structure):
    _fields_ = [("pe", ctypes.c_double), ("vol", ctypes.c_double),
                ("tp", _M9), ("tk", _M9), ("tc", _M9), ("tg", _M9), ("tgdot", _M9),
                ("tgid", _M9), ("fb", _M9), ("ntc", ctypes.c_int32), ("rebuilt", ctypes.c_int32)]


class Thermo(ctypes.Structure):
    _fields_ = [("ke", ctypes.c_double), ("pe", ctypes.c_double), ("te", ctypes.c_double),
                ("h", ctypes.c_double), ("th", ctypes.c_double), ("vol", ctypes.c_double),
                ("s1", ctypes.c_double), ("s2", ctypes.c_double), ("s3", ctypes.c_double),
                ("temp", ctypes.c_double), ("boxke", ctypes.c_double),
                ("ntc", ctypes.c_int32), ("rebuilt", ctypes.c_int32)]


D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int32)
H = ctypes.c_void_p

# name -> argument types (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "moldy_gpu_create": [ctypes.POINTER(Params), ctypes.POINTER(H)],
    "moldy_gpu_destroy": [H],
    "moldy_gpu_last_error": [],
    "moldy_gpu_version": [],
    "moldy_gpu_set_fetm_fe": [H, ctypes.c_int32, D, D, ctypes.c_int32, D, D, ctypes.c_int32,
                              ctypes.c_int32],
    "moldy_gpu_set_tables": [H, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, D, D, D, D, D, D],
    "moldy_gpu_get_tables": [H, D, D, D, D, D, D],
    "moldy_gpu_set_state": [H] + [D] * 12 + [I, D, D, D],
    "moldy_gpu_get_state": [H] + [D] * 13,
    "moldy_gpu_get_forces": [H, D, D, D],
    "moldy_gpu_get_density": [H, D, D, D],
    "moldy_gpu_get_atomstress": [H, D, D, D],
    "moldy_gpu_set_ntc": [H, ctypes.c_int32],
    "moldy_gpu_linkup": [H],
    "moldy_gpu_relink": [H],
    "moldy_gpu_get_linkcells": [H, I, I, I],
    "moldy_gpu_update_neighbourlist": [H],
    "moldy_gpu_get_neighbourlist": [H, I, I],
    "moldy_gpu_get_reverse_list": [H, I, I],
    "moldy_gpu_force": [H, ctypes.POINTER(ForceOut)],
    "moldy_gpu_velocityverlet": [H, ctypes.POINTER(ForceOut)],
    "moldy_gpu_update_therm_avs": [H, D],
    "moldy_gpu_md_init": [H, ctypes.POINTER(ForceOut)],
    "moldy_gpu_md_steps": [H, ctypes.c_int32, ctypes.POINTER(Thermo)],
    "moldy_gpu_energy_calc": [H, D],
    "moldy_gpu_synchronize": [H],
    "moldy_gpu_get_stream": [H, ctypes.POINTER(ctypes.c_void_p)],
    "moldy_gpu_set_profiling": [H, ctypes.c_int32],
    "moldy_gpu_reset_kernel_stats": [H],
    "moldy_gpu_kernel_stats": [H, ctypes.c_int32, D, ctypes.POINTER(ctypes.c_int64)],
    "moldy_gpu_kernel_name": [ctypes.c_int32],
    "moldy_gpu_autotune": [H, ctypes.c_int32, D, I],
    "moldy_gpu_set_variants": [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
    "moldy_gpu_get_list_stats": [H, D],
    "moldy_gpu_set_iron_carbon_fe": [H, ctypes.c_int32],
    "moldy_ic_build_tables": [ctypes.c_int32, D, D, D, D, D, D],
    "moldy_gpu_set_mid_skin": [H, ctypes.c_double],
    "moldy_gpu_set_outer_skin": [H, ctypes.c_double],
    "moldy_gpu_get_outer_builds": [H, ctypes.POINTER(ctypes.c_int32)],
    "moldy_gpu_set_thermostat": [H, ctypes.c_double, ctypes.c_double],
    "moldy_gpu_get_thermostat": [H, D],
    "moldy_gpu_scalev": [H],
    "moldy_gpu_table_gradients": [H, ctypes.c_double, D, D, D, D, D, D, D, D],
    "moldy_gpu_knot_gradients": [H, ctypes.c_double, D, D, D, D, D, D],
    "moldy_gpu_rdf": [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, I, ctypes.c_int32,
                      ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)],
    "moldy_gpu_ackland_jones": [H, ctypes.c_int32, I, ctypes.c_int32, D, I, I, I],
    "moldy_gpu_batch_create": [ctypes.c_int32, I, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(H)],
    "moldy_gpu_batch_destroy": [H],
    "moldy_gpu_batch_set_fetm_fe": [H, ctypes.c_int32, D, D, ctypes.c_int32, D, D, ctypes.c_int32],
    "moldy_gpu_batch_set_state": [H, D, D, D, D, D],
    "moldy_gpu_batch_get_state": [H, D, D, D],
    "moldy_gpu_batch_force": [H, D],
    "moldy_gpu_batch_get_forces": [H, D, D, D],
    "moldy_gpu_batch_get_energies": [H, D, D],
    "moldy_gpu_batch_set_positions": [H, D],
    "moldy_gpu_batch_get_forces_xyz": [H, D],
    "moldy_gpu_batch_get_density": [H, D, D, D],
    "moldy_gpu_batch_quench": [H, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, D],
    "moldy_gpu_batch_set_tiles": [H, ctypes.c_int32, ctypes.c_int32],
    "moldy_gpu_batch_set_skin": [H, ctypes.c_double],
    "moldy_gpu_batch_set_precision": [H, ctypes.c_int32],
    "moldy_gpu_batch_set_energy_calc": [H, ctypes.c_int32],
    "moldy_gpu_batch_autotune": [H, ctypes.c_int32, D, I],
    "moldy_gpu_batch_kernel_times": [H, ctypes.c_int32, D],
    "moldy_gpu_batch_set_references": [H, D, D],
    "moldy_gpu_batch_force_matching": [H, ctypes.c_double, ctypes.c_double, D, D],
    "moldy_gpu_batch_set_gather": [H, ctypes.c_int32],
    "moldy_gpu_batch_set_persistent": [H, ctypes.c_int32],
    "moldy_gpu_batch_set_atom_lanes": [H, ctypes.c_int32],
    "moldy_gpu_batch_persistent_applies": [H, I],
    "moldy_gpu_batch_eval_times": [H, D],
    "moldy_gpu_batch_list_stats": [H, ctypes.POINTER(ctypes.c_int64)],
    "moldy_gpu_batch_row_entries": [H, ctypes.POINTER(ctypes.c_int64)],
    "moldy_gpu_batch_launches": [H, ctypes.POINTER(ctypes.c_int64)],
    "moldy_gpu_batch_get_stream": [H, ctypes.POINTER(ctypes.c_void_p)],
    "moldy_fetm_build_tables": [ctypes.c_int32, D, D, ctypes.c_int32, D, D, ctypes.c_int32,
                                D, D, D, D, D, D],
    "moldy_fetm_knot_vjp": [ctypes.c_int32, D, D, ctypes.c_int32, D, D, ctypes.c_int32,
                            D, D, D, D, D, D, D, D, D, D],
    "moldy_gpu_force_noalloc": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, D, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double] + [ctypes.c_void_p] * 11,
}
NOALLOC_MAX_ATOMS = 262144
KERNEL_FAMILIES = 16
TUNE_VARIANTS = 8
_RESTYPE = {"moldy_gpu_last_error": ctypes.c_char_p, "moldy_gpu_version": ctypes.c_char_p,
            "moldy_gpu_kernel_name": ctypes.c_char_p}

_lib = None


def load(path: str = LIB_PATH):
    """Loads the CUDA library; raises if it is absent (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with moldy_b200.build.build() "
                          "(nvcc, sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != MOLDY_OK:
        msg = load().moldy_gpu_last_error()
        raise MoldyError(rc, msg.decode() if msg else "")
