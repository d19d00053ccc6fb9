"""ctypes loader for libthirring_b200.so and the declarations of its C ABI.

The library is the product: there is no fallback.  If the shared library is
missing or cannot be loaded this module raises, so nothing downstream can
silently run on the CPU.
"""
import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libthirring_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "thirring_b200.h")


class Params(C.Structure):
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("lt", C.c_int), ("ls", C.c_int),
                ("kernel", C.c_int), ("layout", C.c_int), ("ndiag", C.c_int),
                ("am3", C.c_float), ("beta", C.c_float), ("ibound", C.c_int), ("device", C.c_int)]


_v = C.c_void_p
_i = C.c_int
_f = C.c_float
_d = C.c_double
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)

# name -> (restype, argtypes); every function declared in include/thirring_b200.h
SIGNATURES = {
    "thr_create": (_i, [C.POINTER(Params), C.POINTER(_v)]),
    "thr_destroy": (_i, [_v]),
    "thr_status_string": (C.c_char_p, [_i]),
    "thr_set_am3": (_i, [_v, _f]),
    "thr_set_beta": (_i, [_v, _f]),
    "thr_host_register": (_i, [_v, C.c_ulonglong]),
    "thr_host_unregister": (_i, [_v]),
    "thr_coef": (_i, [_v, _v, _v]),
    "thr_set_links": (_i, [_v, _v]),
    "thr_dslash": (_i, [_v, _v, _v, _v, _f, _i]),
    "thr_dslashd": (_i, [_v, _v, _v, _v, _f, _i]),
    "thr_congrad": (_i, [_v, _v, _v, _f, _pi, _f, _i, _pi]),
    "thr_congrad_static": (_i, [C.POINTER(Params), _v, _v, _v, _f, _pi, _f, _i, _pi, _v]),
    "thr_congrad_multi": (_i, [_v, _v, _v, _i, _f, _f, _i, _i, _v, _pi]),
    "thr_congrad_multi_dev": (_i, [_v, _v, _v, _i, _f, _f, _i, _i, _v, _pi]),
    "thr_pack_create": (_i, [_i, C.POINTER(Params), _i, C.POINTER(_v)]),
    "thr_pack_destroy": (_i, [_v]),
    "thr_pack_upload": (_i, [_v, _i, _v, _v, _v]),
    "thr_pack_congrad": (_i, [_v, _f, _f, _i, _i, _v, _pi]),
    "thr_pack_download": (_i, [_v, _i, _v]),
    "thr_pack_zero_x": (_i, [_v]),
    "thr_pack_get_stream": (_i, [_v, C.POINTER(_v)]),
    "thr_meson": (_i, [_v, _f, _f, _i, _i, _i, _v, _v, _v, _v, _pd, _pi, C.POINTER(C.c_float)]),
    "thr_fermion": (_i, [_v, _f, _f, _i, _i, _i, _v, _v, _pi, C.POINTER(C.c_float)]),
    "thr_measure": (_i, [_v, _i, _f, _f, _i, _i, _i, C.POINTER(C.c_float), C.POINTER(C.c_float),
                         C.POINTER(C.c_float), _v, _v]),
    "thr_zolo_coeffs": (_i, [_i, _d, _d, _v]),
    "thr_prep_zolo": (_i, [_v, _d, _d]),
    "thr_zolo_get": (_i, [_v, _v]),
    "thr_odslash": (_i, [_v, _v, _v, _v, _f, _i]),
    "thr_odslashd": (_i, [_v, _v, _v, _v, _f, _i]),
    "thr_congrad_o": (_i, [_v, _v, _v, _f, _pi, _f, _i, _pi]),
    "thr_odslash_dev": (_i, [_v, _v, _v, _f, _i, _i]),
    "thr_multishift_solver": (_i, [_v, _v, _f, _i, _i, _v, _v, _v, _v, _f, _i, _pi, _v]),
    "thr_multishift_solver_sp": (_i, [_v, _v, _f, _i, _i, _v, _v, _v, _v, _f, _i, _pi, _v]),
    "thr_qmrherm": (_i, [_v, _v, _v, _f, _pi, _f, _i, _v, _v, _i, _i, _i, _v, _v, _v, _i]),
    "thr_derivs": (_i, [_v, _v, _v, _d, _i, _f, _i, _v]),
    "thr_init_random": (_i, [_v, _d, _i]),
    "thr_gauss0": (_i, [_v, _v]),
    "thr_gaussp": (_i, [_v, _v]),
    "thr_rano": (_i, [_v, _i, _i, _i, C.POINTER(C.c_float)]),
    "thr_rranget": (_i, [_v, _pd]),
    "thr_rng_state_bytes": (_i, [_v, C.POINTER(C.c_ulonglong)]),
    "thr_rng_save": (_i, [_v, _v]),
    "thr_rng_load": (_i, [_v, _v]),
    "thr_read_con": (_i, [C.c_char_p, _i, _i, _i, _v, _pd, _pi]),
    "thr_write_con": (_i, [C.c_char_p, _i, _i, _i, _v, _d, _i]),
    "thr_readseed": (_i, [C.c_char_p, _pd]),
    "thr_saveseed": (_i, [C.c_char_p, _d]),
    "thr_set_remez": (_i, [_v, _i] + [_v] * 8 + [_i] + [_v] * 8),
    "thr_set_residuals": (_i, [_v, _f, _f, _i, _i]),
    "thr_set_action_precision": (_i, [_v, _i]),
    "thr_force": (_i, [_v, _v, _f, _f, _i, _v, _v]),
    "thr_hamilton": (_i, [_v, _v, _pd, _pd, _pd, _pd, _f, _f, _i, _v, _v]),
    "thr_initialise_phi": (_i, [_v, _v, _f, _i]),
    "thr_initialise_pp": (_i, [_v, _v]),
    "thr_evolve_theta_pp": (_i, [_v, _i, _f, _v, _v, _f, _f, _i, _pi, _v, _v, _v, _i]),
    "thr_trajectory": (_i, [_v, _v, _i, _f, _f, _i, _i, _v]),
    "thr_md_counters": (_i, [_v, _v, _i]),
    "thr_field_create": (_i, [_v, _i, C.POINTER(_v)]),
    "thr_field_destroy": (_i, [_v, _v]),
    "thr_field_upload": (_i, [_v, _v, _i, _v]),
    "thr_field_download": (_i, [_v, _v, _v, _i]),
    "thr_dslash_dev": (_i, [_v, _v, _v, _i, _f, _i, _i]),
    "thr_qmrherm_dev": (_i, [_v, _v, _v, _f, _pi, _f, _i, _v, _v, _i, _i, _i, _v]),
    "thr_dslash_fused_dev": (_i, [_v, _v, _v, _v, _d, _i, _f, _i, _i, _i, _pd]),
    "thr_shift_residuals_dev": (_i, [_v, _v, _v, _i, _v, _f, _i, _v]),
    "thr_derivs_dev": (_i, [_v, _v, _v, _d, _i, _f, _i]),
    "thr_phi_draw_dev": (_i, [_v, _v]),
    "thr_set_solver": (_i, [_v, _i]),
    "thr_set_mixed": (_i, [_v, _d, _d]),
    "thr_mixed_switched_at": (_i, [_v, _pi]),
    "thr_profile": (_i, [_v, _i, _i]),
    "thr_profile_read": (_i, [_v, _i, _pi, _pd, _pd, _pd]),
    "thr_tune_report": (_i, [C.c_char_p, _i]),
    "thr_stencil_timeouts": (_i, [_v, C.POINTER(C.c_ulonglong)]),
    "thr_sync": (_i, [_v]),
    "thr_get_stream": (_i, [_v, C.POINTER(_v)]),
}


def header_functions(path=HEADER):
    """Names of all functions declared in the C header."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|void)\s*\**\s*(thr_\w+)\s*\(", txt, flags=re.M)))


class LibraryMissing(RuntimeError):
    pass


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise LibraryMissing(
            f"{path} is not built; run `python thirring-rhmc_b200/build.py` (the CUDA library is required)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB
