"""Loads libcoral_b200.so (the C-ABI of include/coral_b200.h) with ctypes.

There is no fallback: if the library is missing or fails to load, importing the
solver raises.  Build it with ``python -m coral_b200.build``.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcoral_b200.so")

ERRORS = {
    -1: "CORAL_EBADARG", -2: "CORAL_ENOMEM", -3: "CORAL_ECUDA", -4: "CORAL_ESINGULAR",
    -5: "CORAL_ENONFINITE", -6: "CORAL_EPARSE", -7: "CORAL_EIO", -8: "CORAL_EUNSUPPORTED",
    -9: "CORAL_ENODEV",
}

# every function declared in include/coral_b200.h with (restype, argtypes)
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "coral_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P)]),
    "coral_create_from_files": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                               ctypes.POINTER(_P)]),
    "coral_create_with_args": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                              ctypes.c_char_p, ctypes.POINTER(_P)]),
    "coral_destroy": (None, [_P]),
    "coral_last_error": (ctypes.c_char_p, [_P]),
    "coral_query": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "coral_factorize": (ctypes.c_int, [_P, ctypes.c_double]),
    "coral_march": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int]),
    "coral_synchronize": (ctypes.c_int, [_P]),
    "coral_get_field": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_set_field": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_get_mean_field": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_set_mean_field": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_spec_to_phys": (ctypes.c_int, [_P, _D, _D]),
    "coral_phys_to_spec": (ctypes.c_int, [_P, _D, _D]),
    "coral_get_full_phys": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_import_quicksave": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int]),
    "coral_export_checkpoint": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int]),
    "coral_diagnostics": (ctypes.c_int, [_P, _D]),
    "coral_set_var_phys": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _D]),
    "coral_set_mean_var_profile": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _D]),
    "coral_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "coral_profile_step": (ctypes.c_int, [_P, ctypes.c_double, _D, ctypes.c_int]),
    "coral_spec_to_phys_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _P]),
    "coral_set_timeseries": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "coral_set_timeseries_from_file": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "coral_set_usr_output": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "coral_set_usr_output_from_file": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "coral_export_usr_output": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_longlong]),
    "coral_timeseries": (ctypes.c_int, [_P, _D, ctypes.c_int]),
    "coral_set_time": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_longlong]),
    "coral_get_time": (ctypes.c_int, [_P, _D]),
    "coral_run": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p]),
    "coral_set_z_transform": (ctypes.c_int, [_P, ctypes.c_int]),
    "coral_set_source": (ctypes.c_int, [_P, ctypes.c_int, _D]),
    "coral_set_penalisation_mask": (ctypes.c_int, [_P, _D]),
    "coral_set_hermitian_kx0": (ctypes.c_int, [_P, ctypes.c_int]),
    "coral_var_positions": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]),
    "coral_ensemble_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                             ctypes.POINTER(ctypes.c_char_p), ctypes.c_char_p, ctypes.c_int,
                                             ctypes.POINTER(_P)]),
    "coral_ensemble_destroy": (None, [_P]),
    "coral_ensemble_last_error": (ctypes.c_char_p, [_P]),
    "coral_ensemble_member": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P)]),
    "coral_ensemble_march": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int]),
    "coral_ensemble_synchronize": (ctypes.c_int, [_P]),
    "coral_ensemble_query": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    "coral_closure_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(_P)]),
    "coral_closure_destroy": (None, [_P]),
    "coral_closure_last_error": (ctypes.c_char_p, [_P]),
    "coral_closure_param_count": (ctypes.c_int, []),
    "coral_closure_set_scales": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "coral_closure_get_params": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "coral_closure_set_params": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "coral_closure_get_gradient": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "coral_closure_zero_gradient": (ctypes.c_int, [_P]),
    "coral_closure_train": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P,
                                           ctypes.c_longlong, ctypes.c_float, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]),
    "coral_closure_infer": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P]),
    "coral_closure_attach": (ctypes.c_int, [_P, _P]),
    "coral_autotune": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "coral_set_variant": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int]),
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcoral_b200.so not found at %s; build it with `python -m coral_b200.build`" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
