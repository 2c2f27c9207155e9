"""ctypes binding of libcsrst_gpu.so (the C ABI in include/csrst.h).

The library is the product: there is no CPU path behind these calls.  If
the shared library is missing or cannot be loaded, every call raises.
"""
import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "libcsrst_gpu.so"

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)
U8 = C.POINTER(C.c_uint8)
F32 = C.POINTER(C.c_float)
I64 = C.POINTER(C.c_longlong)


class Config(C.Structure):
    """csrst_config: run set-up mirroring src/main.cpp:111-136."""
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("shape_order", C.c_int), ("flags", C.c_int),
                ("length_before", C.c_double), ("length_after", C.c_double),
                ("width", C.c_double), ("phi_deg", C.c_double), ("ekin_mev", C.c_double),
                ("bz", C.c_double), ("dt", C.c_double), ("charge_mass", C.c_double)]


ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "geometry",
          -4: "no particles", -5: "window fit", -6: "window move", -7: "crossings",
          -8: "window wall", -9: "i/o", -10: "field staging", 1: "outside the patch"}


class CsrstError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"csrst error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_LIB = None


def lib():
    """Loads the CUDA library once; raises if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not SO.exists():
        raise RuntimeError(f"{SO} is missing: build it with `python -m csrst_b200.build`")
    L = C.CDLL(str(SO))
    P = C.c_void_p
    sig = {
        "csrst_create": ([C.POINTER(Config), C.POINTER(P)], C.c_int),
        "csrst_destroy": ([P], C.c_int),
        "csrst_get_error": ([P, C.c_char_p, C.c_size_t], C.c_int),
        "csrst_stream": ([P], C.c_void_p),
        "csrst_sync": ([P], C.c_int),
        "csrst_get_info": ([P, D], C.c_int),
        "csrst_get_geometry": ([P, U8, D, C.c_long, C.POINTER(C.c_long)], C.c_int),
        "csrst_set_static_fields": ([P, D, D, D, D], C.c_int),
        "csrst_get_static_fields": ([P, D, D, D, D], C.c_int),
        "csrst_reset_outside": ([P], C.c_int),
        "csrst_load_particles": ([P, D, D, D, D, D, C.c_size_t], C.c_int),
        "csrst_initial_fields": ([P, C.c_double, C.c_double, C.c_int, D], C.c_int),
        "csrst_ensemble_create": ([C.POINTER(P), C.c_int, C.POINTER(P)], C.c_int),
        "csrst_ensemble_destroy": ([P], C.c_int),
        "csrst_ensemble_get_error": ([P, C.c_char_p, C.c_size_t], C.c_int),
        "csrst_ensemble_stream": ([P], C.c_void_p),
        "csrst_ensemble_step": ([P, C.c_int], C.c_int),
        "csrst_ensemble_sync": ([P, I], C.c_int),
        "csrst_ensemble_set_shape": ([P, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
        "csrst_ensemble_tune": ([P, C.c_int, D, C.c_int, I], C.c_int),
        "csrst_gemm_bf16": ([P, C.c_longlong, C.c_longlong, P, C.c_longlong, C.c_longlong, C.c_int, C.c_int,
                             C.c_int, C.c_int, P, P, P], C.c_int),
        "csrst_gemm_bf16_ex": ([P, C.c_longlong, C.c_longlong, C.c_int, P, C.c_longlong, C.c_longlong, C.c_int,
                                C.c_int, C.c_int, C.c_int, P, P, P], C.c_int),
        "csrst_gemm_set_wait_limit": ([C.c_longlong], C.c_int),
        "csrst_gemm_bf16_dual": ([P, C.c_longlong, C.c_longlong, P, C.c_longlong, C.c_longlong, C.c_int, P,
                                  C.c_longlong, C.c_longlong, P, C.c_longlong, C.c_longlong, C.c_int, C.c_int,
                                  C.c_int, C.c_int, P, P, P], C.c_int),
        "csrst_nn_transpose_bf16": ([P, P, C.c_int, C.c_int, C.c_int, C.c_int, P], C.c_int),
        "csrst_nn_transpose_b32": ([P, P, C.c_int, C.c_int, C.c_int, C.c_int, P], C.c_int),
        "csrst_nn_gelu_bwd": ([P, P, P, P, C.c_longlong, P], C.c_int),
        "csrst_nn_cast_bf16": ([P, P, C.c_longlong, P], C.c_int),
        "csrst_nn_colsum": ([P, C.c_int, C.c_int, P, P, C.c_int, P], C.c_int),
        "csrst_nn_mse": ([P, P, P, C.c_longlong, P, C.c_int, C.c_longlong, C.c_longlong, P, P, P], C.c_int),
        "csrst_nn_adam_tick": ([P, P, C.c_float, C.c_float, C.c_int, C.c_float, C.c_float, P], C.c_int),
        "csrst_nn_adam": ([P, P, P, P, C.c_longlong, P, C.c_float, C.c_float, C.c_float, P], C.c_int),
        "csrst_nn_spectral_pack": ([P, P, C.c_int, C.c_int, P, P, P], C.c_int),
        "csrst_nn_spectral_unpack": ([P, C.c_int, C.c_int, P, P, P], C.c_int),
        "csrst_get_particles": ([P, D, D, D, D], C.c_int),
        "csrst_get_old_positions": ([P, D, D], C.c_int),
        "csrst_get_window": ([P, I, D, I], C.c_int),
        "csrst_get_window_field": ([P, C.c_int, D], C.c_int),
        "csrst_set_pml": ([P, C.c_int, C.c_int, C.c_double], C.c_int),
        "csrst_get_pml": ([P, I, I], C.c_int),
        "csrst_push": ([P, C.c_int], C.c_int),
        "csrst_drift": ([P, C.c_double], C.c_int),
        "csrst_half_h": ([P], C.c_int),
        "csrst_update_e": ([P, C.c_int], C.c_int),
        "csrst_move_window": ([P], C.c_int),
        "csrst_step_first": ([P], C.c_int),
        "csrst_step_second": ([P], C.c_int),
        "csrst_step": ([P, C.c_int], C.c_int),
        "csrst_step_timed": ([P, D], C.c_int),
        "csrst_set_staging_wait_limit": ([C.c_longlong], C.c_int),
        "csrst_release_memory": ([], C.c_int),
        "csrst_diag_moments": ([P, D], C.c_int),
        "csrst_diag_wake": ([P, D, C.c_int], C.c_int),
        "csrst_diag_wake_async": ([P, P, C.c_int, P], C.c_int),
        "csrst_diag_field_energy": ([P, C.c_int, D], C.c_int),
        "csrst_diag_line_fields": ([P, C.c_int, D, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "csrst_get_num_particles": ([P, C.POINTER(C.c_longlong)], C.c_int),
        "csrst_checkpoint_write": ([P, C.c_char_p, C.c_longlong, C.c_double], C.c_int),
        "csrst_checkpoint_read": ([P, C.c_char_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double)], C.c_int),
        "csrst_gather": ([C.c_int, C.c_int, D, C.c_int, C.c_int, D, D, D, D, C.c_size_t, D], C.c_int),
        "csrst_deposit": ([C.c_int, C.c_int, D, D, D, D, D, C.c_size_t, D, D, C.c_double, C.c_int,
                           C.c_int, C.c_int, C.c_int, C.c_double, D], C.c_int),
        "csrst_charge_diff": ([C.c_int, D, D, D, D, D, C.c_size_t, D, D, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_double, D], C.c_int),
        "csrst_flux32": ([C.c_int, C.c_int, I, F32, F32, I, F32, F32, F32, C.c_size_t, C.c_double, C.c_int,
                          C.c_int, C.c_int, C.c_int, I64, I64], C.c_int),
        "csrst_get_bunch32": ([P, C.c_int, I, F32, F32, F32, F32, F32], C.c_int),
        "csrst_deposit_noalloc": ([C.c_int, C.c_int, P, P, P, P, P, C.c_size_t, D, D, C.c_double,
                                   C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, P, P], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def exported_symbols():
    """Names of the entry points the binding declares (all must be exported)."""
    lib()
    return [n for n in dir(_LIB) if n.startswith("csrst_")]


def ptr(a):
    return a.ctypes.data_as(D)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class CsrstWarning(UserWarning):
    """A call that succeeded with a positive CSRST_W_* status."""


def check(code, handle=None):
    """Raises CsrstError on a negative status; a positive one (the call
    succeeded, e.g. CSRST_W_OUTSIDE) is issued as a CsrstWarning."""
    if code != 0:
        buf = C.create_string_buffer(512)
        lib().csrst_get_error(handle, buf, 512)
        msg = buf.value.decode(errors="replace")
        if code > 0:
            import warnings
            warnings.warn(f"csrst warning {code} ({ERRORS.get(code, '?')}): {msg}", CsrstWarning, stacklevel=3)
            return
        raise CsrstError(code, msg)
