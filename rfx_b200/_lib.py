"""ctypes binding of the C ABI in ``include/rfxb200.h``.

The product path has no CPU fallback: if ``librfxb200.so`` cannot be loaded
(or built, where nvcc is available) every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librfxb200.so")

c_float_p = C.POINTER(C.c_float)
c_int32_p = C.POINTER(C.c_int32)


class RfxbDftDesc(C.Structure):
    _fields_ = [("axis", C.c_int), ("index", C.c_int), ("component", C.c_int), ("n_freqs", C.c_int)]


class RfxbFluxDesc(C.Structure):
    _fields_ = [("axis", C.c_int), ("index", C.c_int), ("lo1", C.c_int), ("hi1", C.c_int), ("lo2", C.c_int),
                ("hi2", C.c_int), ("n_freqs", C.c_int)]


class RfxbNtffDesc(C.Structure):
    _fields_ = [("i_lo", C.c_int), ("i_hi", C.c_int), ("j_lo", C.c_int), ("j_hi", C.c_int), ("k_lo", C.c_int),
                ("k_hi", C.c_int), ("n_freqs", C.c_int)]


class RfxbDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dt", C.c_double),
        ("inv_xe_host", c_float_p), ("inv_xh_host", c_float_p),
        ("inv_ye_host", c_float_p), ("inv_yh_host", c_float_p),
        ("inv_ze_host", c_float_p), ("inv_zh_host", c_float_p),
        ("cpml_layers", C.c_int),
        ("cpml_axes", C.c_uint),
        ("cpml_b_host", c_float_p), ("cpml_c_host", c_float_p), ("cpml_kappa_host", c_float_p),
        ("cpml_cell", C.c_double * 6),
        ("pec_axes", C.c_uint),
        ("n_src", C.c_int), ("src_cells_host", c_int32_p),
        ("n_probe", C.c_int), ("probe_cells_host", c_int32_p),
        ("n_dft", C.c_int), ("dft_host", C.POINTER(RfxbDftDesc)),
        ("grad_box", C.c_int * 6),
        ("n_flux", C.c_int), ("flux_host", C.POINTER(RfxbFluxDesc)),
        ("ntff_host", C.POINTER(RfxbNtffDesc)),
    ]


class RfxbLaunchConfig(C.Structure):
    _fields_ = [("fwd_split", C.c_int32), ("fwd_order", C.c_int32), ("adj_lite", C.c_int32),
                ("adj_order", C.c_int32), ("fwd_persist", C.c_int32), ("adj_persist", C.c_int32),
                ("l2_promo", C.c_int32), ("fwd_depth", C.c_int32)]


class RfxbStepIO(C.Structure):
    _fields_ = [
        ("src_wave_dev", C.c_void_p),
        ("probe_out_dev", C.c_void_p),
        ("dft_acc_dev", C.POINTER(C.c_void_p)),
        ("dft_phase_dev", C.POINTER(C.c_void_p)),
        ("flux_acc_dev", C.POINTER(C.c_void_p)),
        ("flux_kernel_dev", C.POINTER(C.c_void_p)),
        ("ntff_acc_dev", C.c_void_p),
        ("ntff_cmp_dev", C.c_void_p),
        ("ntff_phase_dev", C.c_void_p),
    ]


class RfxbAdjointIO(C.Structure):
    _fields_ = [
        ("g_dev", C.c_void_p),
        ("grad_dev", C.c_void_p),
        ("dca_dev", C.c_void_p),
        ("dcb_dev", C.c_void_p),
        ("src_adj_dev", C.c_void_p),
        ("dft_cot_dev", C.POINTER(C.c_void_p)),
        ("dft_phase_dev", C.POINTER(C.c_void_p)),
        ("ntff_cot_dev", C.c_void_p),
        ("ntff_phase_dev", C.c_void_p),
        ("flux_cot_dev", C.POINTER(C.c_void_p)),
        ("flux_kernel_dev", C.POINTER(C.c_void_p)),
    ]


# name -> (restype, argtypes); the set of exported symbols the header declares
SIGNATURES = {
    "rfxb_version": (C.c_int, []),
    "rfxb_last_error": (C.c_char_p, []),
    "rfxb_plan_create": (C.c_int, [C.POINTER(RfxbDesc), C.POINTER(C.c_void_p)]),
    "rfxb_plan_destroy": (None, [C.c_void_p]),
    "rfxb_plan_set_materials": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rfxb_plan_reset": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rfxb_plan_load_fields": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p]),
    "rfxb_plan_store_fields": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p]),
    "rfxb_plan_advance": (C.c_int, [C.c_void_p, C.POINTER(RfxbStepIO), C.c_int, C.c_int, C.c_void_p]),
    "rfxb_forward": (C.c_int, [C.c_void_p, C.POINTER(RfxbStepIO), C.POINTER(C.c_void_p), C.c_int, C.c_int,
                               C.c_void_p]),
    "rfxb_plan_record_history": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "rfxb_plan_checkpoint_reserve": (C.c_int, [C.c_void_p, C.c_int]),
    "rfxb_plan_checkpoint_save": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "rfxb_plan_checkpoint_load": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "rfxb_plan_adjoint_begin": (C.c_int, [C.c_void_p, C.POINTER(RfxbAdjointIO), C.c_int, C.c_void_p]),
    "rfxb_plan_adjoint_advance": (C.c_int, [C.c_void_p, C.POINTER(RfxbAdjointIO), C.c_int, C.c_int, C.c_void_p]),
    "rfxb_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    "rfxb_batch_destroy": (None, [C.c_void_p]),
    "rfxb_batch_advance": (C.c_int, [C.c_void_p, C.POINTER(RfxbStepIO), C.c_int, C.c_int, C.c_void_p]),
    "rfxb_batch_record_history": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "rfxb_batch_adjoint_begin": (C.c_int, [C.c_void_p, C.POINTER(RfxbAdjointIO), C.c_int, C.c_void_p]),
    "rfxb_batch_adjoint_advance": (C.c_int, [C.c_void_p, C.POINTER(RfxbAdjointIO), C.c_int, C.c_int, C.c_void_p]),
    "rfxb_plan_device_bytes": (C.c_int64, [C.c_void_p]),
    "rfxb_plan_device_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rfxb_batch_device_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rfxb_plan_box_energy": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "rfxb_plan_box_energy_weighted": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p]),
    "rfxb_plan_box_flux": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "rfxb_plan_state_bytes": (C.c_longlong, [C.c_void_p]),
    "rfxb_plan_save_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "rfxb_plan_restore_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "rfxb_plan_forward_variant": (C.c_int, [C.c_void_p]),
    "rfxb_batch_forward_variant": (C.c_int, [C.c_void_p]),
    "rfxb_plan_adjoint_variant": (C.c_int, [C.c_void_p]),
    "rfxb_batch_adjoint_variant": (C.c_int, [C.c_void_p]),
    "rfxb_plan_step_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "rfxb_batch_step_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "rfxb_plan_launch_config": (C.c_int, [C.c_void_p, C.POINTER(RfxbLaunchConfig), C.POINTER(RfxbLaunchConfig)]),
    "rfxb_plan_set_launch_config": (C.c_int, [C.c_void_p, C.POINTER(RfxbLaunchConfig)]),
    "rfxb_batch_launch_config": (C.c_int, [C.c_void_p, C.POINTER(RfxbLaunchConfig), C.POINTER(RfxbLaunchConfig)]),
    "rfxb_batch_set_launch_config": (C.c_int, [C.c_void_p, C.POINTER(RfxbLaunchConfig)]),
    "rfxb_debug_work_lists": (C.c_int, [C.c_int, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                        C.c_int32, C.POINTER(C.c_int32)]),
    "rfxb_batch_debug_fault": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "rfxb_batch_debug_poison": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "rfxb_forward_noalloc": (C.c_int, [C.POINTER(RfxbDesc), C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p),
                                       C.POINTER(RfxbStepIO), C.c_int, C.c_int, C.c_void_p]),
}

_lock = threading.Lock()
_lib = None


def load():
    """Load (building first if the library file is missing) and type the ABI."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int, what: str):
    if rc != 0:
        msg = load().rfxb_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed (rfxb code {rc}): {msg}")
