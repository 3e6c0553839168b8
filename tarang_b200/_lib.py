"""ctypes binding of the C ABI declared in include/tarang_gpu.h.

Loading fails loudly when the in-tree library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtarang_gpu.so")

TG_OK = 0
TG_ERR_ARG = -1
TG_ERR_OOM = -2
TG_ERR_NONFINITE = -3
TG_ERR_CUDA = -4
TG_ERR_UNSUPPORTED = -5
TG_ERR_TIMEOUT = -6
TG_DEBUG_SHORT_TMA_WAIT = 1
TG_ERR_STATE = -7
TG_ERR_BUSY = -8

TG_FOUR, TG_SCFT = 0, 1
TG_FLUID, TG_MHD, TG_SCALAR, TG_RB = 0, 1, 2, 3
TG_FP64, TG_FP32_MIXED = 0, 1
TG_EULER, TG_RK2, TG_RK4 = 1, 2, 4
TG_FORCE_DECAY, TG_FORCE_ENERGY_SUPPLY, TG_FORCE_MODES, TG_FORCE_CORIOLIS, TG_FORCE_RB = 0, 1, 5, 21, 51
TG_FORCE_ENERGY_HELICITY = 2
TG_FORCE_LIQUID_METAL = 101
TG_FORCE_RB_ROTATION = 52
TG_FORCE_MODES_KMAX = 64
TG_RING_MAX_SECTORS = 64
TG_RB_PRLARGE, TG_RB_PRSMALL = 0, 1
TG_RB_ULARGE, TG_RB_USMALL = 0, 1

TG_V1, TG_V2, TG_V3 = 0, 1, 2
TG_W1, TG_W2, TG_W3 = 3, 4, 5
TG_T = 6
TG_NLIN1, TG_NLIN2, TG_NLIN3 = 7, 8, 9
TG_WNLIN1, TG_WNLIN2, TG_WNLIN3 = 10, 11, 12
TG_TNLIN = 13
TG_PRESSURE = 14
TG_FORCE1, TG_FORCE2, TG_FORCE3 = 15, 16, 17
TG_WORK0 = 24
TG_NWORK = 8
TG_NFIELDS = 32

TG_ET_UU, TG_ET_BB, TG_ET_UB, TG_ET_BU, TG_ET_TT, TG_ET_ZP, TG_ET_ZM = 0, 1, 2, 3, 4, 5, 6

TG_REQ_QUEUED, TG_REQ_RUNNING, TG_REQ_DONE, TG_REQ_FAILED = 0, 1, 2, 3

ERR_NAMES = {
    TG_ERR_ARG: "TG_ERR_ARG", TG_ERR_OOM: "TG_ERR_OOM", TG_ERR_NONFINITE: "TG_ERR_NONFINITE",
    TG_ERR_CUDA: "TG_ERR_CUDA", TG_ERR_UNSUPPORTED: "TG_ERR_UNSUPPORTED",
    TG_ERR_TIMEOUT: "TG_ERR_TIMEOUT", TG_ERR_STATE: "TG_ERR_STATE", TG_ERR_BUSY: "TG_ERR_BUSY",
}


class tg_config(C.Structure):
    _fields_ = [
        ("N", C.c_int * 3),
        ("basis", C.c_int),
        ("physics", C.c_int),
        ("precision", C.c_int),
        ("dealias", C.c_int),
        ("scheme", C.c_int),
        ("kfactor", C.c_double * 3),
        ("nu", C.c_double),
        ("eta", C.c_double),
        ("kappa", C.c_double),
        ("dt", C.c_double),
        ("force_kind", C.c_int),
        ("force_para", C.c_double * 6),
        ("n_shells", C.c_int),
        ("rb_ra", C.c_double),
        ("rb_pr", C.c_double),
        ("device", C.c_int),
        ("stream", C.c_void_p),
        ("rb_pr_switch", C.c_int),
        ("rb_u_scaling", C.c_int),
        ("rb_temp_grad", C.c_double),
        ("hyper_nu", C.c_double),
        ("hyper_eta", C.c_double),
        ("hyper_kappa", C.c_double),
    ]


class tg_server_config(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_size_t),
        ("max_batch", C.c_int),
        ("device", C.c_int),
        ("use_graphs", C.c_int),
        ("keep_results", C.c_int),
        ("borrow_inputs", C.c_int),
    ]


class tg_request(C.Structure):
    _fields_ = [
        ("cfg", tg_config),
        ("n_steps", C.c_int),
        ("init", C.POINTER(C.c_double)),
        ("n_doubles", C.c_size_t),
    ]


class tg_request_status(C.Structure):
    _fields_ = [
        ("state", C.c_int),
        ("error", C.c_int),
        ("steps_done", C.c_int),
        ("submit_s", C.c_double),
        ("start_s", C.c_double),
        ("finish_s", C.c_double),
        ("final_energy", C.c_double),
        ("t_final", C.c_double),
    ]


class tg_server_stats(C.Structure):
    _fields_ = [
        ("bytes_resident", C.c_size_t),
        ("bytes_peak", C.c_size_t),
        ("n_batches", C.c_int),
        ("n_running", C.c_int),
        ("n_queued", C.c_int),
        ("rounds", C.c_longlong),
        ("request_steps", C.c_longlong),
        ("graph_launches", C.c_longlong),
        ("eager_steps", C.c_longlong),
    ]


TG_SLAB_MAX_RANKS = 64
TG_SLAB_INV_SEND, TG_SLAB_INV_RECV, TG_SLAB_FWD_SEND, TG_SLAB_FWD_RECV = 0, 1, 2, 3
TG_SLAB_SUMS, TG_SLAB_GLOBAL_SUMS = 4, 5


class tg_slab_info(C.Structure):
    _fields_ = [
        ("world", C.c_int), ("rank", C.c_int),
        ("x0", C.c_int), ("nx", C.c_int), ("y0", C.c_int), ("ny", C.c_int),
        ("xs", C.c_int * TG_SLAB_MAX_RANKS), ("xn", C.c_int * TG_SLAB_MAX_RANKS),
        ("ys", C.c_int * TG_SLAB_MAX_RANKS), ("yn", C.c_int * TG_SLAB_MAX_RANKS),
        ("nkx", C.c_int), ("nky", C.c_int), ("nkz", C.c_int), ("kzp", C.c_int),
        ("nin", C.c_int), ("nprod", C.c_int),
        ("elem_bytes", C.c_size_t),
    ]


class tg_batch_stat(C.Structure):
    _fields_ = [
        ("N", C.c_int * 3),
        ("basis", C.c_int),
        ("physics", C.c_int),
        ("precision", C.c_int),
        ("capacity", C.c_int),
        ("n_active", C.c_int),
        ("step_ms_n_active", C.c_int),
        ("step_ms", C.c_double),
        ("device_ms", C.c_double),
        ("steps", C.c_longlong),
    ]


class tg_kernel_stat(C.Structure):
    _fields_ = [
        ("name", C.c_char * 48),
        ("launches", C.c_int),
        ("total_ms", C.c_double),
        ("bytes_per_launch", C.c_double),
    ]


# name -> (restype, argtypes)
_DP = C.POINTER(C.c_double)
_VP = C.c_void_p
SIGNATURES = {
    "tg_config_default": (None, [C.POINTER(tg_config)]),
    "tg_ctx_create": (C.c_int, [C.POINTER(tg_config), C.POINTER(_VP)]),
    "tg_ctx_destroy": (C.c_int, [_VP]),
    "tg_last_error": (C.c_char_p, [_VP]),
    "tg_synchronize": (C.c_int, [_VP]),
    "tg_device_bytes": (C.c_int, [_VP, C.POINTER(C.c_size_t)]),
    "tg_field_upload": (C.c_int, [_VP, C.c_int, _DP, C.c_size_t]),
    "tg_field_download": (C.c_int, [_VP, C.c_int, _DP, C.c_size_t]),
    "tg_field_download_stored": (C.c_int, [_VP, C.c_int, _DP, C.c_size_t]),
    "tg_field_copy": (C.c_int, [_VP, C.c_int, C.c_int]),
    "tg_field_alloc": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "tg_write_field_file": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(C.c_int), C.c_int, C.POINTER(_DP), C.c_int, C.c_int]),
    "tg_read_field_file": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(_DP), C.c_int]),
    "tg_field_free": (C.c_int, [_VP, C.c_int]),
    "tg_write_field_file_reduced": (C.c_int, [C.c_char_p, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(_DP), C.c_int, C.c_int]),
    "tg_read_field_file_reduced": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(_DP), C.c_int]),
    "tg_forward_transform": (C.c_int, [_VP, C.c_int, C.c_int]),
    "tg_inverse_transform": (C.c_int, [_VP, C.c_int, C.c_int]),
    "tg_compute_force": (C.c_int, [_VP]),
    "tg_compute_nlin": (C.c_int, [_VP]),
    "tg_add_force": (C.c_int, [_VP]),
    "tg_set_force_modes": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), _DP]),
    "tg_compute_pressure": (C.c_int, [_VP]),
    "tg_compute_rhs": (C.c_int, [_VP]),
    "tg_get_dt": (C.c_int, [_VP, _DP]),
    "tg_time_advance": (C.c_int, [_VP]),
    "tg_step": (C.c_int, [_VP, C.c_int, _DP]),
    "tg_time": (C.c_int, [_VP, _DP, C.POINTER(C.c_longlong)]),
    "tg_energy": (C.c_int, [_VP, C.c_int, _DP, _DP]),
    "tg_shell_spectrum": (C.c_int, [_VP, C.c_int, _DP, _DP, C.c_int]),
    "tg_et_radii": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_ring_sizes": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "tg_ring_spectrum": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, C.c_int]),
    "tg_cylinder_ring_spectrum": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, C.c_int]),
    "tg_ring_radii": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "tg_shell_spectrum_helicity": (C.c_int, [_VP, C.c_int, _DP, _DP, _DP, C.c_int]),
    "tg_ring_spectrum_helicity": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_cylinder_ring_spectrum_helicity": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_helicity_flux": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_magnetic_helicity_flux": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_helicity_shell_to_shell": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_magnetic_helicity_shell_to_shell": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_ring_to_ring": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_cylinder_radii": (C.c_int, [_VP, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_cylinder_ring_to_ring": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_flux": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "tg_shell_to_shell": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "tg_nusselt": (C.c_int, [_VP, _DP]),
    "tg_force_feed": (C.c_int, [_VP, _DP, C.c_int]),
    "tg_force_feed_group": (C.c_int, [_VP, C.c_int, _DP, C.c_int]),
    "tg_force_feed_ring": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _DP, C.c_int]),
    "tg_energy_noalloc": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, _VP, _VP]),
    "tg_profile_enable": (C.c_int, [_VP, C.c_int]),
    "tg_debug_set": (C.c_int, [_VP, C.c_int, C.c_longlong]),
    "tg_profile_read": (C.c_int, [_VP, C.POINTER(tg_kernel_stat), C.c_int, C.POINTER(C.c_int)]),
    "tg_server_create": (C.c_int, [C.POINTER(tg_server_config), C.POINTER(_VP)]),
    "tg_server_destroy": (C.c_int, [_VP]),
    "tg_server_submit": (C.c_int, [_VP, C.POINTER(tg_request), C.POINTER(C.c_longlong)]),
    "tg_server_pump": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "tg_server_pump_begin": (C.c_int, [_VP]),
    "tg_server_pump_end": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "tg_server_drain": (C.c_int, [_VP, C.c_longlong]),
    "tg_server_poll": (C.c_int, [_VP, C.c_longlong, C.POINTER(tg_request_status)]),
    "tg_server_result": (C.c_int, [_VP, C.c_longlong, _DP, C.c_size_t]),
    "tg_server_release": (C.c_int, [_VP, C.c_longlong]),
    "tg_server_take_finished": (C.c_int, [_VP, C.POINTER(C.c_longlong), C.c_int, C.POINTER(C.c_int)]),
    "tg_server_stats_get": (C.c_int, [_VP, C.POINTER(tg_server_stats)]),
    "tg_server_batch_stats": (C.c_int, [_VP, C.POINTER(tg_batch_stat), C.c_int, C.POINTER(C.c_int)]),
    "tg_slab_create": (C.c_int, [C.POINTER(tg_config), C.c_int, C.c_int, C.POINTER(_VP)]),
    "tg_slab_info_get": (C.c_int, [_VP, C.POINTER(tg_slab_info)]),
    "tg_slab_buffer": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(_VP)]),
    "tg_slab_phase": (C.c_int, [_VP, C.c_int, C.c_int]),
    "tg_slab_upload": (C.c_int, [_VP, C.c_int, _DP]),
    "tg_slab_download": (C.c_int, [_VP, C.c_int, _DP]),
    "tg_slab_scalars": (C.c_int, [_VP, _DP, _DP]),
    "tg_server_clock": (C.c_double, [_VP]),
    "tg_request_bytes": (C.c_int, [C.POINTER(tg_config), C.c_int, C.POINTER(C.c_size_t)]),
}

_lib = None


def load(path: str | None = None):
    """Load the in-tree library (raises if it is missing: the product has no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"tarang_b200: CUDA library {p} is missing; run `python -m tarang_b200.build`")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TarangError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code
