"""ctypes binding of libwamgpu.so (the C ABI declared in include/wamgpu.h)."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwamgpu.so")

# exported entry points and their C signatures
c_int, c_float, c_void_p, c_char_p = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_char_p
PI, PF = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)


class WamgpuConfig(ctypes.Structure):
    """struct wamgpu_config (include/wamgpu.h)."""
    _fields_ = [("kl", c_int), ("ml", c_int), ("fr1", ctypes.c_double), ("iref", c_int), ("iphys", c_int),
                ("shallow_run", c_int), ("spherical_run", c_int), ("refraction_d_run", c_int),
                ("refraction_c_run", c_int), ("reduced_grid", c_int), ("isnonlin", c_int), ("lcflx", c_int),
                ("idelt", c_int), ("idelpro", c_int), ("betamax", ctypes.c_double), ("zalp", ctypes.c_double),
                ("alpha", ctypes.c_double), ("tauwshelter", ctypes.c_double), ("cdfac", ctypes.c_double),
                ("ndepth", c_int), ("deptha", ctypes.c_double), ("depthd", ctypes.c_double),
                ("delphi", ctypes.c_double), ("precision", c_int), ("device", c_int)]


class RestartDates(ctypes.Structure):
    """struct wamgpu_restart_dates: CHARACTER(14) dates, blank-padded."""
    _fields_ = [("cdtpro", ctypes.c_char * 14), ("cdtsou", ctypes.c_char * 14), ("cda", ctypes.c_char * 14),
                ("cdta", ctypes.c_char * 14), ("cdca", ctypes.c_char * 14)]


SIGNATURES = {
    "wamgpu_create": (c_int, [ctypes.POINTER(WamgpuConfig), ctypes.POINTER(c_void_p)]),
    "wamgpu_destroy": (c_int, [c_void_p]),
    "wamgpu_last_error": (c_char_p, [c_void_p]),
    "wamgpu_config_size": (c_int, []),
    "wamgpu_get_table": (c_int, [c_void_p, c_char_p, PF, PI]),
    "wamgpu_host_table": (c_int, [ctypes.POINTER(WamgpuConfig), c_char_p, PF, PI]),
    "wamgpu_set_grid": (c_int, [c_void_p, c_int, PI, PI, PF, PI, c_int, PF, PF, PF]),
    "wamgpu_set_depth": (c_int, [c_void_p, PF]),
    "wamgpu_set_current": (c_int, [c_void_p, PF, PF]),
    "wamgpu_prepare_propagation": (c_int, [c_void_p, PF, PI]),
    "wamgpu_prepare_source": (c_int, [c_void_p]),
    "wamgpu_get_indep": (c_int, [c_void_p, PI]),
    "wamgpu_implsch_host": (c_int, [c_void_p, PF, PF, PF, PF, PF, PF, PF, PF, PF, PI]),
    "wamgpu_propags_host": (c_int, [c_void_p, PF]),
    "wamgpu_implsch_dev": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p]),
    "wamgpu_propags_dev": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "wamgpu_propags_dev_static": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "wamgpu_step_dev": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p]),
    "wamgpu_step_host": (c_int, [c_void_p, PF, c_int, PF, PF, PF, PF, PF, PF, PF]),
    "wamgpu_get_fluxes": (c_int, [c_void_p, PF]),
    "wamgpu_sync": (c_int, [c_void_p]),
    "wamgpu_set_diagnostics": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "wamgpu_restart_write": (c_int, [c_void_p, c_char_p, c_void_p, c_int] + [c_void_p] * 6 +
                             [ctypes.POINTER(RestartDates), PI]),
    "wamgpu_restart_read": (c_int, [c_void_p, c_char_p, c_void_p, c_int] + [c_void_p] * 6 +
                            [ctypes.POINTER(RestartDates), PI]),
    "wamgpu_set_wind_grid": (c_int, [c_void_p] + [c_int] * 11 + [PI, PI]),
    "wamgpu_wind_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "wamgpu_put_points_dev": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, ctypes.c_double, c_void_p]),
    "wamgpu_output_parameters_dev": (c_int, [c_void_p, c_void_p, c_int] + [c_void_p] * 5 + [c_int, c_void_p, c_int,
                                                                                             c_void_p]),
    "wamgpu_output_swell_dev": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p]),
    "wamgpu_set_timing": (c_int, [c_void_p, c_int]),
    "wamgpu_get_timing": (c_int, [c_void_p, PF, PI]),
    "wamgpu_set_owned": (c_int, [c_void_p, c_int, c_int]),
    "wamgpu_set_counter": (c_int, [c_void_p, c_int]),
    "wamgpu_implsch_adj_dev": (c_int, [c_void_p] + [c_void_p, c_int] + [c_void_p] * 9),
    "wamgpu_implsch_tl_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_int] + [c_void_p] * 12),
    "wamgpu_propags_adj_dev": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "wamgpu_checkpoint_reserve": (c_int, [c_void_p, c_int, c_int]),
    "wamgpu_step_ckpt_dev": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_int] + [c_void_p] * 8),
    "wamgpu_step_adj_dev": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int] + [c_void_p] * 7),
    "wamgpu_propags_substep_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "wamgpu_propags_substep_range_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "wamgpu_get_halo_width": (c_int, [c_void_p]),
    "wamgpu_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_int, ctypes.POINTER(c_void_p)]),
    "wamgpu_batch_destroy": (c_int, [c_void_p]),
    "wamgpu_batch_last_error": (c_char_p, [c_void_p]),
    "wamgpu_batch_set_member": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_void_p]),
    "wamgpu_batch_tune": (c_int, [c_void_p, c_void_p, PI, PI]),
    "wamgpu_batch_step": (c_int, [c_void_p, c_void_p]),
    "wamgpu_batch_capture": (c_int, [c_void_p, c_void_p]),
    "wamgpu_batch_sync": (c_int, [c_void_p]),
}

_lib = None


class WamgpuError(RuntimeError):
    pass


def load():
    """Load the in-tree libwamgpu.so; raises if it is missing (there is no CPU path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise WamgpuError(f"{LIB_PATH} not built: run python -m wam_b200.build (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.wamgpu_config_size() != ctypes.sizeof(WamgpuConfig):
            raise WamgpuError("wamgpu_config layout mismatch between header and binding")
        _lib = L
    return _lib
