"""ctypes binding of ``libfftb_b200.so`` (the C ABI declared in include/fftb.h).

There is no fallback: if the shared library is missing or fails to load, every
entry point raises.  Build it with ``python -m fftm_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfftb_b200.so")

# every symbol include/fftb.h declares (checked by the CPU tests)
EXPORTS = [
    "fftb_status_string", "fftb_last_error_message", "fftb_version", "fftb_build_digest",
    "fftb_plan_create", "fftb_plan_get_work_size", "fftb_plan_set_work_area", "fftb_plan_set_stream",
    "fftb_exec", "fftb_exec_direction", "fftb_plan_describe", "fftb_plan_num_launches", "fftb_plan_destroy",
    "fftb_ffts_create", "fftb_ffts_create_ex", "fftb_ffts_profile_report", "fftb_init_options_default",
    "fftb_ffts_destroy", "fftb_ffts_dimension", "fftb_ffts_work_size",
    "fftb_ffts_set_work_area", "fftb_ffts_set_stream", "fftb_ffts_forward", "fftb_ffts_backward",
    "fftb_ffts_backward_normalized", "fftb_ffts_poisson", "fftb_ffts_filter", "fftb_ffts_spectrum_poisson",
    "fftb_ffts_num_launches", "fftb_ffts_timing_enable", "fftb_ffts_timing_read",
    "fftb_poisson3d_f32_noalloc", "fftb_ffts_forward_adjoint", "fftb_ffts_backward_adjoint",
    "fftb_batch_create", "fftb_batch_destroy", "fftb_batch_layout", "fftb_batch_work_size",
    "fftb_batch_set_work_area", "fftb_batch_set_stream", "fftb_batch_set_tuning", "fftb_batch_exec",
    "fftb_batch_status", "fftb_batch_describe", "fftb_batch_set_wait_limit", "fftb_batch_wait_selftest",
    "fftb_ffts_set_strategy", "fftb_ffts_get_strategy",
    "fftb_autotune_load_file", "fftb_autotune_save_file", "fftb_autotune_validate", "fftb_autotune_hardware", "fftb_autotune_signature",
    "fftb_autotune_ffts", "fftb_ffts_apply_config", "fftb_autotune_batch", "fftb_batch_apply_config",
    "fftb_slab_create", "fftb_slab_destroy", "fftb_slab_sizes", "fftb_slab_set_stream", "fftb_slab_set_peers",
    "fftb_slab_forward_local", "fftb_slab_forward_finish", "fftb_slab_backward_local", "fftb_slab_backward_finish",
    "fftb_ffts_spectrum_derivative", "fftb_ffts_derivative", "fftb_ffts_spectrum_truncate", "fftb_ffts_gradient",
]

_lib = None


class InitOptions(ctypes.Structure):
    """fftb_init_options (include/fftb.h): the reference's ffts_init_options."""
    _fields_ = [("profiling_key", ctypes.c_char_p), ("memory_profiling_key", ctypes.c_char_p),
                ("print_profile_summary_on_destroy", ctypes.c_int), ("print_profile_totals_on_destroy", ctypes.c_int),
                ("print_memory_profile_on_destroy", ctypes.c_int), ("print_memory_totals_on_destroy", ctypes.c_int)]


def load():
    """Loads the library (once) and declares the argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"fftb CUDA library not built: {LIB_PATH} is missing "
                          "(run `python -m fftm_b200.build`)")
    L = ctypes.CDLL(LIB_PATH)
    c_int, c_ll, c_vp, c_sz, c_d = ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double
    llp = ctypes.POINTER(c_ll)
    ip = ctypes.POINTER(c_int)
    szp = ctypes.POINTER(c_sz)
    L.fftb_status_string.argtypes = [c_int]
    L.fftb_status_string.restype = ctypes.c_char_p
    L.fftb_version.restype = ctypes.c_char_p
    L.fftb_build_digest.restype = ctypes.c_char_p
    L.fftb_last_error_message.restype = ctypes.c_char_p
    L.fftb_plan_create.argtypes = [c_int, c_int, c_int, llp, llp, c_ll, c_ll, llp, c_ll, c_ll, c_ll,
                                   ctypes.POINTER(c_vp), szp]
    L.fftb_plan_get_work_size.argtypes = [c_vp, szp]
    L.fftb_plan_set_work_area.argtypes = [c_vp, c_vp]
    L.fftb_plan_set_stream.argtypes = [c_vp, c_vp]
    L.fftb_exec.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_exec_direction.argtypes = [c_vp, c_int, c_vp, c_vp]
    L.fftb_plan_describe.argtypes = [c_vp, ip, ip, ip, llp, llp, llp, llp, llp, llp, llp, llp]
    L.fftb_plan_num_launches.argtypes = [c_vp, ip]
    L.fftb_plan_destroy.argtypes = [c_vp]
    L.fftb_ffts_create.argtypes = [c_int, c_ll, c_ll, c_ll, c_ll, c_int, ctypes.POINTER(c_vp)]
    L.fftb_ffts_destroy.argtypes = [c_vp]
    L.fftb_ffts_dimension.argtypes = [c_vp, ip]
    L.fftb_ffts_work_size.argtypes = [c_vp, szp]
    L.fftb_ffts_set_work_area.argtypes = [c_vp, c_vp]
    L.fftb_ffts_set_stream.argtypes = [c_vp, c_vp]
    L.fftb_ffts_forward.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_ffts_backward.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_ffts_backward_normalized.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_ffts_poisson.argtypes = [c_vp, c_vp, c_vp, c_d]
    L.fftb_ffts_filter.argtypes = [c_vp, c_vp, c_vp, c_d, c_d]
    L.fftb_ffts_spectrum_poisson.argtypes = [c_vp, c_vp, c_d, c_d]
    L.fftb_ffts_num_launches.argtypes = [c_vp, c_int, ip]
    L.fftb_ffts_timing_enable.argtypes = [c_vp, c_int]
    L.fftb_ffts_timing_read.argtypes = [c_vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(c_d),
                                        ctypes.c_char_p, c_int, c_int, ip]
    L.fftb_batch_create.argtypes = [c_int, c_int, llp, ctypes.POINTER(c_vp)]
    L.fftb_batch_destroy.argtypes = [c_vp]
    L.fftb_batch_layout.argtypes = [c_vp, llp, llp, llp, llp]
    L.fftb_batch_work_size.argtypes = [c_vp, szp]
    L.fftb_batch_set_work_area.argtypes = [c_vp, c_vp]
    L.fftb_batch_set_stream.argtypes = [c_vp, c_vp]
    L.fftb_batch_set_tuning.argtypes = [c_vp, c_int, c_int]
    L.fftb_batch_exec.argtypes = [c_vp, c_int, c_vp, c_vp, c_d, c_int]
    L.fftb_batch_status.argtypes = [c_vp, c_int, ip]
    L.fftb_batch_describe.argtypes = [c_vp, c_int, c_d, ip, ip, ip, ip]
    L.fftb_ffts_forward_adjoint.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_ffts_backward_adjoint.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_poisson3d_f32_noalloc.argtypes = [c_vp, c_vp, c_ll, c_ll, c_ll, c_d, c_vp]
    cp = ctypes.c_char_p
    L.fftb_ffts_set_strategy.argtypes = [c_vp, c_int, c_int]
    L.fftb_ffts_get_strategy.argtypes = [c_vp, ip, ip]
    L.fftb_autotune_load_file.argtypes = [cp, cp, c_sz, szp]
    L.fftb_autotune_save_file.argtypes = [cp, cp]
    L.fftb_autotune_validate.argtypes = [cp, cp, c_int]
    L.fftb_autotune_hardware.argtypes = [c_int, cp, c_sz, szp]
    L.fftb_autotune_signature.argtypes = [cp, cp, c_sz, szp]
    L.fftb_autotune_ffts.argtypes = [c_int, c_ll, c_ll, c_ll, c_ll, c_int, cp, c_int, c_int, c_int, cp, c_sz, szp, ip]
    L.fftb_ffts_apply_config.argtypes = [c_vp, cp]
    L.fftb_autotune_batch.argtypes = [c_vp, c_int, c_d, cp, c_int, c_int, c_int, cp, c_sz, szp, ip, ip]
    L.fftb_batch_apply_config.argtypes = [c_vp, cp, ip]
    L.fftb_ffts_spectrum_derivative.argtypes = [c_vp, c_vp, c_vp, c_int, c_d]
    L.fftb_ffts_derivative.argtypes = [c_vp, c_vp, c_vp, c_int]
    L.fftb_ffts_spectrum_truncate.argtypes = [c_vp, c_vp, c_int, c_int]
    L.fftb_ffts_gradient.argtypes = [c_vp, c_vp, ctypes.POINTER(c_vp)]
    L.fftb_batch_set_wait_limit.argtypes = [c_vp, c_ll]
    L.fftb_slab_create.argtypes = [c_int, c_ll, c_ll, c_ll, c_ll, c_int, c_int, c_int, ctypes.POINTER(c_vp)]
    L.fftb_slab_destroy.argtypes = [c_vp]
    L.fftb_slab_sizes.argtypes = [c_vp, llp, llp, llp, llp]
    L.fftb_slab_set_stream.argtypes = [c_vp, c_vp]
    L.fftb_slab_set_peers.argtypes = [c_vp, ctypes.POINTER(c_vp)]
    L.fftb_slab_forward_local.argtypes = [c_vp, c_vp, c_vp, c_vp]
    L.fftb_slab_forward_finish.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_slab_backward_local.argtypes = [c_vp, c_vp, c_vp]
    L.fftb_slab_backward_finish.argtypes = [c_vp, c_vp, c_vp, c_vp]
    L.fftb_batch_wait_selftest.argtypes = [c_ll, ip]
    L.fftb_ffts_create_ex.argtypes = [c_int, c_ll, c_ll, c_ll, c_ll, c_int, ctypes.POINTER(InitOptions),
                                      ctypes.POINTER(c_vp)]
    L.fftb_ffts_profile_report.argtypes = [c_vp, c_int, cp, c_sz, szp]
    L.fftb_init_options_default.argtypes = [ctypes.POINTER(InitOptions)]
    for name in EXPORTS:
        if name not in ("fftb_status_string", "fftb_version", "fftb_build_digest", "fftb_last_error_message"):
            getattr(L, name).restype = c_int
    L.fftb_init_options_default.restype = None
    _lib = L
    return L


def status_string(st: int) -> str:
    return load().fftb_status_string(int(st)).decode()


def last_error_message() -> str:
    return load().fftb_last_error_message().decode()
