"""ctypes binding of the in-tree CUDA library ves3d_b200/libves3d_b200.so (C ABI of
include/ves3d_b200.h). There is no CPU fallback: if the library is missing, or a call
needs a GPU that is not there, the call raises."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libves3d_b200.so")

VES3D_OK = 0
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NOMEM", 4: "ERR_STATE", 5: "ERR_NODEV", 6: "ERR_NUMERIC",
          7: "ERR_IO"}
PREC_FP64 = 0
PREC_MIXED = 1

_lib = None

_d = ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_l = ctypes.c_long
_sz = ctypes.c_size_t

# (name, restype, argtypes) for every symbol declared in include/ves3d_b200.h
SIGNATURES = [
    ("ves3d_version", _i, []),
    ("ves3d_last_error", ctypes.c_char_p, []),
    ("ves3d_kernel_launches", ctypes.c_longlong, []),
    ("ves3d_sv_create", _i, [_i, _i, _i, _i, ctypes.POINTER(_vp)]),
    ("ves3d_sv_destroy", _i, [_vp]),
    ("ves3d_sv_set_stream", _i, [_vp, _vp]),
    ("ves3d_sv_set_src_coord", _i, [_vp, _vp, _l, _i]),
    ("ves3d_sv_set_density_sl", _i, [_vp, _vp, _i]),
    ("ves3d_sv_set_density_dl", _i, [_vp, _vp, _i]),
    ("ves3d_sv_get_dl_matrix", _i, [_vp, _vp, _i]),
    ("ves3d_sv_set_order_up", _i, [_vp, _i]),
    ("ves3d_sv_set_trg_coord", _i, [_vp, _vp, _l, _i]),
    ("ves3d_sv_eval_trg", _i, [_vp, _vp, _i]),
    ("ves3d_sv_get_order_up", _i, [_vp, ctypes.POINTER(_i)]),
    ("ves3d_sv_monitor_error", _i, [_vp, _d, _vp, ctypes.POINTER(_d)]),
    ("ves3d_sv_eval", _i, [_vp, _vp, _i]),
    ("ves3d_sv_setup", _i, [_vp]),
    ("ves3d_sv_get_self_matrix", _i, [_vp, _vp, _i]),
    ("ves3d_sv_get_parts", _i, [_vp, _vp, _vp, _i]),
    ("ves3d_sv_stage_times", _i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("ves3d_sv_far_dl_time", _i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("ves3d_sv_set_near_singular", _i, [_vp, _i]),
    ("ves3d_sv_near_info", _i, [_vp, ctypes.POINTER(_d), ctypes.POINTER(ctypes.c_long)]),
    ("ves3d_sv_device_buffer", _i, [_vp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_sz)]),
    ("ves3d_sv_eval_resident", _i, [_vp]),
    ("ves3d_sv_capture_eval", _i, [_vp]),
    ("ves3d_set_autotune", _i, [_i]),
    ("ves3d_set_far_shape", _i, [_i, _i, _i]),
    ("ves3d_autotune_report", _i, [ctypes.c_char_p, _sz, ctypes.POINTER(_sz)]),
    ("ves3d_sv_launch_eval_graph", _i, [_vp]),
    ("ves3d_sht_forward", _i, [_vp, _l, _i, _i, _vp, _vp]),
    ("ves3d_sht_backward", _i, [_vp, _l, _i, _i, _vp, _vp, _vp, _vp]),
    ("ves3d_sht_rotate_all", _i, [_vp, _l, _i, _vp, _vp]),
    ("ves3d_dev_axpy", _i, [_d, _vp, _vp, ctypes.c_size_t, _vp, _vp]),
    ("ves3d_dev_algebraic_dot", _i, [_vp, _vp, ctypes.c_size_t, ctypes.POINTER(_d), _vp]),
    ("ves3d_dev_transpose", _i, [_vp, ctypes.c_size_t, ctypes.c_size_t, _vp, _vp]),
    ("ves3d_dev_reduce", _i, [_vp, _i, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, _vp, _vp]),
    ("ves3d_dev_gemm", _i, [ctypes.c_char, ctypes.c_char, _i, _i, _i, _d, _vp, _i, _vp, _i, _d, _vp, _i, _vp]),
    ("ves3d_sht_filter_coeffs", _i, [_i, _i, _d, _vp]),
    ("ves3d_sht_scale_freq", _i, [_vp, _l, _i, _vp, _vp, _vp]),
    ("ves3d_sht_lowpass", _i, [_vp, _l, _i, _i, _d, _vp, _vp]),
    ("ves3d_sht_pole", _i, [_vp, _l, _i, _vp, _vp]),
    ("ves3d_sht_backward_d2", _i, [_vp, _l, _i, _vp, _vp, _vp, _vp]),
    ("ves3d_vtk_write_grid", _i, [_vp, _vp, _vp, _vp, _l, _i, ctypes.c_char_p, _d, _i, _i]),
    ("ves3d_vtk_write", _i, [_vp, _vp, _l, _i, _i, ctypes.c_char_p, _d, _i, _i, _i]),
    ("ves3d_cuda_stokes_f64", _i, [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("ves3d_cuda_stokes_double_layer_f64", _i, [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("ves3d_stokes_alltoall_f64", None, [_vp, _vp, _sz, _vp, ctypes.POINTER(_vp)]),
    ("ves3d_interaction_free", None, [ctypes.POINTER(_vp)]),
    ("ves3d_stokes_alltoall_device_f64", _i, [_vp, _vp, _sz, _vp, _vp]),
    ("ves3d_tables_export", _i, [_i, _i, ctypes.c_char_p, _vp, _sz, ctypes.POINTER(_sz)]),
    ("ves3d_stokes_alltoall_noalloc_f64", _i, [_vp, _vp, _sz, _vp, _vp]),
    ("ves3d_cuda_stokes_f32", _i, [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("ves3d_dev_aggregate_rotation", _i, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    ("ves3d_move_pole", _i, [_vp, ctypes.c_long, _i, _i, _i, _vp, _vp]),
    ("ves3d_sv_set_implicit_params", _i, [_vp, _d, _d, _d]),
    ("ves3d_sv_set_gravity", _i, [_vp, _d, _d, _d, _d]),
    ("ves3d_sv_set_viscosity_contrast", _i, [_vp, _vp, _l]),
    ("ves3d_sv_surface_op", _i, [_vp, _i, _vp, _vp, _i]),
    ("ves3d_sv_implicit_solve", _i, [_vp, _vp, _vp, ctypes.POINTER(_d), ctypes.POINTER(_i), ctypes.POINTER(_i), _i]),
    ("ves3d_svp_create", _i, [_i, _i, ctypes.POINTER(_vp)]),
    ("ves3d_svp_destroy", _i, [_vp]),
    ("ves3d_svp_set_src_coord", _i, [_vp, _vp, _vp, _l, _i]),
    ("ves3d_svp_set_density_sl", _i, [_vp, _vp, _i]),
    ("ves3d_svp_set_density_dl", _i, [_vp, _vp, _i]),
    ("ves3d_svp_set_viscosity_contrast", _i, [_vp, _vp, _l]),
    ("ves3d_svp_setup", _i, [_vp]),
    ("ves3d_svp_eval", _i, [_vp, _vp, _i]),
    ("ves3d_svp_stage_times", _i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    ("ves3d_svp_capture_eval", _i, [_vp]),
    ("ves3d_svp_launch_eval_graph", _i, [_vp, _vp, _i]),
    ("ves3d_svp_set_implicit_params", _i, [_vp, _d, _d, _d]),
    ("ves3d_svp_set_gravity", _i, [_vp, _d, _d, _d, _d]),
    ("ves3d_svp_set_surface_filter", _i, [_vp, _i]),
    ("ves3d_sv_set_surface_filter", _i, [_vp, _i]),
    ("ves3d_svp_set_precond", _i, [_vp, _i, _i]),
    ("ves3d_svp_implicit_solve", _i, [_vp, _vp, _vp, ctypes.POINTER(_d), ctypes.POINTER(_i), ctypes.POINTER(_i), _i]),
    ("ves3d_svp_solver_stats", _i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    ("ves3d_svp_implicit_combine", _i, [_vp, _i, ctypes.POINTER(_vp), _vp, _vp, _vp, _i]),
    ("ves3d_sv_solver_stats", _i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    ("ves3d_sv_integrals", _i, [_vp, _vp, _vp, _vp, _i]),
    ("ves3d_sv_set_precond", _i, [_vp, _i]),
    ("ves3d_sv_precond_info", _i, [_vp, _dp, ctypes.POINTER(_sz), ctypes.POINTER(_i)]),
    ("ves3d_sv_set_precond_refresh", _i, [_vp, _i]),
    ("ves3d_sv_guess_features", _i, [_vp, _vp, _i]),
    ("ves3d_sv_guess_targets", _i, [_vp, _vp, _vp, _i]),
    ("ves3d_sv_guess_from_targets", _i, [_vp, _vp, _vp, _i]),
    ("ves3d_sv_implicit_combine", _i, [_vp, _i, ctypes.POINTER(_vp), _vp, _dp, _dp, _i]),
    ("ves3d_mlp_create", _i, [_i, _i, _i, _i, ctypes.c_ulonglong, ctypes.POINTER(_vp)]),
    ("ves3d_mlp_destroy", _i, [_vp]),
    ("ves3d_mlp_num_params", _l, [_vp]),
    ("ves3d_mlp_get_params", _i, [_vp, _vp]),
    ("ves3d_mlp_set_params", _i, [_vp, _vp]),
    ("ves3d_mlp_set_scaling", _i, [_vp, _vp, _vp, _vp, _vp]),
    ("ves3d_mlp_forward", _i, [_vp, _vp, _l, _vp, _i]),
    ("ves3d_mlp_gradients", _i, [_vp, _vp, _vp, _l, _vp, ctypes.POINTER(_d), _i]),
    ("ves3d_mlp_train_step", _i, [_vp, _vp, _vp, _l, ctypes.c_float, ctypes.POINTER(_d), _i]),
    ("ves3d_bicgstab_f64", _i, [_vp, _vp, _vp, _vp, _sz, ctypes.POINTER(_d), ctypes.POINTER(_i),
                                ctypes.POINTER(_i), _vp]),
]


class Ves3dError(RuntimeError):
    pass


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Ves3dError(f"{LIB_PATH} is missing: build it with `python -m ves3d_b200.build` "
                             "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status != VES3D_OK:
        msg = lib().ves3d_last_error().decode(errors="replace")
        raise Ves3dError(f"{what}: {STATUS.get(status, status)}: {msg}")
    return status


def kernel_launches():
    return int(lib().ves3d_kernel_launches())


def tables_export(p0, p1, name):
    import numpy as np
    n = _sz(0)
    check(lib().ves3d_tables_export(p0, p1, name.encode(), None, 0, ctypes.byref(n)), "tables_export")
    out = np.empty(n.value)
    check(lib().ves3d_tables_export(p0, p1, name.encode(), out.ctypes.data, out.size, ctypes.byref(n)), "tables_export")
    return out


def filter_coeffs(p, freq=-1, exponent=0.0):
    """SHTrans filter coefficients [p(p+2)] (host): exponent <= 0 the hard cut of
    lowPassFilter, > 0 the polynomial filter of lowPassFilterPoly; freq -1 means 2p/3."""
    import numpy as np
    out = np.empty(p * (p + 2))
    check(lib().ves3d_sht_filter_coeffs(int(p), int(freq), float(exponent), out.ctypes.data), "filter_coeffs")
    return out


def set_autotune(on):
    """Turn the far-field launch-shape autotuner on or off (process-wide)."""
    check(lib().ves3d_set_autotune(1 if on else 0), "set_autotune")


def set_far_shape(waves=0, threads=0, targets_per_thread=0):
    """Fix the far-field launch shape (waves=0: back to the default / autotuned one)."""
    check(lib().ves3d_set_far_shape(int(waves), int(threads), int(targets_per_thread)), "set_far_shape")


def autotune_report():
    """{configuration key: {"waves", "threads", "ms"}} of the tuned far-field launches."""
    n = ctypes.c_size_t(0)
    check(lib().ves3d_autotune_report(None, 0, ctypes.byref(n)), "autotune_report")
    buf = ctypes.create_string_buffer(n.value + 1)
    check(lib().ves3d_autotune_report(buf, n.value + 1, ctypes.byref(n)), "autotune_report")
    out = {}
    for line in buf.value.decode().splitlines():
        key, *fields = line.split()
        out[key] = {k: float(v) if k == "ms" else int(v) for k, v in (f.split("=") for f in fields)}
    return out
