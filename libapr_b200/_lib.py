"""ctypes binding of libaprb200.so (the C ABI declared in include/aprb200.h).

The library is built in-tree by libapr_b200/build.py.  There is no fallback:
importing this module raises if the CUDA library is missing, and every call
that fails returns its aprb_status, which the Python layer turns into an
exception.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaprb200.so")

APRB_OK = 0
STATUS = {
    0: "ok", 1: "invalid argument", 2: "input dimension check failed", 3: "integer overflow",
    4: "unsupported", 5: "out of memory", 6: "CUDA error", 7: "no sm_100 device", 8: "incomplete neighbourhood",
}


class aprb_params(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("dx", "dy", "dz", "psfx", "psfy", "psfz", "Ip_th", "lambda_", "rel_error",
                                         "sigma_th", "sigma_th_max", "grad_th")] + \
               [(n, C.c_int) for n in ("reflect_bc_lis", "neighborhood_optimization", "constant_intensity_scale",
                                       "check_input", "swap_dimensions", "auto_parameters")]


class aprb_apr_info(C.Structure):
    _fields_ = [("l_min", C.c_int), ("l_max", C.c_int), ("org_dims", C.c_int * 3),
                ("y_num", C.c_int * 32), ("x_num", C.c_int * 32), ("z_num", C.c_int * 32),
                ("total_number_particles", C.c_uint64), ("n_level_xz", C.c_uint64), ("n_xz", C.c_uint64),
                ("bspline_offset", C.c_float),
                ("tree_l_min", C.c_int), ("tree_l_max", C.c_int), ("tree_total_number_particles", C.c_uint64),
                ("tree_n_level_xz", C.c_uint64), ("tree_n_xz", C.c_uint64)]


class aprb_volume(C.Structure):
    _fields_ = [("img_dev", C.c_void_p), ("y_num", C.c_int), ("x_num", C.c_int), ("z_num", C.c_int)]


# Every exported entry point and its C signature (include/aprb200.h).
_vp, _u64, _i, _f = C.c_void_p, C.c_uint64, C.c_int, C.c_float
SIGNATURES = {
    "aprb_status_string": ([C.c_int], C.c_char_p),
    "aprb_last_error": ([], C.c_char_p),
    "aprb_default_params": ([C.POINTER(aprb_params)], None),
    "aprb_converter_create": ([_i, C.POINTER(_vp)], _i),
    "aprb_converter_destroy": ([_vp], _i),
    "aprb_converter_keep_intermediates": ([_vp, _i], _i),
    "aprb_converter_keep_input": ([_vp, _i], _i),
    "aprb_smoothing_variants": ([_i, C.POINTER(_i)], _i),
    "aprb_smoothing_schedule_set": ([_i, _i, _i], _i),
    "aprb_smoothing_schedule_get": ([_i, _i, C.POINTER(_i)], _i),
    "aprb_get_apr": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, C.POINTER(_vp)], _i),
    "aprb_get_apr_device": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, _vp, C.POINTER(_vp)], _i),
    "aprb_get_apr_by_block": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, _i, _i, C.POINTER(_vp)], _i),
    "aprb_get_apr_by_block_device": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, _i, _i, _vp, C.POINTER(_vp)],
                                     _i),
    "aprb_get_apr_batch_device": ([_vp, C.POINTER(aprb_params), _i, C.POINTER(aprb_volume), _i, _i, _vp,
                                   C.POINTER(_vp)], _i),
    "aprb_converter_intermediate": ([_vp, _i, _vp, C.c_size_t], _i),
    "aprb_pyramid_bytes": ([_i, _i, _i, C.POINTER(_u64)], _i),
    "aprb_pyramid_fill_tiles_device": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _i, _i,
                                        _vp], _i),
    "aprb_get_apr_from_pyramid_device": ([_vp, C.POINTER(aprb_params), _vp, _i, _i, _i, _vp, C.POINTER(_vp)], _i),
    "aprb_converter_level_margins": ([_vp, C.c_double, C.POINTER(_u64), C.POINTER(_u64)], _i),
    "aprb_apr_free": ([_vp], _i),
    "aprb_apr_get_info": ([_vp, C.POINTER(aprb_apr_info)], _i),
    "aprb_apr_get_parameters": ([_vp, C.POINTER(aprb_params)], _i),
    "aprb_threshold_li": ([_vp, _u64, _i, C.POINTER(C.c_float)], _i),
    "aprb_auto_parameters": ([C.POINTER(aprb_params), _vp, _vp, _vp, _u64, _i, _f], _i),
    "aprb_apr_export": ([_vp, _vp, _vp, _vp], _i),
    "aprb_apr_device_arrays": ([_vp, _vp, _vp, _vp], _i),
    "aprb_apr_from_arrays": ([_i, _i, _i, _vp, _u64, _vp, _u64, _vp, _u64, C.POINTER(_vp)], _i),
    "aprb_sample_image": ([_vp, _vp, _vp], _i),
    "aprb_sample_image_device": ([_vp, _vp, _vp, _vp], _i),
    "aprb_sample_image_by_block": ([_vp, _vp, _i, _i, _vp], _i),
    "aprb_sample_image_by_block_device": ([_vp, _vp, _i, _i, _vp, _vp], _i),
    "aprb_sample_image_noalloc": ([_vp, _vp, _i, _i, _i, _vp, _vp, _vp], _i),
    "aprb_apr_init_tree": ([_vp], _i),
    "aprb_apr_export_tree": ([_vp, _vp, _vp, _vp], _i),
    "aprb_fill_tree_mean": ([_vp, _vp, _vp], _i),
    "aprb_fill_tree_mean_device": ([_vp, _vp, _vp, _vp], _i),
    "aprb_convolve": ([_vp, _vp, _i, _vp, _vp, _i, _i, _i], _i),
    "aprb_convolve_device": ([_vp, _vp, _i, _vp, _vp, _i, _i, _i, _vp], _i),
    "aprb_richardson_lucy": ([_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i], _i),
    "aprb_richardson_lucy_device": ([_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp], _i),
    "aprb_richardson_lucy_fp64": ([_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i], _i),
    "aprb_richardson_lucy_fp64_device": ([_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp], _i),
    "aprb_cnn_layer_forward_device": ([_vp, _vp, _vp, _vp, _i, _vp, _vp], _i),
    "aprb_cnn_layer_backward_device": ([_vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp], _i),
    "aprb_cnn_features_device": ([_vp, _vp, _vp, _vp, _vp, _vp], _i),
    "aprb_cnn_loss_device": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "aprb_cnn_apply_device": ([_vp, _vp, _vp, _vp], _i),
    "aprb_cnn_adam_device": ([_vp, _vp, _vp, _vp, _vp, _u64, _f, _f, _f, _f, _i, _vp], _i),
    "aprb_rl_ratio_device": ([_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _vp], _i),
    "aprb_rl_objective_device": ([_vp, _vp, _vp, _vp, _i, _i, _i, C.POINTER(C.c_double), _vp], _i),
    "aprb_synth_blobs_u16": ([_vp, _i, _i, _i, _i, _f, _f, _f, _f, _f, _u64, _vp], _i),
    "aprb_synth_blobs_f32": ([_vp, _i, _i, _i, _i, _f, _f, _f, _f, _f, _u64, _vp], _i),
    "aprb_kernel_launch_count": ([], _u64),
    "aprb_gradient": ([_vp, _vp, _vp, _i, _f, _i], _i),
    "aprb_gradient_device": ([_vp, _vp, _vp, _i, _f, _i, _vp], _i),
    "aprb_gradient_magnitude": ([_vp, _vp, _vp, _vp, _i], _i),
    "aprb_gradient_magnitude_device": ([_vp, _vp, _vp, _vp, _i, _vp], _i),
    "aprb_reconstruct_constant_u16": ([_vp, _vp, _vp], _i),
    "aprb_reconstruct_constant_f32": ([_vp, _vp, _vp], _i),
    "aprb_reconstruct_level": ([_vp, _vp], _i),
    "aprb_reconstruct_constant_u16_device": ([_vp, _vp, _vp, _vp], _i),
    "aprb_reconstruct_constant_f32_device": ([_vp, _vp, _vp, _vp], _i),
    "aprb_reconstruct_level_device": ([_vp, _vp, _vp], _i),
    "aprb_check_division_by_constant": ([C.c_float, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)], _i),
    "aprb_measure_fp32_fma_peak": ([_vp, C.POINTER(C.c_double)], _i),
    "aprb_profile_enable": ([_i], _i),
    "aprb_profile_reset": ([], _i),
    "aprb_profile_read": ([C.POINTER(C.c_char_p), C.POINTER(C.c_double), C.POINTER(C.c_uint64), _i], _i),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libaprb200.so is not built (run libapr_b200/build.py or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
        apply_schedule_file(L)
    return _lib


# The smoothing schedule chosen by libapr_b200.autotune on the device
# (aprb_smoothing_schedule_set): {"schedule": {"y": [variant per bucket], "x":
# [...], "z": [...]}}, buckets n <= 128, 256, 512, 1024, 2048, longer.
SCHEDULE_FILE = os.path.join(HERE, "data", "smoothing_schedule.json")
AXES = ("y", "x", "z")


def apply_schedule_file(L, path=SCHEDULE_FILE):
    """Sets the library's smoothing schedule from the autotuner's file, when
    there is one; returns the schedule applied (or None)."""
    import json
    if not path or not os.path.exists(path):
        return None
    with open(path) as f:
        sched = json.load(f)["schedule"]
    for a, name in enumerate(AXES):
        for b, v in enumerate(sched.get(name, [])):
            st = L.aprb_smoothing_schedule_set(a, b, int(v))
            if st != APRB_OK:
                raise APRBError(st, "smoothing schedule %s: bucket %d variant %s" % (name, b, v))
    return sched


class APRBError(RuntimeError):
    def __init__(self, status, detail):
        super().__init__("%s: %s" % (STATUS.get(status, status), detail))
        self.status = status


def check(status):
    if status != APRB_OK:
        raise APRBError(status, lib().aprb_last_error().decode())
