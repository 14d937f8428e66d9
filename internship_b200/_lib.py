"""ctypes binding of libmrpnn_b200.so (the C ABI in include/mrpnn_b200.h).

The library is loaded from this package directory only; a missing or stale
build raises immediately -- there is no fallback implementation.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmrpnn_b200.so")

MR_OK, MR_ERR_ARG, MR_ERR_CUDA, MR_ERR_TIMEOUT, MR_ERR_LOOP_CAP, MR_ERR_STATE, MR_ERR_NOMEM, MR_ERR_UNSUPPORTED = range(8)
RT_PT, RT_RPNN, RT_MRPNN, RT_MARCHING_MRPNN = 0, 1, 2, 3
PREC_FP32, PREC_BF16, PREC_FP8 = 0, 1, 2
SAMPLER_EXACT, SAMPLER_TEXTURE = 0, 1
READ_DENSITY, READ_MIP, READ_VARIANCE, READ_TR, READ_HGLUT = range(5)
WEIGHT_TOTAL = 49673

# Every symbol include/mrpnn_b200.h declares (checked by the CPU tests).
EXPORTS = [
    "mr_version", "mr_last_error", "mr_volume_create", "mr_volume_destroy", "mr_volume_set_data",
    "mr_volume_set_data_device", "mr_volume_update", "mr_volume_update_tr", "mr_volume_update_hglut",
    "mr_volume_max_density", "mr_volume_resolution", "mr_volume_read", "mr_network_create",
    "mr_network_destroy", "mr_builtin_stencil", "mr_weights_xavier", "mr_render", "mr_render_host",
    "mr_render_accumulate_f64", "mr_radiance_predict", "mr_gather_descriptors", "mr_sync",
    "mr_volume_counters", "mr_generate_cloud", "mr_cloud_permutation",
    "mr_volume_set_timing", "mr_volume_stage_times", "mr_tc_selftest", "mr_network_check",
    "mr_render_neural_noalloc", "mr_train_points", "mr_train_labels", "mr_train_frames", "mr_trainer_create",
    "mr_trainer_destroy", "mr_trainer_gradient", "mr_trainer_step", "mr_trainer_weights",
    "mr_render_interactive", "mr_denoise", "mr_batch_create", "mr_batch_destroy", "mr_batch_add", "mr_batch_prepare",
    "mr_batch_autotune", "mr_batch_render", "mr_batch_capture", "mr_batch_launch", "mr_batch_counters",
    "mr_tc_selftest_fp8", "mr_sampler_selftest", "mr_tc_selftest_tf32", "mr_render_host_async",
    "mr_render_host_wait", "mr_spiral_stencil", "mr_stream_read_probe", "mr_volume_load", "mr_volume_file_read",
    "mr_tc_wait_selftest", "mr_tc_selftest_mn", "mr_trainer_set_precision", "mr_volume_set_hdri", "mr_volume_load_hdri", "mr_volume_clear_hdri", "mr_hdr_read",
    "mr_batch_set_timing", "mr_batch_frame_times", "mr_volume_set_surface_ior",
]
NOALLOC_MAX_PIXELS = 16384


class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class RenderParams(C.Structure):
    """mr_render_params."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32),
                ("ori", Float3), ("up", Float3), ("right", Float3),
                ("light_dir", Float3), ("light_color", Float3),
                ("alpha", C.c_float), ("g", C.c_float), ("scatter_rate", Float3),
                ("tr_scale", C.c_float), ("env_color", Float3),
                ("max_bounces", C.c_int32), ("spp", C.c_int32),
                ("seed", C.c_uint32), ("sample_offset", C.c_uint32),
                ("render_type", C.c_int32), ("precision", C.c_int32), ("sampler", C.c_int32)]


class Histogram(C.Structure):
    """mr_histogram (the reference's Histogram, core/volume.hpp:14-19)."""
    _fields_ = [("bin", C.c_float * 30), ("total_samples", C.c_float), ("x2", C.c_float), ("x", C.c_float)]


class Interactive(C.Structure):
    """mr_interactive."""
    _fields_ = [("prev_ori", Float3), ("prev_up", Float3), ("prev_right", Float3), ("frame_index", C.c_int32),
                ("checkerboard", C.c_int32), ("tone", C.c_int32), ("denoise", C.c_int32), ("exposure", C.c_float)]


TONE_NONE, TONE_GAMMA, TONE_ACES = 0, 1, 2


class MRError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("mrpnn error %d: %s" % (code, msg))
        self.code = code


_lib = None


def f3(v):
    return Float3(float(v[0]), float(v[1]), float(v[2]))


def load():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libmrpnn_b200.so is not built; run internship_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    vp, sz, i32, u32, fp = C.c_void_p, C.c_size_t, C.c_int32, C.c_uint32, C.c_float
    L.mr_version.restype = C.c_char_p
    L.mr_last_error.restype = C.c_char_p
    L.mr_volume_create.argtypes = [i32, C.POINTER(vp)]
    L.mr_volume_destroy.argtypes = [vp]
    L.mr_volume_set_data.argtypes = [vp, vp, sz]
    L.mr_volume_set_data_device.argtypes = [vp, vp, sz, vp]
    L.mr_volume_update.argtypes = [vp, vp]
    L.mr_volume_update_tr.argtypes = [vp, Float3, fp, vp]
    L.mr_volume_update_hglut.argtypes = [vp, fp, u32, vp]
    L.mr_volume_max_density.argtypes = [vp, C.POINTER(fp)]
    L.mr_volume_resolution.argtypes = [vp, C.POINTER(i32)]
    L.mr_volume_read.argtypes = [vp, i32, i32, vp, sz]
    L.mr_network_create.argtypes = [vp, sz, vp, C.POINTER(vp)]
    L.mr_network_destroy.argtypes = [vp]
    L.mr_builtin_stencil.argtypes = [vp, sz]
    L.mr_spiral_stencil.argtypes = [vp, sz]
    L.mr_stream_read_probe.argtypes = [vp, sz, i32, vp, vp]
    L.mr_volume_load.argtypes = [C.c_char_p, i32, C.POINTER(vp), vp]
    L.mr_tc_wait_selftest.argtypes = [i32, C.POINTER(C.c_int64)]
    L.mr_tc_selftest_mn.argtypes = [i32, i32, i32, i32, vp, vp, vp]
    L.mr_trainer_set_precision.argtypes = [vp, i32]
    L.mr_volume_set_hdri.argtypes = [vp, vp, i32, i32]
    L.mr_batch_set_timing.argtypes = [vp, i32]
    L.mr_volume_set_surface_ior.argtypes = [vp, fp]
    L.mr_batch_frame_times.argtypes = [vp, vp, i32]
    L.mr_volume_load_hdri.argtypes = [vp, C.c_char_p]
    L.mr_volume_clear_hdri.argtypes = [vp]
    L.mr_hdr_read.argtypes = [C.c_char_p, vp, sz, C.POINTER(i32), C.POINTER(i32)]
    L.mr_volume_file_read.argtypes = [C.c_char_p, vp, sz, C.POINTER(i32)]
    L.mr_weights_xavier.argtypes = [u32, vp, sz]
    L.mr_render.argtypes = [vp, vp, C.POINTER(RenderParams), vp, vp]
    L.mr_render_host.argtypes = [vp, vp, C.POINTER(RenderParams), vp]
    L.mr_render_host_async.argtypes = [vp, vp, C.POINTER(RenderParams), vp, vp, C.POINTER(C.c_int64)]
    L.mr_render_host_wait.argtypes = [vp, C.c_int64, i32]
    L.mr_render_accumulate_f64.argtypes = [vp, C.POINTER(RenderParams), vp, vp, vp]
    L.mr_radiance_predict.argtypes = [vp, i32, vp, vp, i32, vp, vp]
    L.mr_gather_descriptors.argtypes = [vp, vp, vp, vp, i32, fp, fp, Float3, vp, vp, vp]
    L.mr_sync.argtypes = [vp, i32]
    L.mr_volume_counters.argtypes = [vp, vp]
    L.mr_generate_cloud.argtypes = [i32, u32, i32, fp, fp, fp, fp, vp, vp]
    L.mr_cloud_permutation.argtypes = [u32, vp]
    L.mr_volume_set_timing.argtypes = [vp, i32]
    L.mr_volume_stage_times.argtypes = [vp, vp, vp, i32]
    L.mr_tc_selftest.argtypes = [i32, i32, vp, vp, vp]
    L.mr_tc_selftest_fp8.argtypes = [i32, i32, vp, vp, vp]
    L.mr_sampler_selftest.argtypes = [i32, vp, vp, vp]
    L.mr_tc_selftest_tf32.argtypes = [i32, i32, vp, vp, vp, i32]
    L.mr_network_check.argtypes = [vp, i32]
    L.mr_render_neural_noalloc.argtypes = [vp, vp, C.POINTER(RenderParams), vp, vp]
    L.mr_train_points.argtypes = [vp, fp, fp, u32, i32, i32, vp, vp, C.POINTER(i32), vp]
    L.mr_train_labels.argtypes = [vp, vp, vp, i32, Float3, fp, fp, fp, i32, i32, u32, vp, vp]
    L.mr_train_frames.argtypes = [vp, i32, Float3, u32, vp, vp]
    L.mr_trainer_create.argtypes = [vp, sz, C.POINTER(vp)]
    L.mr_trainer_destroy.argtypes = [vp]
    L.mr_trainer_gradient.argtypes = [vp, vp, vp, vp, i32, vp, C.POINTER(fp), vp]
    L.mr_trainer_step.argtypes = [vp, vp, vp, vp, i32, fp, C.POINTER(fp), vp]
    L.mr_trainer_weights.argtypes = [vp, vp, sz]
    L.mr_render_interactive.argtypes = [vp, vp, C.POINTER(RenderParams), C.POINTER(Interactive), vp, vp, vp, vp]
    L.mr_denoise.argtypes = [vp, vp, vp, i32, i32, C.POINTER(Interactive), vp]
    L.mr_batch_create.argtypes = [C.POINTER(vp)]
    L.mr_batch_destroy.argtypes = [vp]
    L.mr_batch_add.argtypes = [vp, vp, C.POINTER(RenderParams), vp]
    L.mr_batch_prepare.argtypes = [vp, vp, C.c_int64, vp]
    L.mr_batch_autotune.argtypes = [vp, vp, C.POINTER(C.c_int64), C.POINTER(i32), C.POINTER(i32), vp]
    L.mr_batch_render.argtypes = [vp, vp, vp]
    L.mr_batch_capture.argtypes = [vp, vp, vp]
    L.mr_batch_launch.argtypes = [vp, vp]
    L.mr_batch_counters.argtypes = [vp, vp]
    _lib = L
    return L


def check(rc):
    if rc != MR_OK:
        raise MRError(rc, load().mr_last_error().decode())
    return rc
