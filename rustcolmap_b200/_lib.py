"""Loads the in-tree CUDA libraries and declares their C signatures.

There is no CPU fallback: if librcmvs.so is missing or cannot be loaded the
import raises, and every call reports the library's own error message.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_MVS = os.path.join(_HERE, "librcmvs.so")
_SCENE = os.path.join(_HERE, "librcscene.so")
_mvs = None
_scene = None


class RcmvsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rcmvs error {code}: {msg}")
        self.code = code


def _load(path):
    if not os.path.exists(path):
        raise ImportError(
            f"{os.path.basename(path)} is not built; run `python -m rustcolmap_b200.build` "
            "(there is no CPU fallback for this path)")
    return C.CDLL(path)


def mvs():
    global _mvs
    if _mvs is not None:
        return _mvs
    L = _load(_MVS)
    vp, i32, u64, f64, cp = C.c_void_p, C.c_int32, C.c_uint64, C.c_double, C.c_char_p
    sig = {
        "rcmvs_options_default": ([vp], None),
        "rcmvs_ctx_create": ([C.c_int, vp], C.c_int),
        "rcmvs_ctx_destroy": ([vp], None),
        "rcmvs_last_error": ([vp], cp),
        "rcmvs_ctx_stream": ([vp], vp),
        "rcmvs_ctx_synchronize": ([vp], C.c_int),
        "rcmvs_pass_count": ([vp], C.c_uint64),
        "rcmvs_diag_wait_timeout": ([vp, C.c_uint64], C.c_int),
        "rcmvs_version": ([], cp),
        "rcmvs_census": ([vp, vp, i32, i32, vp], C.c_int),
        "rcmvs_estimate_depth": ([vp, vp, i32, i32, vp, i32, f64, f64, vp, vp, vp, vp], C.c_int),
        "rcmvs_estimate_depth_batch": ([vp, vp, i32, vp, i32, vp, vp], C.c_int),
        "rcmvs_fuse_depth_maps": ([vp, vp, i32, vp, vp, vp, vp, u64, vp, vp], C.c_int),
        "rcmvs_write_ply_binary": ([cp, vp, vp, u64], C.c_int),
        "rcmvs_write_dense_outputs": ([cp, vp, vp, u64, vp, u64], C.c_int),
        "rcmvs_plan": ([vp, vp, i32, vp, vp, vp, vp, vp, vp], C.c_int),
        "rcmvs_run_mvs": ([vp, vp, i32, vp, vp, vp, vp, vp], C.c_int),
        "rcmvs_points_free": ([vp], None),
        "rcmvs_scene_create": ([vp, vp, i32, vp], C.c_int),
        "rcmvs_scene_destroy": ([vp], None),
        "rcmvs_scene_prepare": ([vp, vp], C.c_int),
        "rcmvs_scene_estimate_depth": ([vp, vp, vp, i32, vp], C.c_int),
        "rcmvs_scene_fuse": ([vp, vp, vp, vp, vp, u64, vp, vp], C.c_int),
        "rcmvs_scene_get_depth": ([vp, vp, i32, vp, vp, vp], C.c_int),
        "rcmvs_scene_get_census": ([vp, vp, i32, vp], C.c_int),
        "rcmvs_scene_depth_to_device": ([vp, vp, i32, vp], C.c_int),
        "rcmvs_scene_set_depth": ([vp, vp, i32, vp, i32], C.c_int),
        "rcmvs_scene_fuse_candidates_device": ([vp, vp, vp, vp, vp, i32, vp, vp, vp], C.c_int),
        "rcmvs_scene_candidates_to_device": ([vp, vp, vp, vp], C.c_int),
        "rcmvs_scene_fuse_reduce_device": ([vp, vp, vp, vp, u64, vp, u64, vp, vp], C.c_int),
        "rcmvs_scene_get_points": ([vp, vp, vp, vp, vp], C.c_int),
        "rcmvs_plane_cost_field": ([vp, vp, i32, i32, vp, i32, vp, vp, vp, vp], C.c_int),
        "rcmvs_last_work": ([vp, vp, vp], C.c_int),
        "rcmvs_selftest_f2i": ([vp, vp, i32, vp], C.c_int),
        "rcmvs_ctx_timing": ([vp, C.c_int], C.c_int),
        "rcmvs_ctx_kernel_time": ([vp, cp, vp, vp], C.c_int),
        "rcmvs_estimate_depth_noalloc": ([vp, i32, i32, vp, i32, f64, f64, vp, vp, vp, vp], C.c_int),
        "rcmvs_net_param_count": ([], u64),
        "rcmvs_net_create": ([vp, vp, u64, vp], C.c_int),
        "rcmvs_net_destroy": ([vp], None),
        "rcmvs_net_get_params": ([vp, vp], C.c_int),
        "rcmvs_net_forward": ([vp, vp, vp, i32, i32, i32, vp], C.c_int),
        "rcmvs_net_train_step": ([vp, vp, vp, vp, i32, i32, i32, C.c_float, i32, vp, vp], C.c_int),
        "rcmvs_scene_costvol": ([vp, vp, vp, i32, vp], C.c_int),
        "rcmvs_scene_estimate_depth_learned": ([vp, vp, vp, i32, vp, vp, C.c_float, i32, C.c_float, vp], C.c_int),
        "rcmvs_scene_estimate_depth_seeded": ([vp, vp, vp, i32, vp, vp, i32, C.c_float, i32, C.c_float, vp],
                                              C.c_int),
        "rcmvs_run_mvs_learned": ([vp, vp, i32, vp, vp, vp, C.c_float, i32, C.c_float, vp, vp, vp], C.c_int),
        "rcmvs_autotune": ([vp, vp, vp, i32, vp], C.c_int),
        "rcmvs_tune_table": ([vp, vp, i32, vp], C.c_int),
        "rcmvs_tune_set": ([vp, vp, i32], C.c_int),
        "rcmvs_depth_vis": ([vp, vp, i32, i32, vp, vp], C.c_int),
        "rcmvs_scene_depth_vis": ([vp, vp, i32, vp, vp], C.c_int),
        "rcmvs_write_png_gray": ([cp, vp, i32, i32], C.c_int),
        "rcmvs_working_size": ([i32, i32, C.c_uint32, vp, vp], C.c_int),
        "rcmvs_resize_view": ([vp, vp, i32, i32, i32, i32, i32, vp, vp], C.c_int),
        "rcmvs_fuse_candidates": ([vp, vp, i32, vp, vp, vp, vp, i32, vp, vp, vp], C.c_int),
        "rcmvs_fuse_reduce": ([vp, vp, vp, u64, vp, u64, vp, vp], C.c_int),
        "rcmvs_scene_fuse_candidates": ([vp, vp, vp, vp, vp, i32, vp, vp, vp], C.c_int),
        "rcmvs_sift_options_default": ([vp], None),
        "rcmvs_extract_sift": ([vp, vp, i32, i32, i32, vp, vp], C.c_int),
        "rcmvs_sift_frame_free": ([vp], None),
        "rcmvs_match_pairs": ([vp, vp, vp, i32, vp, i32, C.c_double, vp], C.c_int),
        "rcmvs_matches_free": ([vp], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _mvs = L
    return L


def scene():
    global _scene
    if _scene is not None:
        return _scene
    L = _load(_SCENE)
    vp, i32 = C.c_void_p, C.c_int32
    L.rcscene_render.argtypes = [vp, i32, vp, i32, vp, i32, i32, i32, vp, vp, vp]
    L.rcscene_render.restype = C.c_int
    L.rcscene_last_error.argtypes = []
    L.rcscene_last_error.restype = C.c_char_p
    _scene = L
    return L


def exported_symbols():
    """Names of the functions declared in include/rcmvs.h."""
    return list(_SIG_NAMES)


_SIG_NAMES = [
    "rcmvs_options_default", "rcmvs_pass_count", "rcmvs_ctx_create", "rcmvs_ctx_destroy", "rcmvs_last_error",
    "rcmvs_ctx_stream", "rcmvs_ctx_synchronize", "rcmvs_diag_wait_timeout", "rcmvs_version", "rcmvs_census",
    "rcmvs_estimate_depth", "rcmvs_estimate_depth_batch", "rcmvs_fuse_depth_maps",
    "rcmvs_write_ply_binary", "rcmvs_write_dense_outputs", "rcmvs_plan", "rcmvs_run_mvs", "rcmvs_points_free",
    "rcmvs_scene_create", "rcmvs_scene_destroy", "rcmvs_scene_prepare",
    "rcmvs_scene_estimate_depth", "rcmvs_scene_fuse", "rcmvs_scene_get_depth",
    "rcmvs_scene_get_census", "rcmvs_scene_get_points", "rcmvs_scene_depth_to_device", "rcmvs_scene_set_depth",
    "rcmvs_scene_fuse_candidates_device", "rcmvs_scene_candidates_to_device", "rcmvs_scene_fuse_reduce_device", "rcmvs_plane_cost_field",
    "rcmvs_last_work", "rcmvs_selftest_f2i", "rcmvs_ctx_timing", "rcmvs_ctx_kernel_time",
    "rcmvs_estimate_depth_noalloc", "rcmvs_net_param_count", "rcmvs_net_create", "rcmvs_net_destroy",
    "rcmvs_net_get_params", "rcmvs_net_forward", "rcmvs_net_train_step", "rcmvs_scene_costvol",
    "rcmvs_scene_estimate_depth_learned", "rcmvs_scene_estimate_depth_seeded", "rcmvs_run_mvs_learned", "rcmvs_autotune", "rcmvs_tune_table",
    "rcmvs_tune_set", "rcmvs_depth_vis", "rcmvs_scene_depth_vis", "rcmvs_write_png_gray",
    "rcmvs_working_size", "rcmvs_resize_view", "rcmvs_fuse_candidates", "rcmvs_fuse_reduce",
    "rcmvs_scene_fuse_candidates", "rcmvs_sift_options_default", "rcmvs_extract_sift", "rcmvs_sift_frame_free",
    "rcmvs_match_pairs", "rcmvs_matches_free",
]
