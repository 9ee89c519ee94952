"""ctypes binding of libmupsi_gpu.so (include/mupsi_gpu.h).

The product path has no CPU fallback: if the library is missing or no CUDA
device is present, loading fails with an exception.
"""
import ctypes as C
import os

from . import _abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmupsi_gpu.so")

_lib = None


class MupsiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mupsi error {code}: {msg}")
        self.code = code


def _setup(L):
    vp, i64, i32, u32 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint32
    L.mupsi_gpu_last_error.restype = C.c_char_p
    L.mupsi_gpu_abi_version.restype = i32
    L.mupsi_gpu_launch_count.restype = i64
    L.mupsi_gpu_psi.argtypes = [C.POINTER(_abi.Kernel), i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_psi_value.argtypes = [C.POINTER(_abi.Kernel), i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_probe_make_seed.argtypes = [i64, i32, vp, vp, C.c_int, vp]
    L.mupsi_gpu_probe_random.argtypes = [i64, vp, i32, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_probe_impulses.argtypes = [C.POINTER(_abi.Kernel), i64, vp, vp, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_bvh_build_host.argtypes = [i64, vp, i64, vp, vp, vp, C.POINTER(i64), C.POINTER(u32)]
    L.mupsi_gpu_mesh_create.argtypes = [C.POINTER(_abi.MeshDesc), C.POINTER(vp)]
    L.mupsi_gpu_mesh_destroy.argtypes = [vp]
    L.mupsi_gpu_mesh_destroy.restype = None
    L.mupsi_gpu_bvh_intersect.argtypes = [vp, i64, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_bvh_occluded.argtypes = [vp, i64, vp, vp, C.c_int, vp]
    L.mupsi_gpu_bvh_closest.argtypes = [vp, i64, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_mesh_queries.argtypes = [vp, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_scene_create.argtypes = [C.POINTER(_abi.SceneDesc), C.POINTER(vp)]
    L.mupsi_gpu_scene_destroy.argtypes = [vp]
    L.mupsi_gpu_scene_destroy.restype = None
    L.mupsi_gpu_mean.argtypes = [vp, i32, i64, vp, vp, C.c_int, vp]
    L.mupsi_gpu_medium_eval.argtypes = [vp, i32, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_sample_distance.argtypes = [vp, i32, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_sample_condition.argtypes = [vp, i32, i64, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_trace_samples.argtypes = [vp, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_render.argtypes = [vp, C.POINTER(_abi.RenderArgs)]
    L.mupsi_gpu_trace_samples_noalloc.argtypes = [vp, i64, vp, vp, vp, vp, vp]
    L.mupsi_gpu_scene_profile.argtypes = [vp, i32]
    L.mupsi_gpu_scene_stats.argtypes = [vp, C.POINTER(_abi.RenderStats), i32]
    L.mupsi_gpu_set_tuning.argtypes = [C.POINTER(_abi.Tuning)]
    L.mupsi_gpu_get_tuning.argtypes = [C.POINTER(_abi.Tuning)]
    L.mupsi_gpu_batch_create.argtypes = [i32, C.POINTER(vp), C.POINTER(vp)]
    L.mupsi_gpu_batch_destroy.argtypes = [vp]
    L.mupsi_gpu_batch_render.argtypes = [vp, C.POINTER(_abi.BatchArgs)]
    L.mupsi_gpu_batch_info.argtypes = [vp, C.POINTER(_abi.BatchInfo)]
    L.mupsi_gpu_mlp_create.argtypes = [vp, C.POINTER(vp)]
    L.mupsi_gpu_mlp_destroy.argtypes = [vp]
    L.mupsi_gpu_mlp_get_params.argtypes = [vp, vp]
    L.mupsi_gpu_mlp_infer.argtypes = [vp, i64, vp, vp, C.c_int, vp]
    L.mupsi_gpu_mlp_grad.argtypes = [vp, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_mlp_train.argtypes = [vp, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_scene_set_surrogate.argtypes = [vp, i32, vp, C.c_float, C.c_float, C.c_float, i32]
    L.mupsi_gpu_scene_set_mean_eval.argtypes = [vp, i32, i32]
    L.mupsi_gpu_mesh_set_occlusion.argtypes = [vp, i32]
    L.mupsi_gpu_scene_set_occlusion.argtypes = [vp, i32]
    L.mupsi_gpu_scene_set_sky_texture.argtypes = [vp, i32, i32, vp]
    L.mupsi_gpu_scene_set_albedo_texture.argtypes = [vp, i32, i64, vp, vp, i32, i32, vp]
    L.mupsi_gpu_scene_set_sdf_medium.argtypes = [vp, i32]
    L.mupsi_gpu_scene_set_external_gp_medium.argtypes = [vp, i32, i32, vp, vp, vp, vp, C.c_float]
    L.mupsi_gpu_transmittance.argtypes = [vp, i32, i64, vp, vp, vp, vp, C.c_int, vp]
    L.mupsi_gpu_scene_get_size.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
    L.mupsi_gpu_release_pools.argtypes = []
    L.mupsi_obj_load.argtypes = [C.c_char_p, C.POINTER(_abi.Obj)]
    L.mupsi_obj_free.argtypes = [C.POINTER(_abi.Obj)]
    L.mupsi_obj_free.restype = None
    L.mupsi_gpu_scene_set_skip_medium.argtypes = [vp, i32]
    L.mupsi_gpu_scene_set_gp_mode.argtypes = [vp, i32]
    L.mupsi_gpu_scene_set_kernel.argtypes = [vp, i32, C.POINTER(_abi.Kernel)]
    L.mupsi_gpu_display_create.argtypes = [vp, C.POINTER(vp)]
    L.mupsi_gpu_display_destroy.argtypes = [vp]
    L.mupsi_gpu_display_destroy.restype = None
    L.mupsi_gpu_display_start_progressive.argtypes = [vp, i32, i32]
    L.mupsi_gpu_display_start.argtypes = [vp, i32]
    L.mupsi_gpu_display_cancel.argtypes = [vp]
    L.mupsi_gpu_display_cancel.restype = None
    L.mupsi_gpu_display_stop.argtypes = [vp]
    for f in ("running", "spp_pass_done", "current_spp"):
        getattr(L, "mupsi_gpu_display_" + f).argtypes = [vp]
        getattr(L, "mupsi_gpu_display_" + f).restype = i32
    L.mupsi_gpu_display_ack_spp_pass.argtypes = [vp]
    L.mupsi_gpu_display_ack_spp_pass.restype = None
    L.mupsi_gpu_display_copy_raw.argtypes = [vp, vp, i32, i32]
    L.mupsi_gpu_display_copy_tonemapped.argtypes = [vp, vp, i32, i32]
    return L


def load():
    """Load libmupsi_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m mupsi_b200.build`")
        _lib = _setup(C.CDLL(LIB_PATH))
        if _lib.mupsi_gpu_abi_version() != 4:
            raise RuntimeError("libmupsi_gpu.so ABI version mismatch")
    return _lib


def check(code):
    if code != _abi.OK:
        raise MupsiError(code, load().mupsi_gpu_last_error().decode())
    return code


def launch_count():
    return load().mupsi_gpu_launch_count()
