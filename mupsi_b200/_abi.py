"""ctypes mirror of include/mupsi_gpu.h (struct layouts and enums).

Pure layout definitions: no library is loaded here. The GPU library binding
lives in mupsi_b200.lib; the CPU oracle reuses these layouts.
"""
import ctypes as C

MEM_HOST = 0
MEM_DEVICE = 1

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_CANCELLED = -4
ERR_UNSUPPORTED = -5
ERR_DEVICE_LIMIT = -6
ERR_IO = -7

GP_SINGLE_REALIZATION = 0
GP_RENEWAL_PLUS = 1

BSDF_LAMBERTIAN = 0
BSDF_NULL = 1
BSDF_SPECULAR = 2

MEAN_SPHERE = 0
MEAN_MESH = 1

PRIM_SPHERE = 0
PRIM_MESH = 1

f3 = C.c_float * 3


class Kernel(C.Structure):
    _fields_ = [("sigma", C.c_float), ("kernel_radius", C.c_float), ("aniso", f3), ("points_per_cell", C.c_int32)]


class Cond(C.Structure):
    _fields_ = [("C", f3), ("u_tilde", C.c_float), ("g_tilde", f3), ("active", C.c_uint32)]


class Ray(C.Structure):
    _fields_ = [("o", f3), ("d", f3), ("near_t", C.c_float), ("far_t", C.c_float)]


class MediumSample(C.Structure):
    _fields_ = [("exited", C.c_uint32), ("t", C.c_float), ("p", f3), ("normal", f3)]


class MeshDesc(C.Structure):
    _fields_ = [
        ("num_vertices", C.c_int64),
        ("vertices", C.c_void_p),
        ("num_faces", C.c_int64),
        ("faces", C.c_void_p),
        ("vertex_normals", C.c_void_p),
        ("position", f3),
        ("scale", C.c_float),
    ]


class MediumDesc(C.Structure):
    _fields_ = [
        ("mean_type", C.c_int32),
        ("mean_center", f3),
        ("mean_radius", C.c_float),
        ("mean_mesh", C.c_int32),
        ("kernel", Kernel),
    ]


class PrimitiveDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("center", f3),
        ("radius", C.c_float),
        ("mesh", C.c_int32),
        ("bsdf", C.c_int32),
        ("albedo", f3),
        ("has_emission", C.c_int32),
        ("emission", f3),
        ("int_medium", C.c_int32),
        ("ext_medium", C.c_int32),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("spp", C.c_int32),
        ("max_bounce", C.c_int32),
        ("max_medium_bounce", C.c_int32),
        ("gp_mode", C.c_int32),
        ("cam_pos", f3),
        ("cam_dir", f3),
        ("cam_up", f3),
        ("cam_fov", C.c_float),
        ("eps", C.c_float),
        ("nearteps", C.c_float),
        ("has_sky", C.c_int32),
        ("sky", f3),
        ("num_media", C.c_int32),
        ("media", C.POINTER(MediumDesc)),
        ("num_meshes", C.c_int32),
        ("meshes", C.POINTER(MeshDesc)),
        ("num_primitives", C.c_int32),
        ("primitives", C.POINTER(PrimitiveDesc)),
    ]


ON_SPP = C.CFUNCTYPE(None, C.c_int32, C.c_void_p)


class RenderArgs(C.Structure):
    _fields_ = [
        ("spp_begin", C.c_int32),
        ("spp_end", C.c_int32),
        ("cancel", C.POINTER(C.c_int32)),
        ("on_spp", ON_SPP),
        ("user", C.c_void_p),
        ("rgb_out", C.c_void_p),
        ("out_mem", C.c_int32),
        ("moments_out", C.c_void_p),
        ("stream", C.c_void_p),
    ]


assert C.sizeof(Cond) == 32 and C.sizeof(Ray) == 32 and C.sizeof(MediumSample) == 32


class RenderStats(C.Structure):
    _fields_ = [
        ("march_steps", C.c_uint64),
        ("psi_evals", C.c_uint64),
        ("impulse_evals", C.c_uint64),
        ("marches", C.c_uint64),
        ("march_ms", C.c_double),
        ("shade_ms", C.c_double),
        ("march_launches", C.c_int64),
        ("shade_launches", C.c_int64),
        ("iter_medium", C.c_uint32 * 16),
        ("iter_live", C.c_uint32 * 16),
        ("iter_march_ms", C.c_float * 16),
        ("mean_evals", C.c_uint64),
        ("parity_casts", C.c_uint64),
        ("surr_requests", C.c_uint64),
        ("surr_accepted", C.c_uint64),
        ("bvh_nodes", C.c_uint64),
        ("bvh_tris", C.c_uint64),
    ]


class Obj(C.Structure):
    """mupsi_obj"""
    _fields_ = [("num_vertices", C.c_int64), ("num_faces", C.c_int64), ("num_normals", C.c_int64),
                ("num_texcoords", C.c_int64), ("vertices", C.POINTER(C.c_float)), ("faces", C.POINTER(C.c_int32)),
                ("normals", C.POINTER(C.c_float)), ("texcoords", C.POINTER(C.c_float)),
                ("face_texcoords", C.POINTER(C.c_int32))]


class Tuning(C.Structure):
    _fields_ = [
        ("march_block", C.c_int32),
        ("min_group", C.c_int32),
        ("shade_block", C.c_int32),
        ("wave_paths", C.c_int32),
        ("block_rays", C.c_int32),
        ("lane_rays", C.c_int32),
        ("lane_max_tris", C.c_int32),
        ("mu_batch", C.c_int32),
    ]


class BatchArgs(C.Structure):
    _fields_ = [
        ("spp", C.POINTER(C.c_int32)),
        ("rgb_out", C.POINTER(C.c_void_p)),
        ("out_mem", C.c_int32),
        ("cancel", C.POINTER(C.c_int32)),
        ("done_ms", C.POINTER(C.c_float)),
        ("use_graphs", C.c_int32),
        ("schedule", C.c_int32),
        ("stream", C.c_void_p),
    ]


class BatchInfo(C.Structure):
    _fields_ = [
        ("waves", C.c_int32),
        ("graph_launches", C.c_int32),
        ("graphs_captured", C.c_int32),
        ("max_iters", C.c_int32),
        ("paths", C.c_int64),
    ]


SCHEDULE_SHORTEST_FIRST = 0
SCHEDULE_IN_ORDER = 1
SCHEDULE_INTERLEAVED = 2
