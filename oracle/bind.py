"""ctypes bindings of the CPU oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

Two oracles share one Python surface:
  * `Oracle("port")`  -> oracle/libmupsi_oracle.so, the C restatement (always built);
  * `Oracle("ref")`   -> oracle/_ref/libmupsi_ref_parity.so, the reference's own
    sources compiled against oracle/shim (present where the reference tree was
    available at build time); `Oracle("ref_timing")` is the -O3 OpenMP build used
    as the CPU baseline.
"""
import ctypes as C
import os

import numpy as np

from mupsi_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libmupsi_oracle.so")
REF_LIBS = {
    "ref": os.path.join(HERE, "_ref", "libmupsi_ref_parity.so"),
    "ref_timing": os.path.join(HERE, "_ref", "libmupsi_ref_timing.so"),
}

_f32 = np.ctypeslib.ndpointer(np.float32, flags="C")
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C")
_u32 = np.ctypeslib.ndpointer(np.uint32, flags="C")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C")
_u8 = np.ctypeslib.ndpointer(np.uint8, flags="C")
_i64 = np.ctypeslib.ndpointer(np.int64, flags="C")


def ref_available(kind="ref"):
    return os.path.exists(REF_LIBS[kind])


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _Port:
    """The C restatement (mupsi_oracle.h)."""

    def __init__(self, path=PORT_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        self.L = L
        L.mo_make_seed4.restype = C.c_uint32
        L.mo_make_seed4.argtypes = [C.c_uint32] * 4
        L.mo_make_seed5.restype = C.c_uint32
        L.mo_make_seed5.argtypes = [C.c_uint32] * 5
        L.mo_random_stream.argtypes = [C.c_uint64, C.c_int, _u32, _f32]
        L.mo_constant_sampler.argtypes = [C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_uint32)]
        L.mo_psi.argtypes = [C.POINTER(_abi.Kernel), C.c_int64, _f32, _u32, C.c_void_p, _f32]
        L.mo_psi_f64.argtypes = [C.POINTER(_abi.Kernel), C.c_int64, _f32, _u32, _f64, C.c_void_p]
        L.mo_psi_impulses.argtypes = [C.POINTER(_abi.Kernel), _f32, C.c_uint32, _f32, _f32, _i32, _u32]
        L.mo_bvh_build.restype = C.c_int64
        L.mo_bvh_build.argtypes = [C.c_int64, _f32, C.c_int64, _i32, _u32, _u32, C.POINTER(C.c_uint32)]
        L.mo_scene_create.restype = C.c_void_p
        L.mo_scene_create.argtypes = [C.POINTER(_abi.SceneDesc)]
        L.mo_scene_free.argtypes = [C.c_void_p]
        L.mo_bvh_intersect.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, _u32, _f32]
        L.mo_bvh_occluded.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, _u8]
        L.mo_bvh_closest.argtypes = [C.c_void_p, C.c_int, C.c_int64, _f32, _u32, _f32]
        L.mo_mesh_queries.argtypes = [C.c_void_p, C.c_int, C.c_int64, _f32, _u8, _u32, _f32]
        L.mo_mean.argtypes = [C.c_void_p, C.c_int, C.c_int64, _f32, _f32]
        L.mo_medium_eval.argtypes = [C.c_void_p, C.c_int, C.c_int64, _f32, _u32, C.c_void_p, _f32]
        L.mo_sample_distance.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, _u32, C.c_void_p, C.c_void_p]
        L.mo_sample_condition.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, _u32, C.c_void_p]
        L.mo_transmittance.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, _u32, C.c_void_p, _f32]
        L.mo_scene_set_sdf_medium.argtypes = [C.c_void_p, C.c_int]
        L.mo_scene_set_skip_medium.argtypes = [C.c_void_p, C.c_int]
        L.mo_scene_set_external_gp_medium.argtypes = [C.c_void_p, C.c_int, C.c_int, _f32, _f32, _f32, C.c_void_p,
                                                      C.c_float]
        L.mo_trace.argtypes = [C.c_void_p, C.c_int64, _i32, _i32, _i32, _f32]
        L.mo_trace_work.argtypes = [C.c_void_p, C.c_int64, _i32, _i32, _i32, _i64]
        L.mo_scene_set_sky_texture.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.mo_scene_set_albedo_texture.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int,
                                                  C.c_int, C.c_void_p]
        L.mo_mlp_forward.argtypes = [_f32, _f32, _f32, C.c_float, C.c_int64, _f32, _f32]
        L.mo_mlp_grad.argtypes = [_f32, _f32, _f32, C.c_float, C.c_int64, _f32, _f32, _f64,
                                  C.POINTER(C.c_double)]


def kernel_struct(sigma, kernel_radius, aniso, ppc):
    return _abi.Kernel(sigma, kernel_radius, _abi.f3(*aniso), ppc)


def cond_array(cond):
    """(n, 8) float array [C xyz, u, g xyz, active] -> ctypes Cond array (or None)."""
    if cond is None:
        return None
    cond = np.ascontiguousarray(cond, dtype=np.float32)
    out = np.zeros(len(cond), dtype=np.dtype([("C", "<f4", 3), ("u", "<f4"), ("g", "<f4", 3), ("active", "<u4")]))
    out["C"] = cond[:, 0:3]
    out["u"] = cond[:, 3]
    out["g"] = cond[:, 4:7]
    out["active"] = (cond[:, 7] != 0).astype(np.uint32)
    return out


def ray_array(rays):
    """(n, 8) float array [o xyz, d xyz, near, far] -> packed Ray records (same bytes)."""
    return np.ascontiguousarray(rays, dtype=np.float32)


class PortOracle:
    """Python surface over the C restatement; inputs/outputs are numpy arrays."""

    def __init__(self):
        self.b = _Port()
        self.L = self.b.L

    def make_seed4(self, a, b, c, d):
        return self.L.mo_make_seed4(a & 0xFFFFFFFF, b & 0xFFFFFFFF, c & 0xFFFFFFFF, d & 0xFFFFFFFF)

    def make_seed5(self, a, b, c, d, e):
        return self.L.mo_make_seed5(*(v & 0xFFFFFFFF for v in (a, b, c, d, e)))

    def random_stream(self, seed, n):
        u = np.zeros(n, np.uint32)
        f = np.zeros(n, np.float32)
        self.L.mo_random_stream(seed, n, u, f)
        return u, f

    def constant_sampler(self, seed):
        x, y, i = C.c_float(), C.c_float(), C.c_uint32()
        self.L.mo_constant_sampler(seed, C.byref(x), C.byref(y), C.byref(i))
        return x.value, y.value, i.value

    def mlp_forward(self, params, fourier, center, y_scale, p):
        """Surrogate MLP mu_hat at points p (n, 3) -> (n,) float32."""
        p = _f(p)
        out = np.zeros(len(p), np.float32)
        self.L.mo_mlp_forward(_f(params), _f(fourier), _f(center), float(y_scale), len(p), p, out)
        return out

    def mlp_grad(self, params, fourier, center, y_scale, p, target):
        """(dL/dparams (float64), L) for L = mean((mu_hat - target)^2) / y_scale^2."""
        p = _f(p)
        g = np.zeros(18753, np.float64)
        loss = C.c_double()
        self.L.mo_mlp_grad(_f(params), _f(fourier), _f(center), float(y_scale), len(p), p, _f(target), g,
                           C.byref(loss))
        return g, loss.value

    def psi(self, kernel, p, seed, cond=None):
        p = _f(p)
        n = len(p)
        out = np.zeros((n, 4), np.float32)
        ca = cond_array(cond)
        self.L.mo_psi(C.byref(kernel), n, p, _u(seed), None if ca is None else ca.ctypes.data, out)
        return out

    def psi_f64(self, kernel, p, seed):
        p = _f(p)
        n = len(p)
        out = np.zeros((n, 4), np.float64)
        absv = np.zeros((n, 4), np.float64)
        self.L.mo_psi_f64(C.byref(kernel), n, p, _u(seed), out, absv.ctypes.data)
        return out, absv

    def psi_impulses(self, kernel, p, seed):
        ppc = kernel.points_per_cell
        s = np.zeros((27 * ppc, 3), np.float32)
        w = np.zeros(27 * ppc, np.float32)
        cells = np.zeros((27, 3), np.int32)
        cs = np.zeros(27, np.uint32)
        self.L.mo_psi_impulses(C.byref(kernel), _f(p), seed, s, w, cells, cs)
        return s, w, cells, cs

    def bvh_build(self, verts, faces):
        verts, faces = _f(verts), _i(faces)
        nf = len(faces)
        nodes = np.zeros((max(2 * nf, 1), 8), np.uint32)
        idx = np.zeros(max(nf, 1), np.uint32)
        root = C.c_uint32()
        cnt = self.L.mo_bvh_build(len(verts), verts, nf, faces, nodes, idx, C.byref(root))
        return nodes[:cnt], idx[:nf], root.value

    # scene-level queries take a scene handle from scene_create(desc)
    def scene_create(self, desc):
        h = self.L.mo_scene_create(C.byref(desc))
        return h

    def scene_set_sky(self, h, img):
        """Skydrome BitmapTexture (h, w, 3) float RGB, row 0 at the top; None removes it."""
        if img is None:
            self.L.mo_scene_set_sky_texture(h, 0, 0, None)
            return
        img = np.ascontiguousarray(img, np.float32)
        self.L.mo_scene_set_sky_texture(h, img.shape[1], img.shape[0], img.ctypes.data)

    def scene_set_albedo(self, h, prim, img, texcoords=None, face_texcoords=None):
        """LambertianBsdf(BitmapTexture) on a mesh primitive: (h, w, 3) float RGB
        at the mesh's texcoords (None: the barycentrics); None removes it."""
        if img is None:
            rc = self.L.mo_scene_set_albedo_texture(h, prim, 0, None, None, 0, 0, None)
        else:
            img = np.ascontiguousarray(img, np.float32)
            if texcoords is None:
                n, tc, ft = 0, None, None
            else:
                tc = np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2)
                ft = np.ascontiguousarray(face_texcoords, np.int32).reshape(-1, 3)
                n = len(tc)
            rc = self.L.mo_scene_set_albedo_texture(h, prim, n, None if tc is None else tc.ctypes.data,
                                                    None if ft is None else ft.ctypes.data, img.shape[1],
                                                    img.shape[0], img.ctypes.data)
        if rc != 0:
            raise ValueError("bad albedo texture arguments")

    def scene_from(self, sc):
        """scene_create(sc.desc()) plus the scene's sky and albedo textures."""
        h = self.scene_create(sc.desc())
        for i, m in enumerate(sc.media):
            if m.get("kind") == "sdf":
                self.scene_set_sdf(h, i)
            elif m.get("kind") == "external_gp":
                self.scene_set_external_gp(h, i, m["res"], m["bmin"], m["bmax"], m["mean_grid"], m["var_grid"],
                                           m["noise_scale"])
        if getattr(sc, "sky_texture", None) is not None:
            self.scene_set_sky(h, sc.sky_texture)
        for i, p in enumerate(sc.primitives):
            if p.get("texture") is not None:
                m = sc.meshes[p["mesh"]]
                self.scene_set_albedo(h, i, p["texture"], m.texcoords, m.face_texcoords)
        return h

    def scene_free(self, h):
        self.L.mo_scene_free(h)

    def bvh_intersect(self, h, mesh, rays):
        rays = ray_array(rays)
        n = len(rays)
        tri = np.zeros(n, np.uint32)
        tuv = np.zeros((n, 3), np.float32)
        self.L.mo_bvh_intersect(h, mesh, n, rays.ctypes.data, tri, tuv)
        return tri, tuv

    def bvh_occluded(self, h, mesh, rays):
        rays = ray_array(rays)
        out = np.zeros(len(rays), np.uint8)
        self.L.mo_bvh_occluded(h, mesh, len(rays), rays.ctypes.data, out)
        return out

    def bvh_closest(self, h, mesh, p):
        p = _f(p)
        tri = np.zeros(len(p), np.uint32)
        dq = np.zeros((len(p), 4), np.float32)
        self.L.mo_bvh_closest(h, mesh, len(p), p, tri, dq)
        return tri, dq

    def mesh_queries(self, h, mesh, p):
        p = _f(p)
        n = len(p)
        ins = np.zeros(n, np.uint8)
        tri = np.zeros(n, np.uint32)
        dq = np.zeros((n, 4), np.float32)
        self.L.mo_mesh_queries(h, mesh, n, p, ins, tri, dq)
        return ins, tri, dq

    def mean(self, h, medium, p):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        self.L.mo_mean(h, medium, len(p), p, out)
        return out

    def medium_eval(self, h, medium, p, seed, cond=None):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        ca = cond_array(cond)
        self.L.mo_medium_eval(h, medium, len(p), p, _u(seed), None if ca is None else ca.ctypes.data, out)
        return out

    def sample_distance(self, h, medium, rays, seed, cond=None):
        rays = ray_array(rays)
        n = len(rays)
        out = np.zeros((n, 8), np.float32)
        ca = cond_array(cond)
        self.L.mo_sample_distance(h, medium, n, rays.ctypes.data, _u(seed), None if ca is None else ca.ctypes.data,
                                  out.ctypes.data)
        res = out.copy()
        res[:, 0] = out.view(np.uint32)[:, 0].astype(np.float32)
        return res

    def transmittance(self, h, medium, rays, seed, cond=None):
        rays = ray_array(rays)
        out = np.zeros(len(rays), np.float32)
        ca = cond_array(cond)
        self.L.mo_transmittance(h, medium, len(rays), rays.ctypes.data, _u(seed),
                                None if ca is None else ca.ctypes.data, out)
        return out

    def scene_set_skip_medium(self, h, skip):
        self.L.mo_scene_set_skip_medium(h, 1 if skip else 0)

    def scene_set_sdf(self, h, medium):
        if self.L.mo_scene_set_sdf_medium(h, medium) != 0:
            raise ValueError("bad medium")

    def scene_set_external_gp(self, h, medium, res, bmin, bmax, mean, var=None, noise_scale=1.0):
        v = None if var is None else _f(var).reshape(-1)
        if self.L.mo_scene_set_external_gp_medium(h, medium, res, _f(bmin), _f(bmax), _f(mean).reshape(-1),
                                                  None if v is None else v.ctypes.data, noise_scale) != 0:
            raise ValueError("bad external GP medium")

    def sample_condition(self, h, medium, samples, seed):
        """samples: (n, 7) [exited, p xyz, normal xyz] -> (n, 8) [C, u, g, active]"""
        samples = np.asarray(samples, np.float32)
        n = len(samples)
        ms = np.zeros((n, 8), np.float32)
        ms.view(np.uint32)[:, 0] = samples[:, 0].astype(np.uint32)
        ms[:, 2:5] = samples[:, 1:4]
        ms[:, 5:8] = samples[:, 4:7]
        out = np.zeros((n, 8), np.float32)
        self.L.mo_sample_condition(h, medium, n, ms.ctypes.data, _u(seed), out.ctypes.data)
        res = out.copy()
        res[:, 7] = out.view(np.uint32)[:, 7].astype(np.float32)
        return res

    def trace(self, h, x, y, k):
        x, y, k = _i(x), _i(y), _i(k)
        out = np.zeros((len(x), 3), np.float32)
        self.L.mo_trace(h, len(x), x, y, k, out)
        return out

    def trace_work(self, h, x, y, k):
        x, y, k = _i(x), _i(y), _i(k)
        out = np.zeros(2, np.int64)
        self.L.mo_trace_work(h, len(x), x, y, k, out)
        return out


class RefOracle:
    """The reference's own sources (oracle/_ref), through oracle/ref_harness.cpp."""

    def __init__(self, kind="ref"):
        path = REF_LIBS[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = C.CDLL(path)
        self.L = L
        L.ref_make_seed4.restype = C.c_uint32
        L.ref_make_seed4.argtypes = [C.c_uint32] * 4
        L.ref_make_seed5.restype = C.c_uint32
        L.ref_make_seed5.argtypes = [C.c_uint32] * 5
        L.ref_random_stream.argtypes = [C.c_uint64, C.c_int, _u32, _f32]
        L.ref_constant_sampler.argtypes = [C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_uint32)]
        L.ref_psi.argtypes = [C.c_float, C.c_float, _f32, C.c_int, C.c_long, _f32, _u32, _f32]
        L.ref_kernel_terms.argtypes = [C.c_float, C.c_float, _f32, C.c_long, _f32, _f32, _f32, _f32]
        L.ref_medium_create.restype = C.c_void_p
        L.ref_medium_create.argtypes = [C.c_int, _f32, C.c_float, C.c_char_p, C.c_void_p, C.c_float, C.c_float,
                                        C.c_float, _f32, C.c_int]
        L.ref_medium_free.argtypes = [C.c_void_p]
        L.ref_mean_eval.argtypes = [C.c_void_p, C.c_long, _f32, _f32]
        L.ref_medium_eval.argtypes = [C.c_void_p, C.c_long, _f32, _u32, C.c_void_p, _f32]
        L.ref_sample_distance.argtypes = [C.c_void_p, C.c_long, _f32, _u32, C.c_void_p, _f32]
        L.ref_sample_condition.argtypes = [C.c_void_p, C.c_long, _f32, _u32, C.c_int, _f32]
        L.ref_bvh_build.restype = C.c_void_p
        L.ref_bvh_build.argtypes = [C.c_long, _f32, C.c_long, _i32]
        L.ref_field_create.restype = C.c_void_p
        L.ref_field_create.argtypes = [C.c_int, C.c_int, _f32, C.c_float, C.c_char_p, C.c_void_p, C.c_float, C.c_int,
                                       _f32, _f32, C.c_char_p, C.c_char_p, C.c_float]
        L.ref_field_free.argtypes = [C.c_void_p]
        L.ref_field_eval.argtypes = [C.c_void_p, C.c_long, _f32, _u32, _f32]
        L.ref_field_sample_distance.argtypes = [C.c_void_p, C.c_long, _f32, _u32, _f32]
        L.ref_field_transmittance.argtypes = [C.c_void_p, C.c_long, _f32, _u32, _f32]
        L.ref_grid_eval.argtypes = [C.c_char_p, C.c_int, _f32, _f32, C.c_long, _f32, _f32]
        L.ref_set_skip_medium.argtypes = [C.c_int]
        L.ref_obj_load.restype = C.c_void_p
        L.ref_obj_load.argtypes = [C.c_char_p, C.c_void_p]
        L.ref_obj_arrays.argtypes = [C.c_void_p, _f32, _i32, _f32, _f32, _i32]
        L.ref_obj_free.argtypes = [C.c_void_p]
        L.ref_bvh_free.argtypes = [C.c_void_p]
        L.ref_bvh_node_count.restype = C.c_long
        L.ref_bvh_node_count.argtypes = [C.c_void_p]
        L.ref_bvh_root.restype = C.c_uint32
        L.ref_bvh_root.argtypes = [C.c_void_p]
        L.ref_bvh_nodes.argtypes = [C.c_void_p, _u32, _u32]
        L.ref_bvh_intersect.argtypes = [C.c_void_p, C.c_long, _f32, _u32, _f32]
        L.ref_bvh_occluded.argtypes = [C.c_void_p, C.c_long, _f32, _u8]
        L.ref_bvh_closest.argtypes = [C.c_void_p, C.c_long, _f32, _u32, _f32]
        L.ref_mesh_queries.argtypes = [C.c_void_p, C.c_long, _f32, _u8, _u32, _f32]
        L.ref_scene_load.restype = C.c_void_p
        L.ref_scene_load.argtypes = [C.c_char_p, C.c_float]
        L.ref_scene_add_mesh.restype = C.c_int
        L.ref_scene_add_mesh.argtypes = [C.c_void_p, C.c_char_p, C.c_float]
        L.ref_scene_prepare.argtypes = [C.c_void_p]
        L.ref_scene_free.argtypes = [C.c_void_p]
        L.ref_scene_spp.restype = C.c_int
        L.ref_scene_spp.argtypes = [C.c_void_p]
        L.ref_scene_size.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_trace.argtypes = [C.c_void_p, C.c_long, _i32, _i32, _i32, _f32]
        L.ref_render.restype = C.c_int
        L.ref_render.argtypes = [C.c_void_p, C.c_int, _f32]
        L.ref_num_threads.restype = C.c_int

    def make_seed4(self, a, b, c, d):
        return self.L.ref_make_seed4(a & 0xFFFFFFFF, b & 0xFFFFFFFF, c & 0xFFFFFFFF, d & 0xFFFFFFFF)

    def make_seed5(self, a, b, c, d, e):
        return self.L.ref_make_seed5(*(v & 0xFFFFFFFF for v in (a, b, c, d, e)))

    def random_stream(self, seed, n):
        u = np.zeros(n, np.uint32)
        f = np.zeros(n, np.float32)
        self.L.ref_random_stream(seed, n, u, f)
        return u, f

    def constant_sampler(self, seed):
        x, y, i = C.c_float(), C.c_float(), C.c_uint32()
        self.L.ref_constant_sampler(seed, C.byref(x), C.byref(y), C.byref(i))
        return x.value, y.value, i.value

    def psi(self, kernel, p, seed):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        self.L.ref_psi(kernel.sigma, kernel.kernel_radius, _f(list(kernel.aniso)), kernel.points_per_cell, len(p), p,
                       _u(seed), out)
        return out

    def kernel_terms(self, kernel, s, p, v):
        out = np.zeros((len(p), 8), np.float32)
        self.L.ref_kernel_terms(kernel.sigma, kernel.kernel_radius, _f(list(kernel.aniso)), len(p), _f(s), _f(p), _f(v),
                                out)
        return out

    def medium_create(self, mean_type, kernel, center=(0, 0, 0), radius=70.0, obj_path=None, mesh_pos=None,
                      mesh_scale=1.0):
        mp = _f(mesh_pos) if mesh_pos is not None else None
        h = self.L.ref_medium_create(mean_type, _f(center), radius, obj_path.encode() if obj_path else None,
                                     mp.ctypes.data if mp is not None else None, mesh_scale, kernel.sigma,
                                     kernel.kernel_radius, _f(list(kernel.aniso)), kernel.points_per_cell)
        if not h:
            raise RuntimeError("reference medium could not be created")
        return h

    def medium_free(self, h):
        self.L.ref_medium_free(h)

    def sdf_create(self, mean_type, center=(0, 0, 0), radius=70.0, obj_path=None, mesh_pos=None, mesh_scale=1.0):
        """SDFMedium over a SphereMeanFunction (0) or MeshMeanFunction (1)."""
        mp = _f(mesh_pos) if mesh_pos is not None else None
        h = self.L.ref_field_create(1, mean_type, _f(center), radius, obj_path.encode() if obj_path else None,
                                    mp.ctypes.data if mp is not None else None, mesh_scale, 0, _f([0, 0, 0]),
                                    _f([1, 1, 1]), None, None, 0.0)
        if not h:
            raise RuntimeError("reference SDF medium could not be created")
        return h

    def external_gp_create(self, res, bmin, bmax, mean_path, var_path=None, noise_scale=1.0):
        """ExternalGPMedium over GridMeanFunction files (float32, x-major)."""
        h = self.L.ref_field_create(2, 0, _f([0, 0, 0]), 0.0, None, None, 1.0, res, _f(bmin), _f(bmax),
                                    mean_path.encode(), var_path.encode() if var_path else None, noise_scale)
        if not h:
            raise RuntimeError("reference external GP medium could not be created")
        return h

    def field_free(self, h):
        self.L.ref_field_free(h)

    def field_eval(self, h, p, seed):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        self.L.ref_field_eval(h, len(p), p, _u(seed), out)
        return out

    def field_sample_distance(self, h, rays, seed):
        rays = _f(rays)
        out = np.zeros((len(rays), 8), np.float32)
        self.L.ref_field_sample_distance(h, len(rays), rays, _u(seed), out)
        return out

    def field_transmittance(self, h, rays, seed):
        rays = _f(rays)
        out = np.zeros(len(rays), np.float32)
        self.L.ref_field_transmittance(h, len(rays), rays, _u(seed), out)
        return out

    def grid_eval(self, path, res, bmin, bmax, p):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        self.L.ref_grid_eval(path.encode(), res, _f(bmin), _f(bmax), len(p), p, out)
        return out

    def mean(self, h, p):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        self.L.ref_mean_eval(h, len(p), p, out)
        return out

    def medium_eval(self, h, p, seed, cond=None):
        p = _f(p)
        out = np.zeros((len(p), 4), np.float32)
        c = _f(cond) if cond is not None else None
        self.L.ref_medium_eval(h, len(p), p, _u(seed), c.ctypes.data if c is not None else None, out)
        return out

    def sample_distance(self, h, rays, seed, cond=None):
        rays = _f(rays)
        out = np.zeros((len(rays), 8), np.float32)
        c = _f(cond) if cond is not None else None
        self.L.ref_sample_distance(h, len(rays), rays, _u(seed), c.ctypes.data if c is not None else None, out)
        return out

    def sample_condition(self, h, samples, seed, renewal_plus=True):
        samples = _f(samples)
        out = np.zeros((len(samples), 8), np.float32)
        self.L.ref_sample_condition(h, len(samples), samples, _u(seed), 1 if renewal_plus else 0, out)
        return out

    def bvh_build(self, verts, faces):
        h = self.L.ref_bvh_build(len(verts), _f(verts), len(faces), _i(faces))
        cnt = self.L.ref_bvh_node_count(h)
        nodes = np.zeros((max(cnt, 1), 8), np.uint32)
        idx = np.zeros(max(len(faces), 1), np.uint32)
        self.L.ref_bvh_nodes(h, nodes, idx)
        root = self.L.ref_bvh_root(h)
        return h, nodes[:cnt], idx[: len(faces)], root

    def bvh_free(self, h):
        self.L.ref_bvh_free(h)

    def bvh_intersect(self, h, rays):
        rays = _f(rays)
        tri = np.zeros(len(rays), np.uint32)
        tuv = np.zeros((len(rays), 3), np.float32)
        self.L.ref_bvh_intersect(h, len(rays), rays, tri, tuv)
        return tri, tuv

    def bvh_occluded(self, h, rays):
        rays = _f(rays)
        out = np.zeros(len(rays), np.uint8)
        self.L.ref_bvh_occluded(h, len(rays), rays, out)
        return out

    def bvh_closest(self, h, p):
        p = _f(p)
        tri = np.zeros(len(p), np.uint32)
        dq = np.zeros((len(p), 4), np.float32)
        self.L.ref_bvh_closest(h, len(p), p, tri, dq)
        return tri, dq

    def mesh_queries(self, medium_h, p):
        p = _f(p)
        n = len(p)
        ins = np.zeros(n, np.uint8)
        tri = np.zeros(n, np.uint32)
        dq = np.zeros((n, 4), np.float32)
        self.L.ref_mesh_queries(medium_h, n, p, ins, tri, dq)
        return ins, tri, dq

    def obj_load(self, path):
        """Mesh::fetchFrom: (vertices, faces, normals, texcoords, face_texcoords) or None."""
        sizes = np.zeros(4, np.int64)
        h = self.L.ref_obj_load(path.encode(), sizes.ctypes.data)
        if not h:
            return None
        nv, nf, nn, nt = (int(x) for x in sizes)
        v, f = np.zeros((nv, 3), np.float32), np.zeros((nf, 3), np.int32)
        n, t, ft = np.zeros((nn, 3), np.float32), np.zeros((nt, 2), np.float32), np.zeros((nf, 3), np.int32)
        self.L.ref_obj_arrays(h, v, f, n, t, ft)
        self.L.ref_obj_free(h)
        return v, f, n, t, ft

    def set_skip_medium(self, skip):
        """g_pathTracerSettings.skip_medium for the scenes prepared from now on."""
        self.L.ref_set_skip_medium(1 if skip else 0)

    def scene_load(self, json_path, sky=1.0, extra_meshes=()):
        h = self.L.ref_scene_load(json_path.encode(), -1.0 if sky is None else float(sky))
        if not h:
            raise RuntimeError(f"reference could not load {json_path}")
        for obj, albedo in extra_meshes:
            if self.L.ref_scene_add_mesh(h, obj.encode(), albedo) != 0:
                raise RuntimeError(f"reference could not load {obj}")
        self.L.ref_scene_prepare(h)
        return h

    def scene_free(self, h):
        self.L.ref_scene_free(h)

    def trace(self, h, x, y, k):
        x, y, k = _i(x), _i(y), _i(k)
        out = np.zeros((len(x), 3), np.float32)
        self.L.ref_trace(h, len(x), x, y, k, out)
        return out

    def render(self, h, spp):
        w, hh = C.c_int(), C.c_int()
        self.L.ref_scene_size(h, C.byref(w), C.byref(hh))
        out = np.zeros((hh.value, w.value, 3), np.float32)
        self.L.ref_render(h, spp, out)
        return out

    def num_threads(self):
        return self.L.ref_num_threads()
