"""Host-side mirror of the reference renderer's interfaces, backed by the GPU library.

Names and argument meaning follow the reference (src/gp, src/medium, src/bvh,
src/rendering); every call is a batch over numpy arrays (host memory) or CUDA
torch tensors (device memory) and goes through the C ABI in include/mupsi_gpu.h.
Errors raise MupsiError with the library's message, the counterpart of the
reference's bool + std::cerr returns.
"""
import ctypes as C
import json
import os

import numpy as np

from . import _abi
from .lib import check, load
from .scene import Scene

try:  # torch is optional plumbing: device buffers and streams
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_dev(a):
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _mem(*arrays):
    kinds = {_is_dev(a) for a in arrays if a is not None}
    if len(kinds) > 1:
        raise ValueError("all buffers of one call must be host (numpy) or all device (CUDA tensors)")
    return _abi.MEM_DEVICE if kinds == {True} else _abi.MEM_HOST


def _ptr(a):
    if a is None:
        return None
    if _is_dev(a):
        if not a.is_contiguous():
            raise ValueError("device buffers must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host buffers must be C-contiguous")
    return a.ctypes.data


def _stream(stream):
    if stream is not None:
        return stream
    if torch is not None and torch.cuda.is_available():
        return torch.cuda.current_stream().cuda_stream
    return None


def _need(a, shape, name):
    """An input the library reads `shape` elements of (a None input is absent)."""
    if a is not None and tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(a.shape)}")


def check_buf(a, shape, dtype=np.float32, name="out"):
    """A caller's output buffer must hold exactly `shape` elements of `dtype`
    (the library writes that many through the pointer). Returns a."""
    n = int(np.prod(shape))
    if _is_dev(a):
        tdt = {np.float32: torch.float32, np.float64: torch.float64, np.int32: torch.int32,
               np.uint32: torch.int32}[dtype]
        ok = a.dtype == tdt and a.numel() == n
    else:
        ok = isinstance(a, np.ndarray) and a.dtype == np.dtype(dtype) and a.size == n
    if not ok:
        raise ValueError(f"{name} must hold {tuple(shape)} {np.dtype(dtype).name} values")
    return a


def _empty(like_dev, shape, dtype):
    if like_dev:
        tdt = {np.float32: torch.float32, np.uint32: torch.int32, np.uint8: torch.uint8}[dtype]
        return torch.empty(shape, dtype=tdt, device="cuda")
    return np.empty(shape, dtype=dtype)


def _host(a, dtype):
    if _is_dev(a):
        return a.contiguous()
    return np.ascontiguousarray(a, dtype=dtype)


def cond_records(cond):
    """(n, 8) [C xyz, u, g xyz, active] -> GPConditioningState records (mupsi_cond)."""
    if cond is None:
        return None
    if _is_dev(cond):
        c = cond.float().contiguous().clone()
        c.view(torch.int32)[:, 7] = (cond[:, 7] != 0).int()
        return c
    cond = np.ascontiguousarray(cond, np.float32)
    out = cond.copy()
    out.view(np.uint32)[:, 7] = (cond[:, 7] != 0).astype(np.uint32)
    return out


class SparseSEKernel:
    """SparseSEKernel(sigma, kernelRadius, lengthScale) (gp/kernel.h:39-78)."""

    def __init__(self, sigma, kernel_radius, length_scale=(1.0, 1.0, 1.0)):
        self.sigma = float(sigma)
        self.kernel_radius = float(kernel_radius)
        self.length_scale = tuple(float(v) for v in length_scale)

    def struct(self, impulse_density):
        return _abi.Kernel(self.sigma, self.kernel_radius, _abi.f3(*self.length_scale), int(impulse_density))


class SparseGPNoiseGenerator:
    """SparseGPNoiseGenerator(kernel, impulseDensity) (gp/gpnoise.h:23-49), batched on the GPU."""

    def __init__(self, kernel, impulse_density):
        self.kernel = kernel
        self.impulse_density = int(impulse_density)
        self._k = kernel.struct(impulse_density)

    def raw_noise(self, p, seed, cond=None, out=None, stream=None):
        """RawNoise(p, seed) for n points -> (n, 4) (psi, grad psi); with `cond`
        ((n, 8) [C, u_tilde, g_tilde, active]) the Renewal+ terms are added."""
        p = _host(p, np.float32)
        seed = _host(seed, np.uint32)
        n = p.shape[0]
        c = cond_records(cond)
        _need(p, (n, 3), "p"), _need(seed, (n,), "seed"), _need(c, (n, 8), "cond")
        mem = _mem(p, seed, c, out)
        if out is None:
            out = _empty(mem == _abi.MEM_DEVICE, (n, 4), np.float32)
        check_buf(out, (n, 4))
        check(load().mupsi_gpu_psi(C.byref(self._k), n, _ptr(p), _ptr(seed), _ptr(c), _ptr(out), mem,
                                   _stream(stream)))
        return out

    def raw_noise_value(self, p, seed, cond=None, out=None, stream=None):
        p = _host(p, np.float32)
        seed = _host(seed, np.uint32)
        n = p.shape[0]
        c = cond_records(cond)
        _need(p, (n, 3), "p"), _need(seed, (n,), "seed"), _need(c, (n, 8), "cond")
        mem = _mem(p, seed, c, out)
        if out is None:
            out = _empty(mem == _abi.MEM_DEVICE, (n,), np.float32)
        check_buf(out, (n,))
        check(load().mupsi_gpu_psi_value(C.byref(self._k), n, _ptr(p), _ptr(seed), _ptr(c), _ptr(out), mem,
                                         _stream(stream)))
        return out


def bvh_build_host(vertices, faces):
    """BVH::build node array (bvh.cpp:115-193) from the library's host builder:
    (nodes (count, 8) u32 words, triIndices, root)."""
    v = np.ascontiguousarray(vertices, np.float32)
    f = np.ascontiguousarray(faces, np.int32)
    nodes = np.zeros((max(2 * len(f), 1), 8), np.uint32)
    idx = np.zeros(max(len(f), 1), np.uint32)
    cnt, root = C.c_int64(), C.c_uint32()
    check(load().mupsi_bvh_build_host(len(v), v.ctypes.data, len(f), f.ctypes.data, nodes.ctypes.data,
                                      idx.ctypes.data, C.byref(cnt), C.byref(root)))
    return nodes[: cnt.value], idx[: len(f)], root.value


class DeviceMesh:
    """A Mesh with its BVH on the device (primitives/mesh.h, bvh/bvh.h)."""

    def __init__(self, vertices, faces, vertex_normals=None, position=(0, 0, 0), scale=1.0):
        from .scene import Mesh
        self._mesh = Mesh(vertices, faces, vertex_normals, position, scale)
        self._desc = self._mesh.desc()
        h = C.c_void_p()
        check(load().mupsi_gpu_mesh_create(C.byref(self._desc), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            load().mupsi_gpu_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_occlusion(self, from_root):
        """occluded(): from node 0 as the reference (default) or from the root."""
        check(load().mupsi_gpu_mesh_set_occlusion(self.h, 1 if from_root else 0))

    def intersect(self, rays, stream=None):
        """BVH::intersect: rays (n, 8) [o, d, nearT, farT] -> (tri u32 (0xFFFFFFFF miss), (t, u, v))."""
        rays = _host(rays, np.float32)
        n = rays.shape[0]
        _need(rays, (n, 8), "rays")
        mem = _mem(rays)
        dev = mem == _abi.MEM_DEVICE
        tri, tuv = _empty(dev, (n,), np.uint32), _empty(dev, (n, 3), np.float32)
        check(load().mupsi_gpu_bvh_intersect(self.h, n, _ptr(rays), _ptr(tri), _ptr(tuv), mem, _stream(stream)))
        return tri, tuv

    def occluded(self, rays, stream=None):
        rays = _host(rays, np.float32)
        n = rays.shape[0]
        _need(rays, (n, 8), "rays")
        mem = _mem(rays)
        out = _empty(mem == _abi.MEM_DEVICE, (n,), np.uint8)
        check(load().mupsi_gpu_bvh_occluded(self.h, n, _ptr(rays), _ptr(out), mem, _stream(stream)))
        return out

    def closest(self, p, stream=None):
        """BVH::closest: p (n, 3) -> (tri, (dist, q xyz))"""
        p = _host(p, np.float32)
        n = p.shape[0]
        _need(p, (n, 3), "p")
        mem = _mem(p)
        dev = mem == _abi.MEM_DEVICE
        tri, dq = _empty(dev, (n,), np.uint32), _empty(dev, (n, 4), np.float32)
        check(load().mupsi_gpu_bvh_closest(self.h, n, _ptr(p), _ptr(tri), _ptr(dq), mem, _stream(stream)))
        return tri, dq

    def queries(self, p, stream=None):
        """Mesh::inside and Mesh::distToPoint: -> (inside u8, tri, (dist, q xyz))"""
        p = _host(p, np.float32)
        n = p.shape[0]
        _need(p, (n, 3), "p")
        mem = _mem(p)
        dev = mem == _abi.MEM_DEVICE
        ins, tri, dq = _empty(dev, (n,), np.uint8), _empty(dev, (n,), np.uint32), _empty(dev, (n, 4), np.float32)
        check(load().mupsi_gpu_mesh_queries(self.h, n, _ptr(p), _ptr(ins), _ptr(tri), _ptr(dq), mem,
                                            _stream(stream)))
        return ins, tri, dq


TUNING_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
_TUNING_KEYS = ("march_block", "min_group", "shade_block", "wave_paths", "block_rays", "lane_rays", "lane_max_tris",
                "mu_batch")
_tuning_applied = False


def release_pools():
    """Give the device memory kept from released scenes back to the driver
    (mupsi_gpu_release_pools); call it when no scene is rendering."""
    check(load().mupsi_gpu_release_pools())


def get_tuning():
    """The launch shapes in use (mupsi_gpu_get_tuning) as a dict."""
    t = _abi.Tuning()
    check(load().mupsi_gpu_get_tuning(C.byref(t)))
    return {k: getattr(t, k) for k in _TUNING_KEYS}


def set_tuning(**kw):
    """Change some launch shapes (march_block, min_group, shade_block, wave_paths, block_rays, lane_rays,
    lane_max_tris, mu_batch). The committed tuning file is applied first, so a value set
    here is not replaced when the first scene is created."""
    if kw:
        _ensure_tuning()
    cur = get_tuning()
    for k, v in kw.items():
        if k not in _TUNING_KEYS:
            raise KeyError(k)
        cur[k] = int(v)
    check(load().mupsi_gpu_set_tuning(C.byref(_abi.Tuning(*[cur[k] for k in _TUNING_KEYS]))))
    return cur


def apply_tuning_file(path=TUNING_FILE):
    """Apply the autotuner's choice (mupsi_b200/autotune.py) if its file exists."""
    global _tuning_applied
    _tuning_applied = True
    if not os.path.exists(path):
        return None
    with open(path) as f:
        chosen = json.load(f)["tuning"]
    return set_tuning(**{k: chosen[k] for k in _TUNING_KEYS if k in chosen})


def _ensure_tuning():
    if not _tuning_applied:
        apply_tuning_file()


class GpuScene:
    """A scene on the device: the RenderContext plus GPMedium/MeanFunction batch probes."""

    def __init__(self, scene: Scene):
        _ensure_tuning()
        self.scene = scene
        self._desc = scene.desc()
        h = C.c_void_p()
        check(load().mupsi_gpu_scene_create(C.byref(self._desc), C.byref(h)))
        self.h = h
        for i, m in enumerate(scene.media):
            if m.get("kind") == "sdf":
                self.set_sdf_medium(i)
            elif m.get("kind") == "external_gp":
                self.set_external_gp_medium(i, m["res"], m["bmin"], m["bmax"], m["mean_grid"], m["var_grid"],
                                            m["noise_scale"])
        if getattr(scene, "sky_texture", None) is not None:
            self.set_sky_texture(scene.sky_texture)
        for i, p in enumerate(scene.primitives):
            if p.get("texture") is not None:
                m = scene.meshes[p["mesh"]]
                self.set_albedo_texture(i, p["texture"], m.texcoords, m.face_texcoords)

    def close(self):
        if self.h:
            load().mupsi_gpu_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mean(self, medium, p, stream=None):
        """MeanFunction eval + gradient -> (n, 4)"""
        p = _host(p, np.float32)
        _need(p, (p.shape[0], 3), "p")
        mem = _mem(p)
        out = _empty(mem == _abi.MEM_DEVICE, (p.shape[0], 4), np.float32)
        check(load().mupsi_gpu_mean(self.h, medium, p.shape[0], _ptr(p), _ptr(out), mem, _stream(stream)))
        return out

    def eval_with_gradient(self, medium, p, seed, cond=None, stream=None):
        """GPMedium::evalWithGradient(p, seed, state) -> (n, 4)"""
        p = _host(p, np.float32)
        seed = _host(seed, np.uint32)
        c = cond_records(cond)
        _need(p, (p.shape[0], 3), "p"), _need(seed, (p.shape[0],), "seed"), _need(c, (p.shape[0], 8), "cond")
        mem = _mem(p, seed, c)
        out = _empty(mem == _abi.MEM_DEVICE, (p.shape[0], 4), np.float32)
        check(load().mupsi_gpu_medium_eval(self.h, medium, p.shape[0], _ptr(p), _ptr(seed), _ptr(c), _ptr(out), mem,
                                           _stream(stream)))
        return out

    def sample_distance(self, medium, rays, seed, cond=None, stream=None):
        """GPMedium::sampleDistance -> (n, 8) [exited, t, p xyz, normal xyz] (exited as float)."""
        rays = _host(rays, np.float32)
        seed = _host(seed, np.uint32)
        c = cond_records(cond)
        n = rays.shape[0]
        _need(rays, (n, 8), "rays"), _need(seed, (n,), "seed"), _need(c, (n, 8), "cond")
        mem = _mem(rays, seed, c)
        out = _empty(mem == _abi.MEM_DEVICE, (rays.shape[0], 8), np.float32)
        check(load().mupsi_gpu_sample_distance(self.h, medium, rays.shape[0], _ptr(rays), _ptr(seed), _ptr(c),
                                               _ptr(out), mem, _stream(stream)))
        if mem == _abi.MEM_DEVICE:
            res = out.clone()
            res[:, 0] = out.view(torch.int32)[:, 0].float()
            return res
        res = out.copy()
        res[:, 0] = out.view(np.uint32)[:, 0].astype(np.float32)
        return res

    def transmittance(self, medium, rays, seed, cond=None, stream=None):
        """Medium::transmittance of (n, 8) rays [o xyz, d xyz, near, far] -> (n,) in {0, 1}."""
        rays = _host(rays, np.float32)
        seed = _host(seed, np.uint32)
        c = cond_records(cond)
        n = rays.shape[0]
        _need(rays, (n, 8), "rays"), _need(seed, (n,), "seed"), _need(c, (n, 8), "cond")
        mem = _mem(rays, seed, c)
        out = _empty(mem == _abi.MEM_DEVICE, (rays.shape[0],), np.float32)
        check(load().mupsi_gpu_transmittance(self.h, medium, rays.shape[0], _ptr(rays), _ptr(seed), _ptr(c),
                                             _ptr(out), mem, _stream(stream)))
        return out

    def sample_condition(self, medium, samples, seed, stream=None):
        """GPMedium::sampleCondition: samples (n, 7) [exited, p xyz, normal xyz] -> (n, 8) [C, u, g, active]."""
        samples = np.asarray(samples, np.float32)
        seed = np.ascontiguousarray(seed, np.uint32)
        n = samples.shape[0]
        _need(samples, (n, 7), "samples"), _need(seed, (n,), "seed")
        ms = np.zeros((n, 8), np.float32)
        ms.view(np.uint32)[:, 0] = samples[:, 0].astype(np.uint32)
        ms[:, 2:5] = samples[:, 1:4]
        ms[:, 5:8] = samples[:, 4:7]
        out = np.zeros((n, 8), np.float32)
        check(load().mupsi_gpu_sample_condition(self.h, medium, n, ms.ctypes.data, seed.ctypes.data, out.ctypes.data,
                                                _abi.MEM_HOST, _stream(stream)))
        res = out.copy()
        res[:, 7] = out.view(np.uint32)[:, 7].astype(np.float32)
        return res

    def trace_noalloc(self, x, y, k, out, stream=None):
        """PathTracer::trace for at most 16384 samples without any device
        allocation: x, y, k (int32) and out ((n, 3) float32) must be CUDA tensors.
        Calls share one static scratch array; do not overlap them on the GPU."""
        for a in (x, y, k, out):
            if not _is_dev(a):
                raise ValueError("trace_noalloc takes CUDA tensors only")
        n = x.shape[0]
        for a, nm in ((y, "y"), (k, "k")):
            check_buf(a, (n,), np.int32, nm)
        check_buf(x, (n,), np.int32, "x")
        check_buf(out, (n, 3))
        check(load().mupsi_gpu_trace_samples_noalloc(self.h, x.shape[0], _ptr(x), _ptr(y), _ptr(k), _ptr(out),
                                                     _stream(stream)))
        return out

    def set_sky_texture(self, img):
        """Skydrome BitmapTexture: (h, w, 3) float RGB, row 0 at the top; None removes it."""
        if img is None:
            check(load().mupsi_gpu_scene_set_sky_texture(self.h, 0, 0, None))
            return
        img = np.ascontiguousarray(img, np.float32)
        check(load().mupsi_gpu_scene_set_sky_texture(self.h, img.shape[1], img.shape[0], img.ctypes.data))

    def size(self):
        """(width, height) of the scene's image."""
        w, h = C.c_int32(), C.c_int32()
        check(load().mupsi_gpu_scene_get_size(self.h, C.byref(w), C.byref(h)))
        return w.value, h.value

    def set_gp_mode(self, mode):
        """GPSettings::gpMode: _abi.GP_SINGLE_REALIZATION or _abi.GP_RENEWAL_PLUS."""
        check(load().mupsi_gpu_scene_set_gp_mode(self.h, int(mode)))

    def set_skip_medium(self, skip):
        """PathTracerSettings::skip_medium: pass through media without marching."""
        check(load().mupsi_gpu_scene_set_skip_medium(self.h, 1 if skip else 0))

    def set_kernel(self, medium, kernel):
        """Replace a GP medium's SparseSEKernel (an SparseSEKernel with its
        impulse density: kernel.struct(points_per_cell))."""
        check(load().mupsi_gpu_scene_set_kernel(self.h, medium, C.byref(kernel)))

    def set_sdf_medium(self, medium):
        """Make medium `medium` an SDFMedium over its mean function."""
        check(load().mupsi_gpu_scene_set_sdf_medium(self.h, medium))

    def set_external_gp_medium(self, medium, resolution, bounds_min, bounds_max, mean_grid, variance_grid=None,
                               noise_scale=1.0):
        """Make medium `medium` an ExternalGPMedium over GridMeanFunction grids
        (resolution^3 float32, x-major; variance None: no noise)."""
        mg = np.ascontiguousarray(mean_grid, np.float32).reshape(-1)
        vg = None if variance_grid is None else np.ascontiguousarray(variance_grid, np.float32).reshape(-1)
        cells = int(resolution) ** 3
        if mg.size != cells or (vg is not None and vg.size != cells):
            raise ValueError("grids need resolution^3 samples")
        lo = (C.c_float * 3)(*bounds_min)
        hi = (C.c_float * 3)(*bounds_max)
        check(load().mupsi_gpu_scene_set_external_gp_medium(self.h, medium, int(resolution), lo, hi, mg.ctypes.data,
                                                            None if vg is None else vg.ctypes.data,
                                                            float(noise_scale)))

    def set_albedo_texture(self, primitive, img, texcoords=None, face_texcoords=None):
        """Lambertian BitmapTexture albedo of a mesh primitive: (h, w, 3) float
        RGB, row 0 at the top, at the mesh's texcoords (T, 2) indexed per face
        by face_texcoords (F, 3), or at the hit's barycentrics when texcoords is
        None. img None removes it."""
        if img is None:
            check(load().mupsi_gpu_scene_set_albedo_texture(self.h, primitive, 0, None, None, 0, 0, None))
            return
        img = np.ascontiguousarray(img, np.float32)
        if texcoords is None:
            n, tc, ft = 0, None, None
        else:
            tc = np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2)
            ft = np.ascontiguousarray(face_texcoords, np.int32).reshape(-1, 3)
            n = len(tc)
        check(load().mupsi_gpu_scene_set_albedo_texture(
            self.h, primitive, n, None if tc is None else tc.ctypes.data, None if ft is None else ft.ctypes.data,
            img.shape[1], img.shape[0], img.ctypes.data))

    def set_occlusion(self, from_root):
        """Shadow rays: BVH::occluded from node 0 as the reference (default) or from the root."""
        check(load().mupsi_gpu_scene_set_occlusion(self.h, 1 if from_root else 0))

    def set_mean_eval(self, medium, every_step):
        """Mesh mean at every visited step (the plain exact form) or lazily (default)."""
        check(load().mupsi_gpu_scene_set_mean_eval(self.h, medium, 1 if every_step else 0))

    def profile(self, enable=True, bvh=False):
        """Count march work and time the wavefront kernels with CUDA events;
        bvh=True also counts BVH nodes and triangles (counted traversals: slower,
        so take times from a render without it)."""
        check(load().mupsi_gpu_scene_profile(self.h, (2 if bvh else 1) if enable else 0))

    def stats(self, reset=False):
        st = _abi.RenderStats()
        check(load().mupsi_gpu_scene_stats(self.h, C.byref(st), 1 if reset else 0))
        out = {}
        for f, _ in _abi.RenderStats._fields_:
            v = getattr(st, f)
            out[f] = list(v) if hasattr(v, "__len__") else v
        return out

    def trace(self, x, y, k, stream=None):
        """PathTracer::trace(pixel (x, y), ctx, 42, k) for n samples -> (n, 3) radiance."""
        x, y, k = (_host(a, np.int32) for a in (x, y, k))
        mem = _mem(x, y, k)
        n = x.shape[0]
        _need(x, (n,), "x"), _need(y, (n,), "y"), _need(k, (n,), "k")
        if mem == _abi.MEM_DEVICE:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        else:
            out = np.empty((n, 3), np.float32)
        check(load().mupsi_gpu_trace_samples(self.h, n, _ptr(x), _ptr(y), _ptr(k), _ptr(out), mem, _stream(stream)))
        return out


class GpuRenderer:
    """Renderer (rendering/renderer.h:11-41) on the GPU: prepare_render + start_render_progressive."""

    def __init__(self):
        self.scene = None
        self.cancel_flag = C.c_int32(0)

    def prepare_render(self, scene):
        self.scene = scene if isinstance(scene, GpuScene) else GpuScene(scene)
        return self.scene

    def cancel(self):
        self.cancel_flag.value = 1

    def start_render_progressive(self, target_spp, on_spp=None, spp_begin=0, out=None, moments=False, stream=None):
        """Trace passes [spp_begin, target_spp) and return the averaged framebuffer
        (h, w, 3) (and FP64 moments (h, w, 6) if asked). Returns None if cancelled,
        as the reference returns false."""
        s = self.scene.scene
        h, w = s.height, s.width
        dev = out is not None and _is_dev(out)
        if out is None:
            out = np.empty((h, w, 3), np.float32)
        check_buf(out, (h, w, 3))
        mom = np.zeros((h, w, 6), np.float64) if moments else None
        cb = _abi.ON_SPP(lambda k, user: on_spp(k)) if on_spp else _abi.ON_SPP()
        args = _abi.RenderArgs(spp_begin, target_spp, C.pointer(self.cancel_flag), cb, None, _ptr(out),
                               _abi.MEM_DEVICE if dev else _abi.MEM_HOST, None if mom is None else mom.ctypes.data,
                               _stream(stream))
        code = load().mupsi_gpu_render(self.scene.h, C.byref(args))
        if code == _abi.ERR_CANCELLED:
            return None
        check(code)
        return (out, mom) if moments else out


class GpuDisplay:
    """Headless double-buffered progressive display over one GpuScene
    (Controller's render control, controller/controller.cpp:266-375): a native
    render thread publishes frames; copy_raw / copy_tonemapped read the
    latest complete one."""

    def __init__(self, scene):
        self.scene = scene if isinstance(scene, GpuScene) else GpuScene(scene)
        self.width, self.height = self.scene.size()
        h = C.c_void_p()
        check(load().mupsi_gpu_display_create(self.scene.h, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            load().mupsi_gpu_display_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def start_progressive(self, target_spp, passes_per_frame=1):
        check(load().mupsi_gpu_display_start_progressive(self.h, int(target_spp), int(passes_per_frame)))

    def start(self, spp):
        check(load().mupsi_gpu_display_start(self.h, int(spp)))

    def cancel(self):
        load().mupsi_gpu_display_cancel(self.h)

    def stop(self):
        check(load().mupsi_gpu_display_stop(self.h))

    def running(self):
        return bool(load().mupsi_gpu_display_running(self.h))

    def is_spp_pass_done(self):
        return bool(load().mupsi_gpu_display_spp_pass_done(self.h))

    def ack_spp_pass(self):
        load().mupsi_gpu_display_ack_spp_pass(self.h)

    def current_spp(self):
        return int(load().mupsi_gpu_display_current_spp(self.h))

    def _dst(self, out):
        if out is None:
            return np.empty((self.height, self.width, 3), np.float32)
        if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.ndim == 3 and out.shape[2] == 3
                and out.flags.c_contiguous):
            raise ValueError("out must be a C-contiguous (h, w, 3) float32 array")
        return out

    def copy_raw(self, out=None):
        """The front frame (h, w, 3) float32, un-tonemapped (copyDisplayRawTo).
        The library checks out's size against the scene's."""
        out = self._dst(out)
        check(load().mupsi_gpu_display_copy_raw(self.h, out.ctypes.data, out.shape[1], out.shape[0]))
        return out

    def copy_tonemapped(self, out=None):
        """The front frame Reinhard tonemapped v / (1 + v) (copyDisplayTo)."""
        out = self._dst(out)
        check(load().mupsi_gpu_display_copy_tonemapped(self.h, out.ctypes.data, out.shape[1], out.shape[0]))
        return out


class GpuBatch:
    """Several scenes rendered together (mupsi_gpu_batch_*): one wave stream
    whose paths carry their scene's index. No reference counterpart (the
    reference renders one scene per Renderer)."""

    SCHEDULES = {"shortest_first": _abi.SCHEDULE_SHORTEST_FIRST, "in_order": _abi.SCHEDULE_IN_ORDER,
                 "interleaved": _abi.SCHEDULE_INTERLEAVED}

    def __init__(self, scenes):
        _ensure_tuning()
        self.scenes = [sc if isinstance(sc, GpuScene) else GpuScene(sc) for sc in scenes]
        arr = (C.c_void_p * len(self.scenes))(*[sc.h.value for sc in self.scenes])
        h = C.c_void_p()
        check(load().mupsi_gpu_batch_create(len(self.scenes), arr, C.byref(h)))
        self.h = h
        self.cancel_flag = C.c_int32(0)

    def close(self):
        if self.h:
            load().mupsi_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def cancel(self):
        self.cancel_flag.value = 1

    def render(self, spp, out=None, use_graphs=True, schedule="shortest_first", stream=None):
        """Render scene i at spp[i] passes. `out`: None (host images are
        returned), or a list of (h, w, 3) float32 buffers, all numpy or all CUDA
        tensors (entries may be None). Returns (images, done_ms): done_ms[i] is
        scene i's completion time in ms from the start of the first wave.
        Returns None if cancelled."""
        n = len(self.scenes)
        if len(spp) != n:
            raise ValueError("one spp per scene")
        if out is None:
            out = [np.empty((sc.scene.height, sc.scene.width, 3), np.float32) for sc in self.scenes]
        if len(out) != n:
            raise ValueError("one output per scene")
        for o, sc in zip(out, self.scenes):
            if o is not None:
                check_buf(o, (sc.scene.height, sc.scene.width, 3))
        dev = _mem(*out) == _abi.MEM_DEVICE
        sp = (C.c_int32 * n)(*[int(v) for v in spp])
        ptrs = (C.c_void_p * n)(*[_ptr(o) for o in out])
        done = (C.c_float * n)()
        args = _abi.BatchArgs(sp, ptrs, _abi.MEM_DEVICE if dev else _abi.MEM_HOST, C.pointer(self.cancel_flag), done,
                              1 if use_graphs else 0, self.SCHEDULES[schedule], _stream(stream))
        code = load().mupsi_gpu_batch_render(self.h, C.byref(args))
        if code == _abi.ERR_CANCELLED:
            return None
        check(code)
        return out, np.array(list(done), np.float64)

    def info(self):
        i = _abi.BatchInfo()
        check(load().mupsi_gpu_batch_info(self.h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in _abi.BatchInfo._fields_}
