"""Scene descriptions: scene.json loading and the synthetic benchmark scenes.

`Scene` holds what the reference's Controller::load builds
(controller/controller.cpp:40-264) as flat numpy arrays and turns it into the
C ABI's mupsi_scene_desc (include/mupsi_gpu.h). The arrays stay referenced by
the Scene, so a descriptor is valid while its Scene lives.
"""
import ctypes as C
import json
import math
import os
import warnings

import numpy as np

from . import _abi

DEFAULT_ALBEDO = 0.8  # Bsdf::default_albedo_ (bsdf/bsdf.cpp:11)


class Mesh:
    """Triangle mesh (primitives/mesh.h): object-space vertices/faces + T*S transform."""

    def __init__(self, vertices, faces, vertex_normals=None, position=(0.0, 0.0, 0.0), scale=1.0, texcoords=None,
                 face_texcoords=None):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
        self.vertex_normals = None
        if vertex_normals is not None:
            # Mesh::interpolateNormal indexes normals_ by vertex id (mesh.cpp:163-166):
            # the first len(vertices) normals are the ones read; with fewer normals
            # than vertices the reference reads past its array, so they are dropped
            vn = np.ascontiguousarray(vertex_normals, dtype=np.float32).reshape(-1, 3)
            if len(vn) >= len(self.vertices):
                self.vertex_normals = np.ascontiguousarray(vn[:len(self.vertices)])
            else:
                warnings.warn(f"{len(vn)} normals for {len(self.vertices)} vertices: using face normals")
        self.position = tuple(float(v) for v in position)
        self.scale = float(scale)
        # OBJ texture coordinates (vt) and per-face indices into them; None:
        # a textured primitive reads its texture at the hit's barycentrics
        self.texcoords = None if texcoords is None else np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2)
        self.face_texcoords = (None if face_texcoords is None else
                               np.ascontiguousarray(face_texcoords, np.int32).reshape(-1, 3))
        if (self.texcoords is None) != (self.face_texcoords is None):
            raise ValueError("texcoords and face_texcoords go together")
        if self.face_texcoords is not None and (len(self.face_texcoords) != len(self.faces) or (
                self.face_texcoords.size and (self.face_texcoords.min() < 0 or
                                              self.face_texcoords.max() >= len(self.texcoords)))):
            raise ValueError("face_texcoords must index texcoords, one triple per face")

    def desc(self):
        return _abi.MeshDesc(
            len(self.vertices), self.vertices.ctypes.data, len(self.faces), self.faces.ctypes.data,
            None if self.vertex_normals is None else self.vertex_normals.ctypes.data,
            _abi.f3(*self.position), self.scale)


def load_obj(path, texcoords=False):
    """OBJ file through the library's reader (mupsi_obj_load), which follows
    Mesh::fetchFrom (primitives/mesh.cpp:20-136) down to its number parsing.
    Returns (vertices, faces, normals or None), plus (texcoords,
    face_texcoords) with texcoords=True: None, None for a file without vt
    lines (interpolateTexcoord then yields the barycentrics, mesh.cpp:175-177)."""
    from .lib import check, load
    L = load()
    o = _abi.Obj()
    check(L.mupsi_obj_load(os.fsencode(path), C.byref(o)))
    try:
        def arr(ptr, n, cols, dt):
            if n == 0:
                return None
            return np.ctypeslib.as_array(ptr, shape=(n * cols,)).astype(dt).reshape(n, cols)
        out = (arr(o.vertices, o.num_vertices, 3, np.float32), arr(o.faces, o.num_faces, 3, np.int32),
               arr(o.normals, o.num_normals, 3, np.float32))
        if texcoords:
            out = out + (arr(o.texcoords, o.num_texcoords, 2, np.float32),
                         arr(o.face_texcoords, o.num_faces if o.num_texcoords else 0, 3, np.int32))
        return out
    finally:
        L.mupsi_obj_free(C.byref(o))


def save_obj(path, vertices, faces, texcoords=None, face_texcoords=None):
    """Write a mesh as OBJ (vertices and texcoords at full float32 precision,
    1-based faces, v/vt corners when texcoords are given)."""
    v = np.asarray(vertices, np.float32)
    f = np.asarray(faces, np.int64) + 1
    with open(path, "w") as fh:
        fh.write("".join("v %.9g %.9g %.9g\n" % tuple(r) for r in v.tolist()))
        if texcoords is None:
            fh.write("".join("f %d %d %d\n" % tuple(r) for r in f.tolist()))
        else:
            t = np.asarray(texcoords, np.float32).reshape(-1, 2)
            ft = np.asarray(face_texcoords, np.int64).reshape(-1, 3) + 1
            fh.write("".join("vt %.9g %.9g\n" % tuple(r) for r in t.tolist()))
            fh.write("".join("f %d/%d %d/%d %d/%d\n" % (a, ta, b, tb, c, tc)
                             for (a, b, c), (ta, tb, tc) in zip(f.tolist(), ft.tolist())))


class Scene:
    """Python-side mirror of the scene the reference builds from scene.json."""

    def __init__(self):
        self.width = 256
        self.height = 256
        self.spp = 1
        self.max_bounce = 3          # PathTracerSettings default (trace.h:17)
        self.max_medium_bounce = 3
        self.gp_mode = _abi.GP_SINGLE_REALIZATION
        self.cam_pos = (0.0, 0.0, 0.0)
        self.cam_dir = (0.0, 0.0, -1.0)
        self.cam_up = (0.0, 1.0, 0.0)
        self.cam_fov = 45.0
        self.eps = float(np.float32(1e-4))
        self.nearteps = float(np.float32(1e-4) * np.float32(15))
        self.sky = None              # None = no skydrome; else constant RGB radiance
        self.sky_texture = None      # (h, w, 3) float32 skydrome image, row 0 at the top (replaces `sky`)
        self.media = []              # dicts: mean_type, center, radius, mesh, sigma, length, aniso, ppc
        self.meshes = []             # Mesh
        self.primitives = []         # dicts
        self._keep = []

    # -- construction helpers -------------------------------------------------
    def add_medium(self, mean_type="sphere", center=(0, 0, 0), radius=70.0, mesh=-1, sigma=1.0, length_scale=1.0,
                   aniso=(1.0, 1.0, 1.0), points_per_cell=3, kind="gp"):
        """A GPMedium (kind "gp") over a sphere or mesh mean with an SE kernel,
        or an SDFMedium (kind "sdf": the mean itself is the field; the kernel
        is unused)."""
        if kind not in ("gp", "sdf"):
            raise ValueError(f"unknown medium kind {kind!r}")
        self.media.append(dict(kind=kind, mean_type=_abi.MEAN_SPHERE if mean_type == "sphere" else _abi.MEAN_MESH,
                               center=tuple(center), radius=float(radius), mesh=int(mesh), sigma=float(sigma),
                               length=float(length_scale), aniso=tuple(aniso), ppc=int(points_per_cell)))
        return len(self.media) - 1

    def add_external_gp_medium(self, resolution, bounds_min, bounds_max, mean_grid, variance_grid=None,
                               noise_scale=1.0):
        """An ExternalGPMedium (medium/externalgpmedium.h): GridMeanFunction mean
        and variance grids of resolution^3 float32 samples, x-major
        ((i * res + j) * res + k), over [bounds_min, bounds_max];
        variance_grid None: no noise."""
        res = int(resolution)
        cells = res ** 3
        mg = np.ascontiguousarray(mean_grid, np.float32).reshape(-1)
        vg = None if variance_grid is None else np.ascontiguousarray(variance_grid, np.float32).reshape(-1)
        if res < 2 or mg.size != cells or (vg is not None and vg.size != cells):
            raise ValueError("grids need resolution^3 samples, resolution >= 2")
        self.media.append(dict(kind="external_gp", mean_type=_abi.MEAN_SPHERE, center=(0.0, 0.0, 0.0), radius=1.0,
                               mesh=-1, sigma=1.0, length=1.0, aniso=(1.0, 1.0, 1.0), ppc=3, res=res,
                               bmin=tuple(float(v) for v in bounds_min), bmax=tuple(float(v) for v in bounds_max),
                               mean_grid=mg, var_grid=vg, noise_scale=float(noise_scale)))
        return len(self.media) - 1

    def add_mesh(self, mesh):
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_sphere(self, center, radius, bsdf=_abi.BSDF_LAMBERTIAN, albedo=DEFAULT_ALBEDO, emission=None,
                   int_medium=-1, ext_medium=-1):
        self.primitives.append(dict(type=_abi.PRIM_SPHERE, center=tuple(center), radius=float(radius), mesh=-1,
                                    bsdf=bsdf, albedo=_rgb(albedo), emission=emission, int_medium=int_medium,
                                    ext_medium=ext_medium))

    def add_mesh_primitive(self, mesh_index, bsdf=_abi.BSDF_LAMBERTIAN, albedo=DEFAULT_ALBEDO, emission=None,
                           int_medium=-1, ext_medium=-1, texture=None):
        """texture: (h, w, 3) float RGB albedo image (row 0 at the top) of a
        Lambertian mesh, read at the mesh's texcoords; replaces `albedo`."""
        if texture is not None:
            if bsdf != _abi.BSDF_LAMBERTIAN:
                raise ValueError("albedo textures need a Lambertian BSDF")
            texture = np.ascontiguousarray(texture, np.float32)
            if texture.ndim != 3 or texture.shape[2] != 3 or texture.shape[0] < 1 or texture.shape[1] < 1:
                raise ValueError("texture must be (h, w, 3)")
        self.primitives.append(dict(type=_abi.PRIM_MESH, center=(0, 0, 0), radius=1.0, mesh=mesh_index, bsdf=bsdf,
                                    albedo=_rgb(albedo), emission=emission, int_medium=int_medium,
                                    ext_medium=ext_medium, texture=texture))

    # -- scene.json (controller.cpp:40-264) ------------------------------------
    @classmethod
    def from_json(cls, path_or_dict, sky=None, base_dir=None):
        """Build a Scene the way Controller::load does. `sky` adds a constant
        skydrome (Skydrome() is 1.0) since the reference only takes an image path."""
        if isinstance(path_or_dict, dict):
            j = path_or_dict
            base_dir = base_dir or os.getcwd()
        else:
            with open(path_or_dict) as fh:
                j = json.load(fh)
            base_dir = base_dir or os.path.dirname(os.path.abspath(path_or_dict))
        s = cls()
        if "max_bounce" in j:
            s.max_bounce = int(j["max_bounce"])
        if "max_medium_bounce" in j:
            s.max_medium_bounce = int(j["max_medium_bounce"])
        if "spp" in j:
            s.spp = int(j["spp"])
        s.width = int(j.get("width", 256))
        s.height = int(j.get("height", 256))
        cam = j["camera"]
        s.cam_pos = tuple(float(v) for v in cam["pos"])
        s.cam_dir = tuple(float(v) for v in cam["dir"])
        s.cam_up = tuple(float(v) for v in cam.get("up", [0, 1, 0]))
        s.cam_fov = float(cam.get("fov", 45.0))
        s.gp_mode = _abi.GP_RENEWAL_PLUS if j.get("gp_mode", "single_realization") == "renewal_plus" \
            else _abi.GP_SINGLE_REALIZATION
        # the medium of `int_medium` primitives: gp_medium, else sdf_medium, else
        # external_gp_medium (controller.cpp:225-229)
        gpm_index = -1
        if "gp_medium" in j:
            g = j["gp_medium"]
            mt = g.get("mean_type", "sphere")
            kern = j.get("kernel", {})
            kw = dict(sigma=kern.get("sigma", 1.0), length_scale=kern.get("length_scale", 1.0),
                      aniso=tuple(kern.get("aniso", [1, 1, 1])), points_per_cell=kern.get("points_per_cell", 3))
            if mt == "sphere":
                gpm_index = s.add_medium("sphere", center=g["mean_center"], radius=g.get("mean_radius", 70.0), **kw)
            elif mt == "mesh":
                v, f, n = load_obj(_resolve(base_dir, g["file"]))
                t = g.get("transform", {})
                mi = s.add_mesh(Mesh(v, f, n, position=t.get("position", (0, 0, 0)), scale=t.get("scale", 1.0)))
                gpm_index = s.add_medium("mesh", mesh=mi, **kw)
            else:
                raise ValueError(f"unknown mean_type: {mt}")
        elif "sdf_medium" in j:  # controller.cpp:154-182
            g = j["sdf_medium"]
            mt = g.get("mean_type", "sphere")
            if mt == "sphere":
                gpm_index = s.add_medium("sphere", center=g["mean_center"], radius=g.get("mean_radius", 70.0),
                                         kind="sdf")
            elif mt == "mesh":
                v, f, n = load_obj(_resolve(base_dir, g["file"]))
                t = g.get("transform", {})
                mi = s.add_mesh(Mesh(v, f, n, position=t.get("position", (0, 0, 0)), scale=t.get("scale", 1.0)))
                gpm_index = s.add_medium("mesh", mesh=mi, kind="sdf")
            else:
                raise ValueError(f"unknown sdf_medium mean_type: {mt}")
        elif "external_gp_medium" in j:  # controller.cpp:184-189
            g = j["external_gp_medium"]
            res = int(g.get("resolution", 48))
            # grid files: the config's directory + the name, as a string
            # (an absolute name too ends up under that directory)
            cdir = base_dir.rstrip("/") + "/"
            mean = load_grid(cdir + g["mean_file"], res)
            var = None
            if g.get("variance_file", ""):
                var = load_grid(cdir + g["variance_file"], res)
            gpm_index = s.add_external_gp_medium(res, g["bounds_min"], g["bounds_max"], mean, var,
                                                 g.get("noise_scale", 1.0))
        if "skydrome" in j:
            s.sky_texture = load_texture_image(_resolve(base_dir, j["skydrome"]))
        if sky is not None:
            s.sky = _rgb(sky)
        if "primitives" not in j or not isinstance(j["primitives"], list):
            raise ValueError("no primitives array in config")
        bsdfs = {"lambertian": _abi.BSDF_LAMBERTIAN, "null": _abi.BSDF_NULL, "specular": _abi.BSDF_SPECULAR}
        for pj in j["primitives"]:
            typ = pj.get("type", "sphere")
            bsdf = bsdfs.get(pj.get("bsdf", "lambertian"), _abi.BSDF_LAMBERTIAN)
            if typ == "sphere":
                em = _rgb(pj["emission"]) if "emission" in pj else None
                s.add_sphere(pj["center"], pj.get("radius", 100.0), bsdf=bsdf, emission=em,
                             int_medium=gpm_index if "int_medium" in pj else -1)
            elif typ == "mesh":
                tex = None
                if "texture" in pj and pj.get("bsdf", "lambertian") == "lambertian":  # controller.cpp:240-243
                    tex = load_texture_image(_resolve(base_dir, pj["texture"]))
                v, f, n, tc, ftc = load_obj(_resolve(base_dir, pj["file"]), texcoords=True)
                t = pj.get("transform", {})
                mi = s.add_mesh(Mesh(v, f, n, position=t.get("position", (0, 0, 0)), scale=t.get("scale", 1.0),
                                     texcoords=tc, face_texcoords=ftc))
                s.add_mesh_primitive(mi, bsdf=bsdf, texture=tex)
            # unknown primitive types are skipped, as the reference does
        return s

    # -- C ABI descriptor -------------------------------------------------------
    def desc(self):
        media = (_abi.MediumDesc * max(len(self.media), 1))()
        for i, m in enumerate(self.media):
            media[i] = _abi.MediumDesc(m["mean_type"], _abi.f3(*m["center"]), m["radius"], m["mesh"],
                                       _abi.Kernel(m["sigma"], m["length"], _abi.f3(*m["aniso"]), m["ppc"]))
        meshes = (_abi.MeshDesc * max(len(self.meshes), 1))()
        for i, m in enumerate(self.meshes):
            meshes[i] = m.desc()
        prims = (_abi.PrimitiveDesc * max(len(self.primitives), 1))()
        for i, p in enumerate(self.primitives):
            em = p["emission"]
            prims[i] = _abi.PrimitiveDesc(p["type"], _abi.f3(*p["center"]), p["radius"], p["mesh"], p["bsdf"],
                                          _abi.f3(*p["albedo"]), 0 if em is None else 1,
                                          _abi.f3(*(em if em is not None else (0, 0, 0))), p["int_medium"],
                                          p["ext_medium"])
        d = _abi.SceneDesc()
        d.width, d.height, d.spp = self.width, self.height, self.spp
        d.max_bounce, d.max_medium_bounce, d.gp_mode = self.max_bounce, self.max_medium_bounce, self.gp_mode
        d.cam_pos, d.cam_dir, d.cam_up = _abi.f3(*self.cam_pos), _abi.f3(*self.cam_dir), _abi.f3(*self.cam_up)
        d.cam_fov, d.eps, d.nearteps = self.cam_fov, self.eps, self.nearteps
        d.has_sky = 0 if self.sky is None else 1
        d.sky = _abi.f3(*(self.sky if self.sky is not None else (0, 0, 0)))
        d.num_media, d.media = len(self.media), C.cast(media, C.POINTER(_abi.MediumDesc))
        d.num_meshes, d.meshes = len(self.meshes), C.cast(meshes, C.POINTER(_abi.MeshDesc))
        d.num_primitives, d.primitives = len(self.primitives), C.cast(prims, C.POINTER(_abi.PrimitiveDesc))
        self._keep = [media, meshes, prims]
        return d

    def to_json(self, obj_paths=None, sky_path=None, texture_paths=None, grid_paths=None):
        """scene.json dict the reference's Controller::load accepts for this scene
        (meshes must have been written to `obj_paths` with their texcoords, a sky
        texture to `sky_path` and albedo textures to `texture_paths`, a dict
        primitive index -> path, with save_image_raw; an external GP medium's
        grids to `grid_paths` = (mean, variance or None), named relative to the
        config's directory). Returns (dict, extra_meshes): primitives the schema cannot express (non-default
        albedo) are returned as (obj_path, albedo) pairs for a harness to add."""
        j = {"width": self.width, "height": self.height, "spp": self.spp, "max_bounce": self.max_bounce,
             "max_medium_bounce": self.max_medium_bounce,
             "gp_mode": "renewal_plus" if self.gp_mode == _abi.GP_RENEWAL_PLUS else "single_realization",
             "camera": {"pos": list(self.cam_pos), "dir": list(self.cam_dir), "up": list(self.cam_up),
                        "fov": self.cam_fov}, "primitives": []}
        extra = []
        if self.sky_texture is not None:
            if sky_path is None:
                raise ValueError("a sky texture needs sky_path")
            j["skydrome"] = sky_path
        if self.media:
            if len(self.media) > 1:
                raise ValueError("scene.json holds one medium")
            m = self.media[0]
            kind = m.get("kind", "gp")
            if kind == "external_gp":
                eg = {"resolution": m["res"], "bounds_min": list(m["bmin"]), "bounds_max": list(m["bmax"]),
                      "noise_scale": m["noise_scale"], "mean_file": grid_paths[0]}
                if m["var_grid"] is not None:
                    eg["variance_file"] = grid_paths[1]
                j["external_gp_medium"] = eg
            else:
                key = "gp_medium" if kind == "gp" else "sdf_medium"
                if kind == "gp":
                    j["kernel"] = {"sigma": m["sigma"], "length_scale": m["length"], "aniso": list(m["aniso"]),
                                   "points_per_cell": m["ppc"]}
                if m["mean_type"] == _abi.MEAN_SPHERE:
                    j[key] = {"mean_type": "sphere", "mean_center": list(m["center"]), "mean_radius": m["radius"]}
                else:
                    mm = self.meshes[m["mesh"]]
                    j[key] = {"mean_type": "mesh", "file": obj_paths[m["mesh"]],
                              "transform": {"position": list(mm.position), "scale": mm.scale}}
        names = {_abi.BSDF_LAMBERTIAN: "lambertian", _abi.BSDF_NULL: "null", _abi.BSDF_SPECULAR: "specular"}
        for pi, p in enumerate(self.primitives):
            if p["type"] == _abi.PRIM_SPHERE:
                pj = {"type": "sphere", "center": list(p["center"]), "radius": p["radius"], "bsdf": names[p["bsdf"]]}
                if p["emission"] is not None:
                    pj["emission"] = list(p["emission"])
                if p["int_medium"] >= 0:
                    pj["int_medium"] = True
                j["primitives"].append(pj)
            else:
                mm = self.meshes[p["mesh"]]
                tex = p.get("texture")
                if tex is None and (p["albedo"] != _rgb(DEFAULT_ALBEDO) or mm.position != (0, 0, 0) or
                                    mm.scale != 1.0):
                    extra.append((obj_paths[p["mesh"]], p["albedo"][0]))
                else:
                    pj = {"type": "mesh", "file": obj_paths[p["mesh"]], "bsdf": names[p["bsdf"]]}
                    if tex is not None:
                        pj["texture"] = texture_paths[pi]
                        if mm.position != (0, 0, 0) or mm.scale != 1.0:
                            pj["transform"] = {"position": list(mm.position), "scale": mm.scale}
                    j["primitives"].append(pj)
        return j, extra


def load_grid(path, res):
    """A GridMeanFunction file (meanfunction.cpp:41-56): res^3 float32, x-major.
    As the reference, a short or missing file leaves the remaining samples 0
    (with a warning here)."""
    cells = res ** 3
    out = np.zeros(cells, np.float32)
    try:
        with open(path, "rb") as fh:
            data = np.frombuffer(fh.read(cells * 4), np.float32)
    except OSError:
        data = np.zeros(0, np.float32)
    if data.size < cells:
        warnings.warn(f"GridMeanFunction {path}: {data.size} of {cells} samples; the rest are 0")
    out[:data.size] = data
    return out


def load_texture_image(path):
    """An image as BitmapTexture::load reads it (texture.cpp:12-50): .hdr/.exr
    as float, other formats as 8-bit / 255, RGB, row 0 at the top. Files
    written by save_image_raw are read directly (a float one only under a
    .hdr/.exr name, as the reference asks for float pixels only there);
    everything else needs OpenCV (cv2)."""
    with open(path, "rb") as fh:
        head = fh.read(10)
    is_hdr = os.path.splitext(path)[1] in (".hdr", ".exr")
    if head == b"MUPSI_RGBF":
        if not is_hdr:
            raise OSError(f"{path}: a float image needs a .hdr or .exr name")
        return load_image_raw(path)
    if head == b"MUPSI_RGB8":
        return (load_image_raw(path).astype(np.float32) / np.float32(255.0)).astype(np.float32)
    import cv2
    img = cv2.imread(path, (cv2.IMREAD_ANYDEPTH | cv2.IMREAD_COLOR) if is_hdr else cv2.IMREAD_COLOR)
    if img is None:
        raise OSError(f"cannot load {path}")
    img = cv2.cvtColor(img, cv2.COLOR_BGR2RGB)
    return (img.astype(np.float32) if is_hdr else img.astype(np.float32) / np.float32(255.0)).copy()


def save_image_raw(path, img):
    """Write an RGB image (h, w, 3), rows from the top, in the raw formats the
    CPU oracle's image reader takes: float32 texels after "MUPSI_RGBF w h\n",
    or uint8 texels after "MUPSI_RGB8 w h\n" for a uint8 array."""
    img = np.asarray(img)
    if img.dtype != np.uint8:
        img = img.astype(np.float32)
    img = np.ascontiguousarray(img)
    magic = "MUPSI_RGB8" if img.dtype == np.uint8 else "MUPSI_RGBF"
    with open(path, "wb") as fh:
        fh.write(f"{magic} {img.shape[1]} {img.shape[0]}\n".encode())
        fh.write(img.tobytes())


def load_image_raw(path):
    """Read save_image_raw's formats: float32 or uint8 (h, w, 3)."""
    with open(path, "rb") as fh:
        magic, w, h = fh.readline().split()
        if magic not in (b"MUPSI_RGBF", b"MUPSI_RGB8"):
            raise OSError(f"{path} is not a raw MUPSI image")
        w, h = int(w), int(h)
        dt = np.float32 if magic == b"MUPSI_RGBF" else np.uint8
        n = w * h * 3
        data = np.frombuffer(fh.read(n * np.dtype(dt).itemsize), dt)
    if data.size != n:
        raise OSError(f"{path}: truncated")
    return data.reshape(h, w, 3).copy()


# the skydrome reads its image through the same BitmapTexture
load_sky_image = load_texture_image
save_sky_raw = save_image_raw


def _rgb(v):
    if isinstance(v, (int, float)):
        return (float(v),) * 3
    return tuple(float(x) for x in v)


def _resolve(base, f):
    return f if os.path.isabs(f) else os.path.join(base, f)


# ---------------------------------------------------------------------------
# Synthetic scenes
# ---------------------------------------------------------------------------

def icosphere(level):
    """Unit icosphere: 20*4^level faces, 10*4^level+2 vertices, deterministic order."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, np.int64)
    for _ in range(level):
        nv = len(verts)
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (nv + 1), uniq % (nv + 1)
        mid = verts[a] + verts[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        verts = np.concatenate([verts, mid], axis=0)
        m = inv.reshape(3, -1) + nv
        m01, m12, m20 = m[0], m[1], m[2]
        v0, v1, v2 = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.stack([np.stack([v0, m01, m20], 1), np.stack([v1, m12, m01], 1), np.stack([v2, m20, m12], 1),
                          np.stack([m01, m12, m20], 1)], axis=1).reshape(-1, 3)
    return verts, faces


def _real_sh(l, m, theta, phi):
    """Orthonormal real spherical harmonic Y_lm (theta polar, phi azimuth)."""
    x = np.cos(theta)
    am = abs(m)
    # associated Legendre P_l^|m|(x) by the standard upward recurrence
    pmm = np.ones_like(x)
    somx2 = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    fact = 1.0
    for _ in range(am):
        pmm = -pmm * fact * somx2
        fact += 2.0
    if l == am:
        plm = pmm
    else:
        pmmp1 = x * (2 * am + 1) * pmm
        if l == am + 1:
            plm = pmmp1
        else:
            for ll in range(am + 2, l + 1):
                pll = ((2 * ll - 1) * x * pmmp1 - (ll + am - 1) * pmm) / (ll - am)
                pmm, pmmp1 = pmmp1, pll
            plm = pmmp1
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    if m > 0:
        return math.sqrt(2.0) * norm * plm * np.cos(m * phi)
    if m < 0:
        return math.sqrt(2.0) * norm * plm * np.sin(am * phi)
    return norm * plm


def displaced_icosphere(level, radius=60.0, center=(0.0, 0.0, -300.0), n_harmonics=8, max_degree=6, max_amp=5.0,
                        seed=0):
    """Icosphere of `radius` displaced radially by a seeded sum of real spherical
    harmonics (degree <= max_degree, amplitudes U(0, max_amp)), baked to world space."""
    rng = np.random.default_rng(seed)
    verts, faces = icosphere(level)
    theta = np.arccos(np.clip(verts[:, 2], -1.0, 1.0))
    phi = np.arctan2(verts[:, 1], verts[:, 0])
    r = np.full(len(verts), float(radius))
    for _ in range(n_harmonics):
        l = int(rng.integers(1, max_degree + 1))
        m = int(rng.integers(-l, l + 1))
        a = float(rng.uniform(0.0, max_amp))
        r += a * _real_sh(l, m, theta, phi)
    world = verts * r[:, None] + np.asarray(center, np.float64)[None, :]
    return world.astype(np.float32), faces.astype(np.int32)


def floor_quad(y=-80.0, x0=-1000.0, x1=1000.0, z0=-1600.0, z1=400.0):
    """Two-triangle quad at height y with face normals +y."""
    v = np.array([[x0, y, z0], [x1, y, z0], [x1, y, z1], [x0, y, z1]], np.float32)
    f = np.array([[0, 2, 1], [0, 3, 2]], np.int32)
    return v, f


def config0_scene(width=256, height=256, spp=20):
    """Plain method, small: sphere mean (0,0,-500) r=70 inside a null sphere r=130,
    renewal_plus, SE kernel sigma 1, length 1, aniso (1,1,1), 3 points/cell,
    camera at the origin along -z, fov 45, constant sky 1.0, max_bounce 10."""
    s = Scene()
    s.width, s.height, s.spp = width, height, spp
    s.max_bounce = 10
    s.max_medium_bounce = 10
    s.gp_mode = _abi.GP_RENEWAL_PLUS
    s.sky = (1.0, 1.0, 1.0)
    m = s.add_medium("sphere", center=(0, 0, -500), radius=70.0, sigma=1.0, length_scale=1.0, aniso=(1, 1, 1),
                     points_per_cell=3)
    s.add_sphere((0, 0, -500), 130.0, bsdf=_abi.BSDF_NULL, int_medium=m)
    return s


def textured_floor_scene(texture, with_texcoords=True, width=24, height=24, spp=2):
    """Configuration 0 plus an emissive Lambertian sphere (a light for
    next-event estimation) and the floor quad under a Lambertian BitmapTexture
    albedo `texture` ((h, w, 3) float RGB, row 0 at the top): at texcoords from
    -0.75 to 3.5, so the lookup wraps, or, without texcoords, at the hit's
    barycentrics. The floor is primitive 2."""
    sc = config0_scene(width, height, spp)
    sc.add_sphere((40.0, 160.0, -380.0), 45.0, emission=(6.0, 5.0, 4.0))
    fv, ff = floor_quad()
    tc = ftc = None
    if with_texcoords:
        tc = np.array([[-0.75, -0.5], [3.5, -0.5], [3.5, 2.25], [-0.75, 2.25]], np.float32)
        ftc = ff.copy()
    fm = sc.add_mesh(Mesh(fv, ff, texcoords=tc, face_texcoords=ftc))
    sc.add_mesh_primitive(fm, texture=texture)
    return sc


def external_gp_grids(res=16, seed=0, center=(0.0, 0.0, -500.0), radius=70.0, half=130.0):
    """Seeded GridMeanFunction samples for an ExternalGPMedium over the cube of
    half-width `half` around `center`: mean = distance to the sphere of
    `radius` plus a smooth seeded ripple of amplitude 6, variance ~ U(0.2, 2).
    Returns (bounds_min, bounds_max, mean, variance), grids (res, res, res)."""
    rng = np.random.default_rng(seed)
    c = np.asarray(center, np.float64)
    bmin, bmax = c - half, c + half
    ax = [bmin[a] + (np.arange(res) + 0.5) * (2 * half / res) for a in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    ph = rng.uniform(0, 2 * np.pi, 3)
    mean = (np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - radius
            + 6.0 * np.sin(X / 23.0 + ph[0]) * np.sin(Y / 19.0 + ph[1]) * np.sin(Z / 29.0 + ph[2]))
    var = rng.uniform(0.2, 2.0, (res, res, res))
    return (tuple(np.float32(bmin).tolist()), tuple(np.float32(bmax).tolist()), mean.astype(np.float32),
            var.astype(np.float32))


def field_scene(kind, width=24, height=24, spp=2, seed=0):
    """Configuration 0's layout (null sphere of radius 130 at (0, 0, -500),
    constant sky 1.0, 10 bounces) seen from (0, 0, -250) along -z, so that
    every pixel enters the null sphere, with a field medium inside it, plus an emissive Lambertian sphere so that
    next-event estimation crosses the medium's transmittance:
    "sdf_sphere": SDFMedium over the sphere mean of radius 70;
    "sdf_mesh": SDFMedium over a displaced icosphere (level 2, radius 60);
    "external_gp": ExternalGPMedium over external_gp_grids(16, seed), noise scale 1;
    "external_gp_mean": the same without the variance grid (no noise)."""
    s = Scene()
    s.width, s.height, s.spp = width, height, spp
    s.max_bounce = 10
    s.max_medium_bounce = 10
    s.gp_mode = _abi.GP_RENEWAL_PLUS
    s.sky = (1.0, 1.0, 1.0)
    s.cam_pos = (0.0, 0.0, -250.0)
    c = (0.0, 0.0, -500.0)
    if kind == "sdf_sphere":
        m = s.add_medium("sphere", center=c, radius=70.0, kind="sdf")
    elif kind == "sdf_mesh":
        v, f = displaced_icosphere(2, radius=60.0, center=c, seed=seed)
        m = s.add_medium("mesh", mesh=s.add_mesh(Mesh(v, f)), kind="sdf")
    elif kind in ("external_gp", "external_gp_mean"):
        bmin, bmax, mean, var = external_gp_grids(16, seed, c)
        m = s.add_external_gp_medium(16, bmin, bmax, mean, var if kind == "external_gp" else None, 1.0)
    else:
        raise ValueError(f"unknown field scene {kind!r}")
    s.add_sphere(c, 130.0, bsdf=_abi.BSDF_NULL, int_medium=m)
    s.add_sphere((40.0, 160.0, -380.0), 45.0, emission=(6.0, 5.0, 4.0))
    return s


def config_mesh_scene(level=6, width=512, height=512, spp=64, seed=0):
    """Mesh mean: displaced icosphere (r 60 at (0,0,-300)) as the GP mean inside a
    null sphere r=100, Lambertian floor quad (albedo 0.7) at y=-80, renewal_plus,
    SE kernel sigma 1, length 2, 3 points/cell."""
    s = Scene()
    s.width, s.height, s.spp = width, height, spp
    s.max_bounce = 10
    s.max_medium_bounce = 10
    s.gp_mode = _abi.GP_RENEWAL_PLUS
    s.sky = (1.0, 1.0, 1.0)
    v, f = displaced_icosphere(level, seed=seed)
    mesh = s.add_mesh(Mesh(v, f))
    m = s.add_medium("mesh", mesh=mesh, sigma=1.0, length_scale=2.0, aniso=(1, 1, 1), points_per_cell=3)
    s.add_sphere((0, 0, -300), 100.0, bsdf=_abi.BSDF_NULL, int_medium=m)
    fv, ff = floor_quad()
    fm = s.add_mesh(Mesh(fv, ff))
    s.add_mesh_primitive(fm, bsdf=_abi.BSDF_LAMBERTIAN, albedo=0.7)
    return s


def batch_scenes(n=64, seed=4):
    """Uneven scene instances for one batched render, seeded: resolution from
    {64^2, 128^2, 256^2, 512^2}, spp in [4, 64], max_bounce in [2, 10],
    length_scale ~ U(0.25, 4), points_per_cell from {1, 3, 8}, a sphere mean of
    radius r ~ U(20, 100) inside a null bounding sphere of radius 1.8 r, and half
    of the instances single_realization, half renewal_plus. Each instance is the
    plain-method scene (camera at the origin along -z, fov 45, constant sky 1)
    with the bounding sphere framed as config0_scene frames its r = 130 sphere."""
    rng = np.random.default_rng(seed)
    modes = rng.permutation([_abi.GP_SINGLE_REALIZATION] * (n // 2) + [_abi.GP_RENEWAL_PLUS] * (n - n // 2))
    out = []
    for i in range(n):
        res = int(rng.choice([64, 128, 256, 512]))
        spp = int(rng.integers(4, 65))
        mb = int(rng.integers(2, 11))
        ls = float(rng.uniform(0.25, 4.0))
        ppc = int(rng.choice([1, 3, 8]))
        r = float(rng.uniform(20.0, 100.0))
        big = 1.8 * r
        z = -500.0 * big / 130.0
        s = Scene()
        s.width = s.height = res
        s.spp = spp
        s.max_bounce = s.max_medium_bounce = mb
        s.gp_mode = int(modes[i])
        s.sky = (1.0, 1.0, 1.0)
        m = s.add_medium("sphere", center=(0, 0, z), radius=r, sigma=1.0, length_scale=ls, aniso=(1, 1, 1),
                         points_per_cell=ppc)
        s.add_sphere((0, 0, z), big, bsdf=_abi.BSDF_NULL, int_medium=m)
        out.append(s)
    return out
