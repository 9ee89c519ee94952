"""Generate the golden fixtures from the reference's own sources.

Runs the reference compiled from source (oracle/_ref/libmupsi_ref_parity.so,
built by `make -C oracle ref` from the reference tree) on seeded synthetic
inputs and stores inputs and outputs as .npz files next to this script. The
reference ships no tests or golden vectors, so these fixtures are what pins
the CPU oracle (oracle/libmupsi_oracle.so) in the CPU-only test suite.

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py trace_sky  # one of them
"""
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)
from oracle import bind  # noqa: E402
from mupsi_b200 import scene as S  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
FMAX = np.finfo(np.float32).max


def psi_sweep(R, rng):
    """ConfigGP-noise sweep points: L in {0.5,1,4} x aniso {(1,1,1),(1,1,4)} x ppc {1,3,8}."""
    out = {}
    n = 96
    for L in (0.5, 1.0, 4.0):
        for an in ((1, 1, 1), (1, 1, 4)):
            for ppc in (1, 3, 8):
                k = bind.kernel_struct(1.0, L, an, ppc)
                p = rng.uniform(-150, 150, (n, 3)).astype(np.float32)
                # include negative coordinates near cell boundaries (trunc vs floor)
                p[:8] = (np.round(p[:8] / L) * L).astype(np.float32)
                p[8:16] = -np.abs(p[8:16]) * 1e-3
                s = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
                key = f"L{L}_a{an[2]}_p{ppc}"
                out[key + "_p"] = p
                out[key + "_seed"] = s
                out[key + "_psi"] = R.psi(k, p, s)
    return out


def trace_sky(R, td):
    """Skydrome with a BitmapTexture: configuration 0 at 24x24, 2 passes, the
    sky a seeded 64x32 float image the reference loads through its
    BitmapTexture (the oracle's OpenCV stand-in reads the raw format)."""
    sc = S.config0_scene(24, 24, 2)
    sky = np.random.default_rng(11).uniform(0.2, 3.0, (32, 64, 3)).astype(np.float32)
    sc.sky_texture = sky
    skyp = os.path.join(td, "sky.hdr")
    S.save_sky_raw(skyp, sky)
    j, _ = sc.to_json(sky_path=skyp)
    jp = os.path.join(td, "sky.json")
    json.dump(j, open(jp, "w"))
    rh = R.scene_load(jp, sky=None)
    xs, ys, ks = np.meshgrid(np.arange(24), np.arange(24), np.arange(2), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    rad = R.trace(rh, xs, ys, ks)
    # the texture was loaded (a failed load shows magenta (1, 0, 1))
    assert len(np.unique(rad[:, 0])) > 100 and not np.all(rad[:, 1] == 0)
    np.savez_compressed(os.path.join(OUT, "trace_sky.npz"), x=xs, y=ys, k=ks, radiance=rad, sky=sky)


def trace_tex(R, td):
    """Lambertian meshes with a BitmapTexture albedo: an 8-bit 16x12 image at
    OBJ texcoords (scene a) and a float 8x8 image at the barycentrics (scene b,
    an OBJ without vt lines)."""
    rng = np.random.default_rng(12)
    tex8 = rng.integers(0, 256, (12, 16, 3), dtype=np.uint8)
    texf = rng.uniform(0.05, 0.95, (8, 8, 3)).astype(np.float32)
    xs, ys, ks = np.meshgrid(np.arange(24), np.arange(24), np.arange(2), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    out = dict(x=xs, y=ys, k=ks, tex8=tex8, texf=texf)
    for name, with_tc, tex, tname in (("a", True, tex8, "albedo.png"), ("b", False, texf, "albedo.hdr")):
        tp = os.path.join(td, name + tname)
        S.save_image_raw(tp, tex)
        sc = S.textured_floor_scene(S.load_texture_image(tp), with_tc)
        m = sc.meshes[-1]
        obj = os.path.join(td, name + "floor.obj")
        S.save_obj(obj, m.vertices, m.faces, m.texcoords, m.face_texcoords)
        j, extra = sc.to_json(obj_paths=[obj], texture_paths={2: tp})
        assert not extra
        jp = os.path.join(td, name + "tex.json")
        json.dump(j, open(jp, "w"))
        rh = R.scene_load(jp, sky=1.0)
        rad = R.trace(rh, xs, ys, ks)
        # the texture was loaded (a failed load shows magenta (1, 0, 1))
        assert len(np.unique(rad[:, 0])) > 100
        out["radiance_" + name] = rad
    np.savez_compressed(os.path.join(OUT, "trace_tex.npz"), **out)


FIELD_KINDS = ("sdf_sphere", "sdf_mesh", "external_gp", "external_gp_mean")


def _field_files(sc, td, name):
    """Write what the reference loads for a field scene: the SDF mesh as OBJ,
    the external GP grids as raw float32. Returns (obj_paths, grid_paths, ref medium kwargs)."""
    m = sc.media[0]
    obj_paths, grid_paths = [], None
    for i, mesh in enumerate(sc.meshes):
        op = os.path.join(td, f"{name}_{i}.obj")
        S.save_obj(op, mesh.vertices, mesh.faces)
        obj_paths.append(op)
    if m["kind"] == "external_gp":
        mp = f"{name}_mean.bin"
        m["mean_grid"].tofile(os.path.join(td, mp))
        vp = None
        if m["var_grid"] is not None:
            vp = f"{name}_var.bin"
            m["var_grid"].tofile(os.path.join(td, vp))
        grid_paths = (mp, vp)
    return obj_paths, grid_paths


def _field_rays(rng, n_out=256, n_in=64):
    """Rays from the camera towards the medium (jittered), rays starting inside
    the null sphere in random directions, and shadow-ray-like finite ones."""
    d = np.stack([rng.normal(0, 0.12, n_out), rng.normal(0, 0.12, n_out), -np.ones(n_out)], 1)
    o = np.zeros((n_out, 3))
    o2 = np.float64([0, 0, -500]) + rng.uniform(-100, 100, (n_in, 3))
    d2 = rng.normal(0, 1, (n_in, 3))
    o = np.concatenate([o, o2])
    d = np.concatenate([d, d2])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3:6] = d
    rays[:, 6] = 1e-3
    rays[:, 7] = 3e38
    rays[n_out + n_in // 2:, 7] = rng.uniform(20, 200, n_in - n_in // 2)  # finite farT
    return rays


def field_media(R, td):
    """SDFMedium / ExternalGPMedium / GridMeanFunction per point and per ray,
    from the reference's own classes (ref_field_* in oracle/ref_harness.cpp)."""
    rng = np.random.default_rng(21)
    out = {}
    for kind in FIELD_KINDS:
        sc = S.field_scene(kind)
        obj_paths, grid_paths = _field_files(sc, td, kind)
        m = sc.media[0]
        if kind == "sdf_sphere":
            h = R.sdf_create(0, center=m["center"], radius=m["radius"])
        elif kind == "sdf_mesh":
            h = R.sdf_create(1, obj_path=obj_paths[0])
        else:
            h = R.external_gp_create(m["res"], m["bmin"], m["bmax"], os.path.join(td, grid_paths[0]),
                                     os.path.join(td, grid_paths[1]) if grid_paths[1] else None, m["noise_scale"])
        rays = _field_rays(rng)
        seed = rng.integers(0, 2 ** 32, len(rays), dtype=np.uint64).astype(np.uint32)
        p = (np.float32([0, 0, -500]) + rng.uniform(-140, 140, (256, 3))).astype(np.float32)
        pseed = rng.integers(0, 2 ** 32, len(p), dtype=np.uint64).astype(np.uint32)
        sd = R.field_sample_distance(h, rays, seed)
        assert 0.2 < (sd[:, 0] == 0).mean() < 0.9, kind
        out[kind + "_rays"] = rays
        out[kind + "_seed"] = seed
        out[kind + "_sd"] = sd
        out[kind + "_tr"] = R.field_transmittance(h, rays, seed)
        out[kind + "_p"] = p
        out[kind + "_pseed"] = pseed
        out[kind + "_eval"] = R.field_eval(h, p, pseed)
        if kind.startswith("external"):
            out[kind + "_grid"] = R.grid_eval(os.path.join(td, grid_paths[0]), m["res"], m["bmin"], m["bmax"], p)
        R.field_free(h)
    np.savez_compressed(os.path.join(OUT, "field_media.npz"), **out)


def trace_field(R, td):
    """Full traces of the field scenes through Controller::load's sdf_medium /
    external_gp_medium keys: 24x24, 2 passes."""
    xs, ys, ks = np.meshgrid(np.arange(24), np.arange(24), np.arange(2), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    out = dict(x=xs, y=ys, k=ks)
    for kind in FIELD_KINDS:
        sc = S.field_scene(kind)
        obj_paths, grid_paths = _field_files(sc, td, kind)
        j, extra = sc.to_json(obj_paths=obj_paths, grid_paths=grid_paths)
        assert not extra
        jp = os.path.join(td, kind + ".json")
        json.dump(j, open(jp, "w"))
        rh = R.scene_load(jp, sky=1.0)
        rad = R.trace(rh, xs, ys, ks)
        R.scene_free(rh)
        assert len(np.unique(rad[:, 0])) > 50, kind
        out[kind] = rad
    np.savez_compressed(os.path.join(OUT, "trace_field.npz"), **out)


def trace_skip(R, td):
    """PathTracerSettings::skip_medium (trace.cpp:142) on the 16x16 mesh scene:
    the reference renders with the global set, as Controller::startProgressive
    (targetSpp, true) leaves it."""
    sc = S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5)
    objs = []
    for i, m in enumerate(sc.meshes):
        p = os.path.join(td, f"skip{i}.obj")
        S.save_obj(p, m.vertices, m.faces)
        objs.append(p)
    j, extra = sc.to_json(objs)
    jp = os.path.join(td, "skip.json")
    json.dump(j, open(jp, "w"))
    R.set_skip_medium(True)
    try:
        rh = R.scene_load(jp, sky=1.0, extra_meshes=extra)
    finally:
        R.set_skip_medium(False)
    xs, ys, ks = np.meshgrid(np.arange(16), np.arange(16), np.arange(2), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    rad = R.trace(rh, xs, ys, ks)
    R.scene_free(rh)
    np.savez_compressed(os.path.join(OUT, "trace_skip.npz"), x=xs, y=ys, k=ks, radiance=rad)


OBJ_TEXT = """# tricky numbers and records for Mesh::fetchFrom
v 0.1 0.2 0.3
v 1.00000005960464477539 -2.5e-3 3.4028235e38
v 1e-45 -0 123456789.123456789
v .5 -.25 7
vn 0 0 1
vn 0.577350269 0.577350269 0.577350269
vt 0.333333343267 0.666666686535 0.9
vt -1.5 2.5
vt 0.1 0.7
o object
g group
s 1
usemtl m
f 1/1/1 2/2/2 3/3/1
f 2//1 3//2 4//1
f -1/-1 -2/-2 -3/-3
f 1 2 3 4
f 1 2
f 4/3 1 2/1\r
"""


def obj_parse(R, td):
    """Mesh::fetchFrom on an OBJ with long decimals, exponents, relative and
    missing indices, CR line ends and skipped records and faces."""
    p = os.path.join(td, "tricky.obj")
    with open(p, "w", newline="") as fh:
        fh.write(OBJ_TEXT.replace("\\r", "\r"))
    v, f, n, t, ft = R.obj_load(p)
    np.savez_compressed(os.path.join(OUT, "obj_parse.npz"), text=np.frombuffer(open(p, "rb").read(), np.uint8),
                        vertices=v, faces=f, normals=n, texcoords=t, face_texcoords=ft)


def main():
    if len(sys.argv) > 1:
        with tempfile.TemporaryDirectory() as td:
            for name in sys.argv[1:]:
                globals()[name](bind.RefOracle("ref"), td)
        print("fixtures written to", OUT)
        return
    R = bind.RefOracle("ref")
    rng = np.random.default_rng(20261203)
    data = {}
    # math/random.h: make_seed, Random stream, ConstantSampler
    args = rng.integers(-2**31, 2**31, (64, 5)).astype(np.int64)
    data["seed_args"] = args
    data["seed4"] = np.array([R.make_seed4(*map(int, a[:4])) for a in args], np.uint32)
    data["seed5"] = np.array([R.make_seed5(*map(int, a)) for a in args], np.uint32)
    seeds = np.array([0, 1, 42, 2**32 - 1, 123456789], np.uint64)
    data["rng_seeds"] = seeds
    data["rng_u32"] = np.stack([R.random_stream(int(s), 16)[0] for s in seeds])
    data["rng_f32"] = np.stack([R.random_stream(int(s), 16)[1] for s in seeds])
    data["cs_seeds"] = seeds.astype(np.uint32)
    cs = [R.constant_sampler(int(s) & 0xFFFFFFFF) for s in seeds]
    data["cs_xy"] = np.array([[c[0], c[1]] for c in cs], np.float32)
    data["cs_i"] = np.array([c[2] for c in cs], np.uint32)
    np.savez_compressed(os.path.join(OUT, "random.npz"), **data)

    np.savez_compressed(os.path.join(OUT, "psi_sweep.npz"), **psi_sweep(R, rng))

    # BVH on a displaced icosphere (level 3, 1280 faces)
    v, f = S.displaced_icosphere(3, seed=7)
    h, nodes, idx, root = R.bvh_build(v, f)
    n = 512
    o = rng.uniform(-400, 400, (n, 3)).astype(np.float32)
    o[:, 2] -= 300
    tgt = (rng.normal(size=(n, 3)) * 40 + np.array([0, 0, -300])).astype(np.float32)
    d = (tgt - o).astype(np.float32)
    d[n // 2:] = rng.normal(size=(n - n // 2, 3)).astype(np.float32)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3], rays[:, 3:6], rays[:, 7] = o, d, FMAX
    rays[::7, 6] = 50.0  # some nonzero nearT
    tri, tuv = R.bvh_intersect(h, rays)
    occ = R.bvh_occluded(h, rays)
    q = (rng.uniform(-120, 120, (n, 3)) + np.array([0, 0, -300])).astype(np.float32)
    ctri, cdq = R.bvh_closest(h, q)
    td = tempfile.mkdtemp()
    obj = os.path.join(td, "mesh.obj")
    S.save_obj(obj, v, f)
    kmesh = bind.kernel_struct(1.0, 2.0, (1, 1, 1), 3)
    mh = R.medium_create(1, kmesh, obj_path=obj)
    ins, mtri, mdq = R.mesh_queries(mh, q)
    mean = R.mean(mh, q)
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    cond = np.zeros((n, 8), np.float32)
    cond[:, :3] = q + rng.normal(size=(n, 3)).astype(np.float32)
    cond[:, 3] = rng.normal(size=n)
    cond[:, 4:7] = rng.normal(size=(n, 3))
    cond[::2, 7] = 1
    meval = R.medium_eval(mh, q, seeds, cond)
    np.savez_compressed(os.path.join(OUT, "bvh_mesh.npz"), verts=v, faces=f, nodes=nodes, tri_idx=idx,
                        root=np.uint32(root), rays=rays, hit_tri=tri, hit_tuv=tuv, occluded=occ, points=q,
                        closest_tri=ctri, closest_dq=cdq, inside=ins, mesh_tri=mtri, mesh_dq=mdq, mean=mean,
                        seeds=seeds, cond=cond, medium_eval=meval)

    # sphere-mean medium: march and conditioning (config 0 kernel)
    k1 = bind.kernel_struct(1.0, 1.0, (1, 1, 1), 3)
    sh = R.medium_create(0, k1, center=(0, 0, -500), radius=70.0)
    m = 128
    o = (rng.uniform(-60, 60, (m, 3)) + np.array([0, 0, -380])).astype(np.float32)
    tgt = (np.array([0, 0, -500]) + rng.normal(size=(m, 3)) * 30).astype(np.float32)
    d = (tgt - o).astype(np.float32)
    d[m // 2:] = rng.normal(size=(m - m // 2, 3)).astype(np.float32)
    rays = np.zeros((m, 8), np.float32)
    rays[:, :3], rays[:, 3:6], rays[:, 6], rays[:, 7] = o, d, np.float32(1.5e-3), FMAX
    mseeds = rng.integers(0, 2**32, m, dtype=np.uint64).astype(np.uint32)
    mcond = np.zeros((m, 8), np.float32)
    mcond[:, :3] = o + rng.normal(size=(m, 3)).astype(np.float32) * 2
    mcond[:, 3] = rng.normal(size=m)
    mcond[:, 4:7] = rng.normal(size=(m, 3))
    mcond[m // 2:, 7] = 1
    sd = R.sample_distance(sh, rays, mseeds, mcond)
    hits = np.concatenate([sd[:, :1], sd[:, 2:8]], axis=1)
    sc = R.sample_condition(sh, hits, mseeds, True)
    sp = (rng.uniform(-100, 100, (m, 3)) + np.array([0, 0, -500])).astype(np.float32)
    seval = R.medium_eval(sh, sp, mseeds, mcond)
    np.savez_compressed(os.path.join(OUT, "medium_sphere.npz"), rays=rays, seeds=mseeds, cond=mcond,
                        sample_distance=sd, sample_condition=sc, points=sp, medium_eval=seval)

    # full trace loop: configuration-0 scene at 24x24, passes 0..2
    sc0 = S.config0_scene(24, 24, 3)
    j, _ = sc0.to_json()
    jp = os.path.join(td, "c0.json")
    json.dump(j, open(jp, "w"))
    rh = R.scene_load(jp, sky=1.0)
    xs, ys, ks = np.meshgrid(np.arange(24), np.arange(24), np.arange(3), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    rad = R.trace(rh, xs, ys, ks)
    fb = R.render(rh, 3)
    np.savez_compressed(os.path.join(OUT, "trace_c0.npz"), x=xs, y=ys, k=ks, radiance=rad, framebuffer=fb)

    # mesh-mean scene with a Lambertian floor: level-2 mesh at 16x16, 2 passes
    scm = S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5)
    objs = []
    for i, mm in enumerate(scm.meshes):
        pth = os.path.join(td, f"m{i}.obj")
        S.save_obj(pth, mm.vertices, mm.faces)
        objs.append(pth)
    j, extra = scm.to_json(objs)
    jp = os.path.join(td, "cm.json")
    json.dump(j, open(jp, "w"))
    rh = R.scene_load(jp, sky=1.0, extra_meshes=extra)
    xs, ys, ks = np.meshgrid(np.arange(16), np.arange(16), np.arange(2), indexing="ij")
    xs, ys, ks = xs.ravel().astype(np.int32), ys.ravel().astype(np.int32), ks.ravel().astype(np.int32)
    rad = R.trace(rh, xs, ys, ks)
    np.savez_compressed(os.path.join(OUT, "trace_mesh.npz"), x=xs, y=ys, k=ks, radiance=rad)
    trace_sky(R, td)
    trace_tex(R, td)
    field_media(R, td)
    trace_field(R, td)
    trace_skip(R, td)
    obj_parse(R, td)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
