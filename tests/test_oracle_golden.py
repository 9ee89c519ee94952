"""The CPU oracle (C restatement) against fixtures generated by the reference's
own sources (tests/golden/make_golden.py). Integer outputs and every float the
reference computes are compared bit for bit."""
import numpy as np
import pytest

from oracle import bind
from mupsi_b200 import scene as S


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_make_seed_and_pcg(port, golden):
    g = golden("random.npz")
    for a, s4, s5 in zip(g["seed_args"], g["seed4"], g["seed5"]):
        assert port.make_seed4(*map(int, a[:4])) == s4
        assert port.make_seed5(*map(int, a)) == s5
    for s, u, f in zip(g["rng_seeds"], g["rng_u32"], g["rng_f32"]):
        pu, pf = port.random_stream(int(s), 16)
        assert np.array_equal(pu, u) and np.array_equal(bits(pf), bits(f))
    for s, xy, i in zip(g["cs_seeds"], g["cs_xy"], g["cs_i"]):
        x, y, ii = port.constant_sampler(int(s))
        assert ii == i and np.float32(x) == xy[0] and np.float32(y) == xy[1]


def test_psi_sweep_bit_exact(port, golden):
    g = golden("psi_sweep.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    assert len(keys) == 18
    for key in keys:
        L = float(key.split("_")[0][1:])
        az = float(key.split("_")[1][1:])
        ppc = int(key.split("_")[2][1:])
        k = bind.kernel_struct(1.0, L, (1, 1, az), ppc)
        out = port.psi(k, g[key + "_p"], g[key + "_seed"])
        assert np.array_equal(bits(out), bits(g[key + "_psi"])), key


def test_bvh_build_and_queries(port, golden):
    g = golden("bvh_mesh.npz")
    nodes, idx, root = port.bvh_build(g["verts"], g["faces"])
    assert np.array_equal(nodes, g["nodes"]) and np.array_equal(idx, g["tri_idx"]) and root == g["root"]
    sc = S.Scene()
    mi = sc.add_mesh(S.Mesh(g["verts"], g["faces"]))
    sc.add_medium("mesh", mesh=mi, length_scale=2.0)
    h = port.scene_create(sc.desc())
    try:
        tri, tuv = port.bvh_intersect(h, 0, g["rays"])
        assert np.array_equal(tri, g["hit_tri"]) and np.array_equal(bits(tuv), bits(g["hit_tuv"]))
        assert np.array_equal(port.bvh_occluded(h, 0, g["rays"]), g["occluded"])
        ctri, cdq = port.bvh_closest(h, 0, g["points"])
        assert np.array_equal(ctri, g["closest_tri"]) and np.array_equal(bits(cdq), bits(g["closest_dq"]))
        ins, mtri, mdq = port.mesh_queries(h, 0, g["points"])
        assert np.array_equal(ins, g["inside"]) and np.array_equal(mtri, g["mesh_tri"])
        assert np.array_equal(bits(mdq), bits(g["mesh_dq"]))
        assert np.array_equal(bits(port.mean(h, 0, g["points"])), bits(g["mean"]))
        me = port.medium_eval(h, 0, g["points"], g["seeds"], g["cond"])
        assert np.array_equal(bits(me), bits(g["medium_eval"]))
    finally:
        port.scene_free(h)


def test_sphere_medium_march_and_condition(port, golden):
    g = golden("medium_sphere.npz")
    sc = S.config0_scene(8, 8, 1)
    h = port.scene_create(sc.desc())
    try:
        sd = port.sample_distance(h, 0, g["rays"], g["seeds"], g["cond"])
        assert np.array_equal(bits(sd), bits(g["sample_distance"]))
        hits = np.concatenate([g["sample_distance"][:, :1], g["sample_distance"][:, 2:8]], axis=1)
        c = port.sample_condition(h, 0, hits, g["seeds"])
        assert np.array_equal(bits(c), bits(g["sample_condition"]))
        me = port.medium_eval(h, 0, g["points"], g["seeds"], g["cond"])
        assert np.array_equal(bits(me), bits(g["medium_eval"]))
    finally:
        port.scene_free(h)


def test_trace_config0(port, golden):
    g = golden("trace_c0.npz")
    sc = S.config0_scene(24, 24, 3)
    h = port.scene_create(sc.desc())
    try:
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g["radiance"]))
    finally:
        port.scene_free(h)
    # the framebuffer is the per-pixel pass-ordered sum times 1/spp (framebuffer.cpp:28-35)
    r = g["radiance"].reshape(24, 24, 3, 3)  # x, y, k, rgb
    s = np.zeros((24, 24, 3), np.float32)
    for k in range(3):
        s = (s + r[:, :, k, :]).astype(np.float32)
    fb = (s * np.float32(1.0 / 3)).astype(np.float32).transpose(1, 0, 2)
    assert np.array_equal(bits(fb), bits(g["framebuffer"]))


def test_trace_mesh_scene(port, golden):
    g = golden("trace_mesh.npz")
    sc = S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5)
    h = port.scene_create(sc.desc())
    try:
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g["radiance"]))
    finally:
        port.scene_free(h)


def test_trace_sky_texture(port, golden):
    """Skydrome BitmapTexture lookup (skydrome.cpp, texture.cpp) against the
    reference run on the same image."""
    g = golden("trace_sky.npz")
    sc = S.config0_scene(24, 24, 2)
    h = port.scene_create(sc.desc())
    try:
        port.scene_set_sky(h, g["sky"])
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g["radiance"]))
        assert len(np.unique(rad[:, 0])) > 100
    finally:
        port.scene_free(h)


def test_skydrome_json_round_trip(tmp_path):
    sky = np.random.default_rng(3).uniform(0, 5, (8, 16, 3)).astype(np.float32)
    sc = S.config0_scene(8, 8, 1)
    sc.sky_texture = sky
    p = str(tmp_path / "sky.hdr")
    S.save_sky_raw(p, sky)
    j, _ = sc.to_json(sky_path="sky.hdr")
    back = S.Scene.from_json(j, base_dir=str(tmp_path))
    assert np.array_equal(back.sky_texture, sky)
    sc.sky_texture = None
    j, _ = sc.to_json()
    assert "skydrome" not in j


def textured_scene(g, name):
    """The fixture's scenes: an 8-bit image at OBJ texcoords (a) or a float
    image at the barycentrics (b)."""
    if name == "a":
        return S.textured_floor_scene((g["tex8"].astype(np.float32) / np.float32(255.0)).astype(np.float32), True)
    return S.textured_floor_scene(g["texf"], False)


@pytest.mark.parametrize("name", ["a", "b"])
def test_trace_albedo_texture(port, golden, name):
    """LambertianBsdf(BitmapTexture) on a mesh (bsdf.cpp:14-37, mesh.cpp:175-181,
    texture.cpp:52-69) against the reference run on the same images."""
    g = golden("trace_tex.npz")
    sc = textured_scene(g, name)
    h = port.scene_from(sc)
    try:
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g["radiance_" + name]))
        port.scene_set_albedo(h, 2, None)  # the constant albedo again: a different image
        flat = port.trace(h, g["x"], g["y"], g["k"])
        assert (np.any(bits(flat) != bits(rad), axis=1)).mean() > 0.2
    finally:
        port.scene_free(h)


def test_obj_texcoords_round_trip(tmp_path):
    """load_obj follows Mesh::fetchFrom's vt and face-index rules (mesh.cpp:55-111)."""
    p = tmp_path / "m.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvt 0.25 0.5\nvt 1 0\nvt 0 1\n"
                 "f 1/1 2/2 3/3\nf 2/-2 4 -1/-1\nf 1 2 3 4\n")
    v, f, n, tc, ftc = S.load_obj(str(p), texcoords=True)
    assert f.tolist() == [[0, 1, 2], [1, 3, 3]]
    assert ftc.tolist() == [[0, 1, 2], [1, 0, 2]]  # missing vt -> 0; negative -> count + i
    assert tc.tolist() == [[0.25, 0.5], [1.0, 0.0], [0.0, 1.0]]
    q = tmp_path / "q.obj"
    S.save_obj(str(q), v, f, tc, ftc)
    v2, f2, n2, tc2, ftc2 = S.load_obj(str(q), texcoords=True)
    assert np.array_equal(v2, v) and np.array_equal(f2, f) and np.array_equal(tc2, tc) and np.array_equal(ftc2, ftc)
    S.save_obj(str(q), v, f)
    assert S.load_obj(str(q), texcoords=True)[3:] == (None, None)


def test_texture_json_round_trip(tmp_path):
    sc = S.config0_scene(8, 8, 1)
    fv, ff = S.floor_quad()
    tc = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    fm = sc.add_mesh(S.Mesh(fv, ff, texcoords=tc, face_texcoords=ff.copy()))
    tex8 = np.random.default_rng(1).integers(0, 256, (4, 6, 3), dtype=np.uint8)
    sc.add_mesh_primitive(fm, texture=tex8.astype(np.float32) / np.float32(255.0))
    S.save_image_raw(str(tmp_path / "t.png"), tex8)
    S.save_obj(str(tmp_path / "f.obj"), fv, ff, tc, ff)
    j, extra = sc.to_json(obj_paths=["f.obj"], texture_paths={1: "t.png"})
    assert not extra and j["primitives"][1]["texture"] == "t.png"
    back = S.Scene.from_json(j, base_dir=str(tmp_path))
    p = back.primitives[1]
    assert np.array_equal(p["texture"], sc.primitives[1]["texture"])
    assert np.array_equal(back.meshes[p["mesh"]].texcoords, tc)
    j["primitives"][1]["bsdf"] = "specular"  # the reference reads a texture for Lambertian meshes only
    assert S.Scene.from_json(j, base_dir=str(tmp_path)).primitives[1]["texture"] is None
    with pytest.raises(OSError):  # float pixels only under .hdr / .exr names
        S.save_image_raw(str(tmp_path / "f.png"), tex8.astype(np.float32))
        S.load_texture_image(str(tmp_path / "f.png"))


def test_obj_loader_matches_fetch_from(golden, tmp_path):
    """mupsi_obj_load against Mesh::fetchFrom on the same bytes (long
    decimals, a denormal, -0, relative and missing indices, CR line ends,
    skipped records and faces): identical arrays, bit for bit."""
    g = golden("obj_parse.npz")
    p = tmp_path / "tricky.obj"
    p.write_bytes(bytes(g["text"]))
    v, f, n, t, ft = S.load_obj(str(p), texcoords=True)
    assert np.array_equal(bits(v), bits(g["vertices"]))
    assert np.array_equal(f, g["faces"]) and np.array_equal(ft, g["face_texcoords"])
    assert np.array_equal(bits(n), bits(g["normals"])) and np.array_equal(bits(t), bits(g["texcoords"]))
    with pytest.warns(UserWarning):  # 2 normals for 4 vertices: the reference would read past them
        m = S.Mesh(v, f, n)
    assert m.vertex_normals is None
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(Exception):
        S.load_obj(str(bad))
