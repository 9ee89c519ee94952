"""The CPU oracle (C restatement) against fixtures generated by the reference's
own sources (tests/golden/make_golden.py). Integer outputs and every float the
reference computes are compared bit for bit."""
import numpy as np

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
