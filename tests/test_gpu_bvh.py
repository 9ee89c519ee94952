"""BVH intersect / occluded / closest and Mesh inside / distToPoint on the GPU:
bit-exact against the CPU oracle and the reference's fixtures."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import DeviceMesh, GpuScene

pytestmark = pytest.mark.gpu
FMAX = np.finfo(np.float32).max


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _rays(rng, n, center=(0, 0, -300), spread=40.0):
    o = (rng.uniform(-400, 400, (n, 3)) + np.array([0, 0, -300])).astype(np.float32)
    tgt = (rng.normal(size=(n, 3)) * spread + np.array(center)).astype(np.float32)
    d = (tgt - o).astype(np.float32)
    d[n // 2:] = rng.normal(size=(n - n // 2, 3)).astype(np.float32)
    d[::11, 0] = 0.0  # axis-parallel slabs
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 3:6], r[:, 7] = o, d, FMAX
    r[::5, 6] = rng.uniform(0, 300, len(r[::5]))
    return r


def test_bvh_fixture(gpu, golden):
    g = golden("bvh_mesh.npz")
    m = DeviceMesh(g["verts"], g["faces"])
    tri, tuv = m.intersect(g["rays"])
    assert np.array_equal(tri, g["hit_tri"]) and np.array_equal(bits(tuv), bits(g["hit_tuv"]))
    assert np.array_equal(m.occluded(g["rays"]), g["occluded"])
    ctri, cdq = m.closest(g["points"])
    assert np.array_equal(ctri, g["closest_tri"]) and np.array_equal(bits(cdq), bits(g["closest_dq"]))
    ins, mtri, mdq = m.queries(g["points"])
    assert np.array_equal(ins, g["inside"]) and np.array_equal(mtri, g["mesh_tri"])
    assert np.array_equal(bits(mdq), bits(g["mesh_dq"]))


@pytest.mark.parametrize("level,position,scale", [(4, (0, 0, 0), 1.0), (5, (0, 0, 0), 1.0), (3, (5, -2, 30), 1.5)])
def test_bvh_against_oracle(gpu, port, level, position, scale):
    rng = np.random.default_rng(level)
    v, f = S.displaced_icosphere(level, seed=level)
    m = DeviceMesh(v, f, position=position, scale=scale)
    sc = S.Scene()
    mi = sc.add_mesh(S.Mesh(v, f, position=position, scale=scale))
    sc.add_medium("mesh", mesh=mi)
    h = port.scene_create(sc.desc())
    try:
        rays = _rays(rng, 20000)
        tri, tuv = m.intersect(rays)
        otri, otuv = port.bvh_intersect(h, 0, rays)
        assert np.array_equal(tri, otri) and np.array_equal(bits(tuv), bits(otuv))
        assert (tri != 0xFFFFFFFF).sum() > 1000
        assert np.array_equal(m.occluded(rays), port.bvh_occluded(h, 0, rays))
        q = (rng.uniform(-120, 120, (20000, 3)) + np.array([0, 0, -300])).astype(np.float32)
        ctri, cdq = m.closest(q)
        octri, ocdq = port.bvh_closest(h, 0, q)
        assert np.array_equal(ctri, octri) and np.array_equal(bits(cdq), bits(ocdq))
        ins, mtri, mdq = m.queries(q)
        oins, omtri, omdq = port.mesh_queries(h, 0, q)
        assert np.array_equal(ins, oins) and np.array_equal(mtri, omtri) and np.array_equal(bits(mdq), bits(omdq))
        assert 0 < ins.sum() < len(ins)
    finally:
        port.scene_free(h)


def test_bvh_edge_cases(gpu, port):
    # a single triangle (one leaf, root 0), a degenerate triangle, and rays along faces
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 2, 2], [2, 2, 2], [3, 3, 3]], np.float32)
    f = np.array([[0, 1, 2], [3, 4, 5]], np.int32)
    m = DeviceMesh(v, f)
    rays = np.array([[0.2, 0.2, 1, 0, 0, -1, 0, FMAX], [0.2, 0.2, 1, 0, 0, 1, 0, FMAX],
                     [-1, 0, 0, 1, 0, 0, 0, FMAX], [0.5, 0.5, -1, 0, 0, 1, 0, FMAX]], np.float32)
    sc = S.Scene()
    sc.add_mesh(S.Mesh(v, f))
    h = port.scene_create(sc.desc())
    try:
        tri, tuv = m.intersect(rays)
        otri, otuv = port.bvh_intersect(h, 0, rays)
        assert np.array_equal(tri, otri) and np.array_equal(bits(tuv), bits(otuv))
        assert tri[0] == 0 and tri[1] == 0xFFFFFFFF
        q = np.array([[2, 2, 2], [0.1, 0.1, 0.0], [5, 5, 5]], np.float32)
        assert np.array_equal(bits(m.closest(q)[1]), bits(port.bvh_closest(h, 0, q)[1]))
    finally:
        port.scene_free(h)



def test_occlusion_from_root_matches_intersect(gpu):
    """MUPSI_OCCLUSION_ROOT: occluded() answers exactly as an intersect within
    [near_t, far_t]; the reference's start at node 0 (the default) misses
    occluders outside the first leaf."""
    rng = np.random.default_rng(9)
    v, f = S.displaced_icosphere(4, seed=4)
    m = DeviceMesh(v, f)
    rays = _rays(rng, 20000)
    tri, _ = m.intersect(rays)
    hit = tri != 0xFFFFFFFF
    reference = m.occluded(rays).astype(bool)
    m.set_occlusion(True)
    root = m.occluded(rays).astype(bool)
    assert np.array_equal(root, hit)
    assert (reference != root).sum() > 100
    m.set_occlusion(False)
    assert np.array_equal(m.occluded(rays).astype(bool), reference)


def test_bvh_work_counting_changes_nothing(gpu):
    """Profiling mode 2 runs counted copies of the BVH traversals (nodes loaded,
    triangles tested, for the bench's algorithmic BVH bytes): the image is the
    same bit for bit and the counts are those of real traversals."""
    from mupsi_b200.api import GpuRenderer
    sc = S.config_mesh_scene(level=4, width=32, height=32, spp=2, seed=3)
    g = GpuScene(sc)
    r = GpuRenderer()
    r.prepare_render(g)
    plain = r.start_render_progressive(2)
    g.profile(True, bvh=True)
    g.stats(reset=True)
    counted = r.start_render_progressive(2)
    st = g.stats(reset=True)
    g.profile(True)
    again = r.start_render_progressive(2)
    st1 = g.stats(reset=True)
    g.profile(False)
    assert np.array_equal(plain.view(np.uint32), counted.view(np.uint32))
    assert np.array_equal(plain.view(np.uint32), again.view(np.uint32))
    assert st["bvh_nodes"] > 0 and st["bvh_tris"] > 0 and st["mean_evals"] > 0
    assert st1["bvh_nodes"] == 0 and st1["bvh_tris"] == 0  # mode 1 does not count BVH work
    # every query loads at least its root node
    assert st["bvh_nodes"] >= st["mean_evals"]
