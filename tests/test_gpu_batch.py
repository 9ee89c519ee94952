"""Batched multi-instance renders (mupsi_gpu_batch_*): one wave stream over many
scene instances of different sizes, pass counts, bounce limits, GP modes and
impulse densities. Every instance's image must be bit-identical to the
single-scene render of the same scene, whatever the wave packing, schedule,
graph replay or launch shapes, because a path depends only on its scene and
(x, y, k) and psi sums are added in one fixed order for every lane-group size."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuBatch, GpuRenderer, GpuScene, get_tuning, set_tuning
from mupsi_b200.lib import MupsiError

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture
def tuning_restored():
    saved = get_tuning()
    yield
    set_tuning(**saved)


def small_instances():
    sc = S.batch_scenes(n=8, seed=11)
    for i, s in enumerate(sc):
        s.width = s.height = [8, 12, 16, 20][i % 4]
        s.spp = [3, 5, 2, 4, 6, 1, 3, 2][i]
    return sc


def single_renders(scenes):
    out = []
    for s in scenes:
        r = GpuRenderer()
        r.prepare_render(s)
        out.append(r.start_render_progressive(s.spp))
    return out


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("schedule", ["shortest_first", "in_order", "interleaved"])
def test_batch_equals_single_renders(gpu, tuning_restored, graphs, schedule):
    scenes = small_instances()
    ref = single_renders(scenes)
    set_tuning(wave_paths=700)  # several waves, instances split across them
    b = GpuBatch(scenes)
    imgs, done = b.render([s.spp for s in scenes], use_graphs=graphs, schedule=schedule)
    for i, (a, r) in enumerate(zip(imgs, ref)):
        assert np.array_equal(bits(a), bits(r)), f"instance {i}"
    info = b.info()
    assert info["waves"] > 1
    assert info["paths"] == sum(s.width * s.height * s.spp for s in scenes)
    assert info["graph_launches"] == (info["waves"] if graphs else 0)
    assert np.all(done > 0)
    if schedule == "interleaved":  # every instance has passes in the last wave
        assert np.all(done == done.max())
    # a second render replays the captured graphs without new captures
    before = info["graphs_captured"]
    imgs2, _ = b.render([s.spp for s in scenes], use_graphs=graphs, schedule=schedule)
    assert all(np.array_equal(bits(a), bits(c)) for a, c in zip(imgs, imgs2))
    assert b.info()["graphs_captured"] == before
    b.close()


@pytest.mark.parametrize("scene", ["sphere", "mesh"])
def test_results_do_not_depend_on_launch_shape(gpu, tuning_restored, scene):
    # sphere: the fixed psi order; mesh: also the group-parallel closest-point
    # query (lowest triangle index among ties)
    sc = S.config0_scene(20, 20, 3) if scene == "sphere" else S.config_mesh_scene(level=4, width=20, height=20, spp=3)
    gs = GpuScene(sc)
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(20), np.arange(20), np.arange(3),
                                                                 indexing="ij"))
    base = None
    # block_rays: 0 keeps every march on lane groups; >= 1 marches these small
    # queues one ray per block with speculated psi steps (sphere means)
    for mb, mg, sb, br in [(128, 4, 128, 0), (64, 16, 64, 1), (96, 8, 32, 16), (128, 32, 96, 2), (32, 4, 128, 1)]:
        set_tuning(march_block=mb, min_group=mg, shade_block=sb, block_rays=br)
        rad = gs.trace(xs, ys, ks)
        if base is None:
            base = rad
        assert np.array_equal(bits(rad), bits(base)), (mb, mg, sb, br)


def test_lane_rays_render_matches(gpu, tuning_restored):
    """Long sphere-mean queues marched one ray per lane (psi pooled per warp)
    or by lane groups, under several launch shapes: identical images."""
    sc = S.config0_scene(160, 160, 6)
    imgs = []
    for lr, mb, mg, br in ((0, 128, 16, 8), (4, 128, 16, 8), (1, 64, 4, 0), (16, 96, 32, 16), (0, 32, 4, 0)):
        set_tuning(lane_rays=lr, march_block=mb, min_group=mg, block_rays=br)
        r = GpuRenderer()
        g = GpuScene(sc)
        r.prepare_render(g)
        g.profile(True)
        imgs.append(r.start_render_progressive(6))
        st = g.stats(reset=True)
        g.profile(False)
        assert st["iter_medium"][1] > 2 * 148 * 8 * 4  # bounce 1's queue is long enough for one ray per lane
    for im in imgs[1:]:
        assert np.array_equal(bits(imgs[0]), bits(im))
    assert (imgs[0][..., 0] < 1).sum() > 100


def test_lane_rays_mesh_render_matches(gpu, tuning_restored):
    """Mesh means marched one ray per lane (the lazy mean's closest-point
    queries on one lane with the lane-group tie rule, over the four-wide tree;
    with mu_batch > 0 a warp's marches that need the exact mean wait and query
    the BVH together) or by lane groups (binary tree), and a mesh above
    lane_max_tris kept on lane groups: identical images."""
    sc = S.config_mesh_scene(level=5, width=128, height=128, spp=4, seed=2)
    imgs = []
    for lr, lmt, mb in ((0, 1 << 18, 16), (1, 1 << 18, 0), (1, 1 << 18, 16), (4, 1 << 18, 8), (1, 1 << 18, 32),
                        (1, 0, 16)):
        set_tuning(lane_rays=lr, lane_max_tris=lmt, mu_batch=mb)
        r = GpuRenderer()
        g = GpuScene(sc)
        r.prepare_render(g)
        g.profile(True)
        imgs.append(r.start_render_progressive(4))
        st = g.stats(reset=True)
        g.profile(False)
        assert st["iter_medium"][1] > 2 * 148 * 16 * 4 and st["mean_evals"] > 0
    for im in imgs[1:]:
        assert np.array_equal(bits(imgs[0]), bits(im))
    assert (imgs[0][..., 0] < 0.9).sum() > 500


def test_block_rays_render_matches(gpu, tuning_restored):
    """A full 96x96x6 configuration-0 render with the block-per-ray march for
    every short queue (block_rays 16) and for none (0): identical images."""
    sc = S.config0_scene(96, 96, 6)
    imgs = []
    for br in (0, 16, 1):
        set_tuning(block_rays=br)
        r = GpuRenderer()
        r.prepare_render(GpuScene(sc))
        imgs.append(r.start_render_progressive(6))
    assert np.array_equal(bits(imgs[0]), bits(imgs[1])) and np.array_equal(bits(imgs[0]), bits(imgs[2]))
    assert (imgs[0][..., 0] < 1).sum() > 100


def test_batch_completion_order_and_device_output(gpu, tuning_restored):
    import torch
    scenes = small_instances()
    set_tuning(wave_paths=600)
    b = GpuBatch(scenes)
    spp = [s.spp for s in scenes]
    host, done = b.render(spp, schedule="shortest_first")
    work = np.array([s.width * s.height * s.spp for s in scenes])
    order = np.argsort(work, kind="stable")
    assert np.all(np.diff(done[order]) >= 0)  # shortest first: completion in work order
    dev = [torch.empty((s.height, s.width, 3), dtype=torch.float32, device="cuda") for s in scenes]
    got, _ = b.render(spp, out=dev)
    torch.cuda.synchronize()
    for h, d in zip(host, got):
        assert np.array_equal(bits(h), bits(d.cpu().numpy()))


def test_batch_zero_spp_and_errors(gpu):
    scenes = small_instances()[:3]
    scenes[1].spp = 2
    ref = single_renders([scenes[1]])[0]
    b = GpuBatch(scenes)
    imgs, done = b.render([0, 2, 0])
    assert done[0] == 0 and done[2] == 0 and done[1] > 0
    assert np.array_equal(bits(imgs[1]), bits(ref))
    with pytest.raises(MupsiError):
        b.render([1, -1, 1])
    with pytest.raises(ValueError):
        b.render([1, 1])
    b.cancel()
    assert b.render([1, 1, 1]) is None
    with pytest.raises(MupsiError):
        set_tuning(min_group=3)
    with pytest.raises(MupsiError):
        set_tuning(min_group=2)
    with pytest.raises(MupsiError):
        set_tuning(march_block=256)
    with pytest.raises(MupsiError):
        set_tuning(block_rays=257)
    with pytest.raises(MupsiError):
        set_tuning(mu_batch=33)
