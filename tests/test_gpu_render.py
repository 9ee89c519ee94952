"""The wavefront trace loop against PathTracer::trace (CPU oracle and the
reference's fixtures). The GPU draws the same PCG streams per (x, y, k,
bounce), so most samples replay the reference path exactly; a path diverges
only where the GPU's exp flips the sign of an f within ~1e-6 of zero. Asserted:
per-sample radiance agreement >= 97%, and per-pixel means inside a 3-sigma
Monte Carlo band around the reference's render."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuRenderer, GpuScene

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_trace_fixture_config0(gpu, golden):
    g = golden("trace_c0.npz")
    gs = GpuScene(S.config0_scene(24, 24, 3))
    rad = gs.trace(g["x"], g["y"], g["k"])
    same = np.all(bits(rad) == bits(g["radiance"]), axis=1)
    assert same.mean() >= 0.97, same.mean()
    r = GpuRenderer()
    r.prepare_render(gs)
    fb = r.start_render_progressive(3)
    ok = np.all(bits(fb) == bits(g["framebuffer"]), axis=2)
    assert ok.mean() >= 0.95


def test_trace_fixture_mesh(gpu, golden):
    g = golden("trace_mesh.npz")
    gs = GpuScene(S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5))
    rad = gs.trace(g["x"], g["y"], g["k"])
    same = np.all(bits(rad) == bits(g["radiance"]), axis=1)
    assert same.mean() >= 0.97, same.mean()


def test_trace_fixture_sky_texture(gpu, golden):
    """Escaping paths read the skydrome BitmapTexture (skydrome.cpp,
    texture.cpp); the fixture is the reference's trace on the same image."""
    g = golden("trace_sky.npz")
    sc = S.config0_scene(24, 24, 2)
    sc.sky_texture = g["sky"]
    gs = GpuScene(sc)
    rad = gs.trace(g["x"], g["y"], g["k"])
    same = np.all(bits(rad) == bits(g["radiance"]), axis=1)
    assert same.mean() >= 0.97, same.mean()
    r = GpuRenderer()
    r.prepare_render(gs)
    fb = r.start_render_progressive(2)
    rr = g["radiance"].reshape(24, 24, 2, 3)
    ref = ((rr[:, :, 0] + rr[:, :, 1]).astype(np.float32) * np.float32(0.5)).transpose(1, 0, 2)
    ok = np.all(bits(fb) == bits(ref), axis=2)
    assert ok.mean() >= 0.95, ok.mean()
    gs.set_sky_texture(None)  # back to the scene's constant skydrome
    rad0 = gs.trace(g["x"], g["y"], g["k"])
    plain = GpuScene(S.config0_scene(24, 24, 2)).trace(g["x"], g["y"], g["k"])
    assert np.array_equal(bits(rad0), bits(plain))
    assert not np.array_equal(bits(rad0), bits(rad))


@pytest.mark.parametrize("name", ["a", "b"])
def test_trace_fixture_albedo_texture(gpu, golden, name):
    """Lambertian meshes with a BitmapTexture albedo (bsdf.cpp:14-37,
    mesh.cpp:175-181): at OBJ texcoords with an 8-bit image (a) and at the
    barycentrics with a float image (b); the fixture is the reference's trace."""
    g = golden("trace_tex.npz")
    if name == "a":
        sc = S.textured_floor_scene((g["tex8"].astype(np.float32) / np.float32(255.0)).astype(np.float32), True)
    else:
        sc = S.textured_floor_scene(g["texf"], False)
    gs = GpuScene(sc)
    rad = gs.trace(g["x"], g["y"], g["k"])
    same = np.all(bits(rad) == bits(g["radiance_" + name]), axis=1)
    assert same.mean() >= 0.97, same.mean()
    with pytest.raises(Exception):  # spheres take no albedo texture
        gs.set_albedo_texture(1, g["texf"])
    with pytest.raises(Exception):  # face texcoord index out of range
        gs.set_albedo_texture(2, g["texf"], np.zeros((2, 2), np.float32), np.full((2, 3), 2, np.int32))
    gs.set_albedo_texture(2, None)
    flat = gs.trace(g["x"], g["y"], g["k"])
    assert (np.any(bits(flat) != bits(rad), axis=1)).mean() > 0.2


@pytest.mark.parametrize("mode", ["renewal_plus", "single_realization"])
def test_trace_replay_vs_oracle(gpu, port, mode):
    sc = S.config0_scene(48, 48, 4)
    if mode == "single_realization":
        sc.gp_mode = 0
    gs = GpuScene(sc)
    h = port.scene_create(sc.desc())
    try:
        xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(48), np.arange(48), np.arange(4),
                                                                     indexing="ij"))
        got = gs.trace(xs, ys, ks)
        ref = port.trace(h, xs, ys, ks)
        same = np.all(bits(got) == bits(ref), axis=1)
        assert same.mean() >= 0.97, same.mean()
        assert (ref[:, 0] < 1).sum() > 100  # the GP surface is in view
    finally:
        port.scene_free(h)


def test_render_statistics_and_progressive(gpu, port):
    """Per-pixel 3-sigma band of the GPU's 64-pass render around the oracle's
    64-pass mean, and progressive passes equal one full render."""
    W = H = 24
    spp = 64
    sc = S.config0_scene(W, H, spp)
    gs = GpuScene(sc)
    r = GpuRenderer()
    r.prepare_render(gs)
    full, mom = r.start_render_progressive(spp, moments=True)
    # progressive: 0..16 then 16..64 continues the same running sum
    part = r.start_render_progressive(16)
    assert part is not None
    cont = r.start_render_progressive(spp, spp_begin=16)
    assert np.array_equal(bits(cont), bits(full))
    # moments are the per-pixel FP64 sums of the same samples
    assert np.allclose(mom[:, :, :3] / spp, full, rtol=1e-5, atol=1e-6)
    h = port.scene_create(sc.desc())
    try:
        xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(W), np.arange(H), np.arange(spp),
                                                                     indexing="ij"))
        ref = port.trace(h, xs, ys, ks).reshape(W, H, spp, 3)
    finally:
        port.scene_free(h)
    ref_mean = ref.mean(axis=2).transpose(1, 0, 2)
    var = mom[:, :, 3:] / spp - (mom[:, :, :3] / spp) ** 2
    sigma = np.sqrt(np.maximum(var, 0) / spp + ref.var(axis=2).transpose(1, 0, 2) / spp) + 1e-6
    z = np.abs(full - ref_mean) / sigma
    assert np.mean(z <= 3.0) >= 0.99, np.mean(z <= 3.0)


def test_render_cancel_and_callback(gpu):
    sc = S.config0_scene(16, 16, 8)
    r = GpuRenderer()
    r.prepare_render(sc)
    seen = []
    assert r.start_render_progressive(8, on_spp=seen.append) is not None
    assert seen and seen[-1] == 8
    r.cancel()
    assert r.start_render_progressive(8) is None


def test_release_pools_between_renders(gpu):
    """Scenes released and their cached buffers handed back to the driver: a
    scene created afterwards renders the same image."""
    from mupsi_b200.api import release_pools
    sc = S.config0_scene(32, 32, 2)
    imgs = []
    for _ in range(2):
        gs = GpuScene(sc)
        r = GpuRenderer()
        r.prepare_render(gs)
        imgs.append(r.start_render_progressive(2))
        gs.close()
        release_pools()
    assert np.array_equal(bits(imgs[0]), bits(imgs[1]))
