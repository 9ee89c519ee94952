"""SDF and external GP media on the GPU (k_march_field, the shade kernel's
transmittance, the single-op entries) against fixtures made by the reference's
own SDFMedium / ExternalGPMedium / GridMeanFunction, and full traces of scenes
loaded through Controller::load's sdf_medium / external_gp_medium keys.
Per-ray and per-point results carry no transcendental the GPU rounds
differently, so they are bit-exact; traces replay >= 97% of samples exactly
(the light and BSDF samplers' sin/cos/exp are the GPU's own)."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuBatch, GpuRenderer, GpuScene
from mupsi_b200.lib import MupsiError

pytestmark = pytest.mark.gpu
KINDS = ["sdf_sphere", "sdf_mesh", "external_gp", "external_gp_mean"]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kind", KINDS)
def test_field_medium_per_ray(gpu, golden, kind):
    g = golden("field_media.npz")
    gs = GpuScene(S.field_scene(kind))
    rays, seed = g[kind + "_rays"], g[kind + "_seed"]
    sd = gs.sample_distance(0, rays, seed)
    assert np.array_equal(bits(sd), bits(g[kind + "_sd"]))
    assert np.array_equal(bits(gs.transmittance(0, rays, seed)), bits(g[kind + "_tr"]))
    assert np.array_equal(bits(gs.eval_with_gradient(0, g[kind + "_p"], g[kind + "_pseed"])), bits(g[kind + "_eval"]))
    if kind.startswith("external"):
        assert np.array_equal(bits(gs.mean(0, g[kind + "_p"])), bits(g[kind + "_grid"]))


@pytest.mark.parametrize("kind", KINDS)
def test_field_trace(gpu, golden, kind):
    g = golden("trace_field.npz")
    gs = GpuScene(S.field_scene(kind))
    rad = gs.trace(g["x"], g["y"], g["k"])
    same = np.all(bits(rad) == bits(g[kind]), axis=1)
    assert same.mean() >= 0.97, same.mean()
    r = GpuRenderer()
    r.prepare_render(gs)
    fb = r.start_render_progressive(2)
    rr = g[kind].reshape(24, 24, 2, 3)
    ref = ((rr[:, :, 0] + rr[:, :, 1]).astype(np.float32) * np.float32(0.5)).transpose(1, 0, 2)
    assert np.all(bits(fb) == bits(ref), axis=2).mean() >= 0.95


def test_field_batch_and_noalloc(gpu):
    """A batch mixing field and GP scenes (one with a light, whose shadow rays
    through the GP medium are marched by the shadow passes) renders each as
    alone; the allocation-free trace runs the field march too."""
    import torch
    tex = np.random.default_rng(2).uniform(0.1, 0.9, (8, 8, 3)).astype(np.float32)
    scenes = [S.field_scene("sdf_mesh", 32, 32, 3), S.config0_scene(32, 32, 3), S.field_scene("external_gp", 32, 32, 3),
              S.textured_floor_scene(tex, True, 32, 32, 3)]
    alone = []
    for sc in scenes:
        r = GpuRenderer()
        r.prepare_render(GpuScene(sc))
        alone.append(r.start_render_progressive(3))
    for graphs in (True, False):
        imgs, _ = GpuBatch(scenes).render([3, 3, 3, 3], use_graphs=graphs)
        for a, b in zip(imgs, alone):
            assert np.array_equal(bits(a), bits(b))
    gs = GpuScene(S.field_scene("external_gp", 32, 32, 2))
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(32), np.arange(32), np.arange(2),
                                                                 indexing="ij"))
    ref = gs.trace(xs, ys, ks)
    out = torch.full((len(xs), 3), -1.0, dtype=torch.float32, device="cuda")
    gs.trace_noalloc(*(torch.from_numpy(a).cuda() for a in (xs, ys, ks)), out)
    torch.cuda.synchronize()
    assert np.array_equal(bits(out.cpu().numpy()), bits(ref))


def test_field_medium_rejects_gp_only_calls(gpu):
    gs = GpuScene(S.field_scene("sdf_sphere"))
    smp = np.zeros((4, 7), np.float32)
    with pytest.raises(MupsiError):  # only a GPMedium conditions
        gs.sample_condition(0, smp, np.zeros(4, np.uint32))
    with pytest.raises(MupsiError):
        gs.set_mean_eval(0, "every_step")
    with pytest.raises(MupsiError):
        gs.set_external_gp_medium(0, 1, (0, 0, 0), (1, 1, 1), np.zeros(1, np.float32))
    with pytest.raises(MupsiError):  # empty bounds
        gs.set_external_gp_medium(0, 2, (0, 0, 0), (1, 0, 1), np.zeros(8, np.float32))
