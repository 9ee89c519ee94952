"""Images in expectation at the configurations' own sizes.

The GPU renders through the public render entry (mupsi_gpu_render:
Renderer::startRenderProgressive, rendering/renderer.cpp:22-49, with
Framebuffer::accumulate, framebuffer.cpp:28-35); the CPU oracle traces
PathTracer::trace (rendering/trace.cpp:118-213) on a seeded random subset of
the pixels. The two sides draw DIFFERENT passes (the GPU passes 0..spp-1, the
oracle passes spp..2spp-1), so their samples are independent draws of the same
per-pixel distribution, and a per-pixel 3-sigma band is a real test of equality
in expectation (same-pass draws replay the same paths and would agree
trivially).

Bars (stated here):
  * configuration 0 (256x256, 20 spp): >= 98.5% of the subset's pixels inside
    the band |mean_gpu - mean_cpu| <= 3 sqrt(var_gpu/20 + var_cpu/20) (a t test
    with 38 degrees of freedom leaves 0.5% outside by chance), and the subset's
    mean difference inside 3 standard errors;
  * a 4096-spp render accumulated in FP64 (passes 40..4135, independent of
    both) is the reference image: the 20-spp GPU image's RMSE against it is
    within 10% of the Monte Carlo prediction sqrt(mean var (1/20 + 1/4096)),
    and the GPU's and the oracle's RMSE on the same pixels agree within 15%;
  * configuration 2 (level-6 displaced icosphere mesh mean, 512x512): the
    GPU's 64-spp image against 4 oracle passes per pixel of a 256-pixel subset,
    with the GPU's per-pixel variance (64 samples) standing in for both sides:
    >= 96% inside the band, mean difference inside 3 standard errors;
  * replayed samples (same passes on both sides): at most 3% differ, and the
    differing ones agree in mean within 3 standard errors (a path only parts
    from the reference's where the GPU's exp moves an f within ~1e-6 of zero
    across the sign test; both continuations are valid draws).
"""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuRenderer, GpuScene

pytestmark = pytest.mark.gpu


def _subset(rng, w, h, n):
    pix = rng.permutation(w * h)[:n]
    return (pix % w).astype(np.int32), (pix // w).astype(np.int32)


def _oracle_samples(port, sc, px, py, k0, passes):
    xs = np.repeat(px, passes)
    ys = np.repeat(py, passes)
    ks = np.tile(np.arange(k0, k0 + passes, dtype=np.int32), len(px))
    h = port.scene_create(sc.desc())
    try:
        return port.trace(h, xs, ys, ks).reshape(len(px), passes, 3).astype(np.float64)
    finally:
        port.scene_free(h)


def _render(gs, spp_begin, spp_end):
    r = GpuRenderer()
    r.prepare_render(gs)
    img, mom = r.start_render_progressive(spp_end, spp_begin=spp_begin, moments=True)
    n = spp_end - spp_begin
    mean = mom[:, :, :3] / n
    var = np.maximum(mom[:, :, 3:] / n - mean * mean, 0.0) * n / max(n - 1, 1)
    return img, mean, var


@pytest.fixture(scope="module")
def config0():
    sc = S.config0_scene(256, 256, 20)
    return sc, GpuScene(sc)


def test_config0_band_and_rmse_vs_4096spp(gpu, port, config0):
    sc, gs = config0
    spp = 20
    img, g_mean, g_var = _render(gs, 0, spp)
    # the framebuffer is the pass-ordered float running sum / spp: equal to the
    # FP64 mean within float rounding
    assert np.allclose(img, g_mean, rtol=1e-5, atol=1e-6)
    rng = np.random.default_rng(20)
    # half over the whole image, half in the central box the GP object covers
    px, py = _subset(rng, 256, 256, 512)
    cx, cy = (rng.integers(80, 176, 512).astype(np.int32) for _ in range(2))
    px, py = np.concatenate([px, cx]), np.concatenate([py, cy])
    cpu = _oracle_samples(port, sc, px, py, spp, spp)  # passes 20..39
    c_mean, c_var = cpu.mean(axis=1), cpu.var(axis=1, ddof=1)
    gm, gv = g_mean[py, px], g_var[py, px]
    sig = np.sqrt(gv / spp + c_var / spp)
    diff = gm - c_mean
    inside = np.all((np.abs(diff) <= 3 * sig) | ((sig == 0) & (diff == 0)), axis=1)
    assert inside.mean() >= 0.985, f"band {inside.mean():.4f}"
    se = np.sqrt(np.sum(sig * sig, axis=0)) / len(px)
    assert np.all(np.abs(diff.mean(axis=0)) <= 3 * se), (diff.mean(axis=0), se)
    assert (gm[:, 0] < 0.9).mean() > 0.15  # the GP surface covers part of the subset

    # 4096-spp FP64 reference image (passes 40..4135)
    _, ref, ref_var = _render(gs, 2 * spp, 2 * spp + 4096)
    rmse_gpu = np.sqrt(np.mean((g_mean - ref) ** 2))
    pred = np.sqrt(np.mean(ref_var) * (1.0 / spp + 1.0 / 4096))
    assert abs(rmse_gpu / pred - 1.0) < 0.10, (rmse_gpu, pred)
    ref_s = ref[py, px]
    rmse_gpu_s = np.sqrt(np.mean((gm - ref_s) ** 2))
    rmse_cpu_s = np.sqrt(np.mean((c_mean - ref_s) ** 2))
    assert abs(rmse_gpu_s / rmse_cpu_s - 1.0) < 0.15, (rmse_gpu_s, rmse_cpu_s)
    print(f"config0: band {inside.mean():.4f}; RMSE vs 4096 spp: GPU {rmse_gpu:.5f} (predicted {pred:.5f}), "
          f"subset GPU {rmse_gpu_s:.5f} CPU oracle {rmse_cpu_s:.5f}")


def test_config0_replay_divergence_bounded(gpu, port, config0):
    """Same passes on both sides over a 4096-pixel subset x 20 passes: the
    samples that do not replay bit for bit are few and unbiased."""
    sc, gs = config0
    rng = np.random.default_rng(21)
    px, py = _subset(rng, 256, 256, 4096)
    xs, ys = np.repeat(px, 20), np.repeat(py, 20)
    ks = np.tile(np.arange(20, dtype=np.int32), len(px))
    got = gs.trace(xs, ys, ks).astype(np.float64)
    h = port.scene_create(sc.desc())
    try:
        ref = port.trace(h, xs, ys, ks).astype(np.float64)
    finally:
        port.scene_free(h)
    differ = np.any(got.astype(np.float32).view(np.uint32) != ref.astype(np.float32).view(np.uint32), axis=1)
    frac = differ.mean()
    assert frac <= 0.03, frac
    if differ.sum() >= 10:
        d = got[differ] - ref[differ]
        se = d.std(axis=0, ddof=1) / np.sqrt(len(d)) + 1e-12
        assert np.all(np.abs(d.mean(axis=0)) <= 3 * se), (d.mean(axis=0), se)
    # where they sit: pixels whose replayed paths reach the GP surface
    # (radiance below the sky's 1.0 in some pass)
    hit_pix = (ref.reshape(len(px), 20, 3)[:, :, 0] < 1.0).any(axis=1)
    at_surface = hit_pix[np.nonzero(differ)[0] // 20].mean() if differ.any() else 1.0
    print(f"config0 replay: {frac:.4%} of {len(xs)} samples differ; mean |d| "
          f"{np.abs(got[differ] - ref[differ]).mean() if differ.any() else 0:.4f}; "
          f"{at_surface:.1%} of them in pixels that see the surface")


def test_config2_mesh_band(gpu, port):
    sc = S.config_mesh_scene(level=6, width=512, height=512, spp=64)
    gs = GpuScene(sc)
    spp = 64
    _, g_mean, g_var = _render(gs, 0, spp)
    rng = np.random.default_rng(22)
    # a subset weighted to the mesh: half of it inside the image's central box
    px, py = _subset(rng, 512, 512, 128)
    cx, cy = (rng.integers(160, 352, 128).astype(np.int32) for _ in range(2))
    px, py = np.concatenate([px, cx]), np.concatenate([py, cy])
    passes = 4
    cpu = _oracle_samples(port, sc, px, py, spp, passes)  # passes 64..67
    gm, gv = g_mean[py, px], g_var[py, px]
    c_mean = cpu.mean(axis=1)
    sig = np.sqrt(gv * (1.0 / spp + 1.0 / passes))
    diff = gm - c_mean
    inside = np.all((np.abs(diff) <= 3 * sig) | ((sig == 0) & (diff == 0)), axis=1)
    assert inside.mean() >= 0.96, f"band {inside.mean():.4f}"
    se = np.sqrt(np.sum(sig * sig, axis=0)) / len(px)
    assert np.all(np.abs(diff.mean(axis=0)) <= 3 * se), (diff.mean(axis=0), se)
    assert (gm[:, 0] < 0.9).mean() > 0.2  # the mesh medium's surface is in the subset
    print(f"config2: band {inside.mean():.4f} over {len(px)} pixels")
