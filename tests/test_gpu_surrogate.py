"""Marching with the learned surrogate of a mesh mean (mupsi_gpu_scene_set_surrogate):
the network, trained on the GPU on exact BVH distances from the GPU's own mean,
answers the marches' far-field mean queries in batched tensor-core launches.
Shown here: what it gains (fewer exact BVH mean evaluations), that images stay
equal to the exact-mean render wherever its bound holds, and detaching."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200 import surrogate as SG
from mupsi_b200.api import GpuRenderer, GpuScene

pytestmark = pytest.mark.gpu

CENTER = np.array([0.0, 0.0, -300.0], np.float32)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def trained():
    sc = S.config_mesh_scene(level=4, width=40, height=40, spp=3, seed=2)
    gs = GpuScene(sc)
    m = sc.meshes[0]
    lo, hi = CENTER - 100, CENTER + 100
    P = SG.training_points(m.vertices, m.faces, 1 << 18, lo, hi, seed=0)
    T = gs.mean(0, P)[:, 0].copy()
    sm = SG.SurrogateMean(CENTER, 32.0, seed=0)
    losses = sm.train(P, T, steps=3000, batch=16384, lr=3e-3, lr_final=1e-5, seed=0)
    Q = SG.training_points(m.vertices, m.faces, 1 << 16, lo, hi, seed=1)
    TQ = gs.mean(0, Q)[:, 0].copy()
    pred = sm.infer(Q)
    margin = SG.bound_margin(pred, TQ, band=3.0, scale=1.5)
    return sc, gs, sm, margin, losses, np.abs(pred - TQ)


def render(gs, spp):
    r = GpuRenderer()
    r.prepare_render(gs)
    gs.profile(True)
    gs.stats(reset=True)
    img = r.start_render_progressive(spp)
    st = gs.stats(reset=True)
    gs.profile(False)
    return img, st


def test_surrogate_fits_held_out(trained):
    _, _, _, margin, losses, err = trained
    assert losses[-50:].mean() < 0.01 * losses[:5].mean()
    assert np.median(err) < 1.0 and margin < 20.0, (np.median(err), margin)


def test_surrogate_march_gains_and_matches_exact(gpu, trained):
    sc, gs, sm, margin, _, _ = trained
    exact, st_e = render(gs, sc.spp)
    gs2 = GpuScene(sc)
    SG.attach(gs2, 0, sm, band=3.0, scale=1.5, margin=margin, max_requests=8)
    surr, st_s = render(gs2, sc.spp)
    print("exact", st_e["mean_evals"], "surrogate", st_s["mean_evals"], st_s["surr_requests"], st_s["surr_accepted"])
    assert st_s["surr_requests"] > 0 and st_s["surr_accepted"] > 0
    # the gain: far-field exact BVH mean evaluations replaced by predictions
    assert st_s["mean_evals"] < 0.8 * st_e["mean_evals"], (st_s["mean_evals"], st_e["mean_evals"])
    same = np.all(bits(surr) == bits(exact), axis=2)
    assert same.mean() >= 0.97, same.mean()
    rmse = np.sqrt(np.mean((surr - exact) ** 2)) / max(1e-6, float(np.mean(exact)))
    assert rmse < 0.01, rmse
    # per-sample traces agree the same way
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(40), np.arange(40), np.arange(2),
                                                                 indexing="ij"))
    a, b = gs.trace(xs, ys, ks), gs2.trace(xs, ys, ks)
    assert np.all(bits(a) == bits(b), axis=1).mean() >= 0.97
    # detaching restores the exact render bit for bit
    SG.attach(gs2, 0, None)
    again, st_d = render(gs2, sc.spp)
    assert np.array_equal(bits(again), bits(exact)) and st_d["surr_requests"] == 0
    gs2.close()


def test_surrogate_rejects_bad_settings(gpu, trained):
    from mupsi_b200.lib import MupsiError
    sc, _, sm, _, _, _ = trained
    g = GpuScene(sc)
    for kw in [dict(scale=0.5), dict(margin=-1.0), dict(max_requests=0), dict(max_requests=33)]:
        with pytest.raises(MupsiError):
            SG.attach(g, 0, sm, **kw)
    with pytest.raises(MupsiError):
        SG.attach(g, 5, sm)
    s0 = S.config0_scene(8, 8, 1)  # a sphere mean has no surrogate
    with pytest.raises(MupsiError):
        SG.attach(GpuScene(s0), 0, sm)
    g.close()


def test_plain_every_step_mean_matches_lazy(gpu):
    """The plain exact form (BVH parity cast + closest point at every visited
    step) and the lazy exact form give the same samples: the lazy mean's bounds,
    crossings and intervals only skip queries whose answer they already know."""
    sc = S.config_mesh_scene(level=3, width=24, height=24, spp=2, seed=3)
    lazy, plain = GpuScene(sc), GpuScene(sc)
    plain.set_mean_eval(0, every_step=True)
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(24), np.arange(24), np.arange(2),
                                                                 indexing="ij"))
    a, b = lazy.trace(xs, ys, ks), plain.trace(xs, ys, ks)
    assert np.all(bits(a) == bits(b), axis=1).mean() >= 0.99
    plain.profile(True)
    plain.stats(reset=True)
    plain.trace(xs, ys, ks)
    st = plain.stats()
    assert st["mean_evals"] == 0  # no lazy evaluations: every step went through the full mean
    from mupsi_b200.lib import MupsiError
    with pytest.raises(MupsiError):
        plain.set_mean_eval(3, every_step=True)
