"""Mean functions, GPMedium::evalWithGradient, sampleDistance and sampleCondition
on the GPU against the CPU oracle and the reference's fixtures.

Bit-exact: mean values/gradients (sphere and mesh), march step t and hit
point p, conditioning point C. Within tolerance: f and grad f of
evalWithGradient to 1e-5 of the scale of their noise terms (the sum of the
absolute values of the psi impulse terms and of the Renewal+ conditioning
terms; the mean part is bit-exact and adds nothing) plus one rounding of the
final sum, 2^-22 |f|; u_tilde, g_tilde to 1e-4.
The march outcome depends on signs of f, which the GPU's exp can flip only
when f is within ~1e-6 of zero, so march agreement is asserted per ray at
>= 99.5% with every disagreement reported."""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuScene

pytestmark = pytest.mark.gpu
FMAX = np.finfo(np.float32).max


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _cond(rng, p, spread=2.0, active_every=2):
    n = len(p)
    c = np.zeros((n, 8), np.float32)
    c[:, :3] = p + rng.normal(size=(n, 3)).astype(np.float32) * spread
    c[:, 3] = rng.normal(size=n)
    c[:, 4:7] = rng.normal(size=(n, 3))
    c[::active_every, 7] = 1
    return c


def _noise_tol(port, med, p, seed, cond, f):
    """1e-5 of the per-output scale of the noise terms at p, plus one rounding
    of f = mu + psi + conditioning (2^-22 |f| covers two roundings' spread)."""
    from oracle import bind
    k = bind.kernel_struct(med["sigma"], med["length"], med["aniso"], med["ppc"])
    _, s_psi = port.psi_f64(k, p, seed)
    L2 = float(np.float32(med["aniso"][0]) ** 2 + (np.float32(med["aniso"][1]) ** 2 + np.float32(med["aniso"][2]) ** 2))
    c2, c4 = -2.0 / L2, 4.0 / (L2 * L2)
    r = p.astype(np.float64) - cond[:, :3]
    h = np.exp(-np.sum(r * r, axis=1) / L2)
    u, g = cond[:, 3].astype(np.float64), cond[:, 4:7].astype(np.float64)
    hg = (h * c2)[:, None] * r
    rg = np.sum(r * g, axis=1)
    s_c = np.zeros((len(p), 4))
    s_c[:, 0] = np.abs(u * h) + np.sum(np.abs(g * hg), axis=1)
    s_c[:, 1:] = np.abs(u[:, None] * hg) + np.abs(h[:, None] * c2 * g) + np.abs((h * c4 * rg)[:, None] * r)
    s_c[cond[:, 7] == 0] = 0.0
    return 1e-5 * (s_psi + s_c) + 2.0 ** -22 * np.abs(f)


@pytest.fixture(scope="module")
def sphere_scene():
    return S.config0_scene(16, 16, 1)


@pytest.fixture(scope="module")
def mesh_scene():
    return S.config_mesh_scene(level=4, width=16, height=16, spp=1, seed=3)


def test_mean_bit_exact(gpu, port, sphere_scene, mesh_scene):
    rng = np.random.default_rng(0)
    for sc, c in ((sphere_scene, -500), (mesh_scene, -300)):
        g = GpuScene(sc)
        h = port.scene_create(sc.desc())
        try:
            q = (rng.uniform(-150, 150, (20000, 3)) + np.array([0, 0, c])).astype(np.float32)
            assert np.array_equal(bits(g.mean(0, q)), bits(port.mean(h, 0, q)))
        finally:
            port.scene_free(h)


def test_medium_eval(gpu, port, sphere_scene, mesh_scene):
    rng = np.random.default_rng(1)
    for sc, c in ((sphere_scene, -500), (mesh_scene, -300)):
        g = GpuScene(sc)
        h = port.scene_create(sc.desc())
        try:
            q = (rng.uniform(-100, 100, (8192, 3)) + np.array([0, 0, c])).astype(np.float32)
            s = rng.integers(0, 2**32, len(q), dtype=np.uint64).astype(np.uint32)
            cond = _cond(rng, q)
            got = g.eval_with_gradient(0, q, s, cond)
            ref = port.medium_eval(h, 0, q, s, cond)
            tol = _noise_tol(port, sc.media[0], q, s, cond, ref)
            err = np.abs(got.astype(np.float64) - ref)
            assert np.all(err <= tol), f"max err/tol {np.max(err / tol):.3g}"
        finally:
            port.scene_free(h)


def test_medium_fixtures(gpu, port, golden):
    g = golden("medium_sphere.npz")
    sc0 = S.config0_scene(8, 8, 1)
    gs = GpuScene(sc0)
    got = gs.eval_with_gradient(0, g["points"], g["seeds"], g["cond"])
    ref = g["medium_eval"].astype(np.float64)
    assert np.all(np.abs(got - ref) <= _noise_tol(port, sc0.media[0], g["points"], g["seeds"], g["cond"], ref))
    sd = gs.sample_distance(0, g["rays"], g["seeds"], g["cond"])
    ref = g["sample_distance"]
    same = (sd[:, 0] == ref[:, 0]) & (bits(sd[:, 1]) == bits(ref[:, 1]))
    assert same.mean() >= 0.99, np.nonzero(~same)
    hit = same & (ref[:, 0] == 0)
    assert np.array_equal(bits(sd[hit, 2:5]), bits(ref[hit, 2:5]))
    assert np.all(np.abs(sd[hit, 5:8] - ref[hit, 5:8]) < 1e-4)
    mb = golden("bvh_mesh.npz")
    sc = S.Scene()
    mi = sc.add_mesh(S.Mesh(mb["verts"], mb["faces"]))
    sc.add_medium("mesh", mesh=mi, length_scale=2.0)
    gm = GpuScene(sc)
    assert np.array_equal(bits(gm.mean(0, mb["points"])), bits(mb["mean"]))
    got = gm.eval_with_gradient(0, mb["points"], mb["seeds"], mb["cond"])
    ref = mb["medium_eval"].astype(np.float64)
    assert np.all(np.abs(got - ref) <= _noise_tol(port, sc.media[0], mb["points"], mb["seeds"], mb["cond"], ref))


def _march_rays(rng, n, center, rin, rout, nt=1.5e-3):
    o = np.zeros((n, 3), np.float32)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    o[:] = np.array(center) + dirs * rng.uniform(rin, rout, (n, 1))
    tgt = np.array(center) + rng.normal(size=(n, 3)) * 30
    d = (tgt - o).astype(np.float32)
    d[n // 2:] = rng.normal(size=(n - n // 2, 3)).astype(np.float32)
    r = np.zeros((n, 8), np.float32)
    r[:, :3], r[:, 3:6], r[:, 6], r[:, 7] = o, d, nt, FMAX
    return r


@pytest.mark.parametrize("which", ["sphere", "mesh"])
def test_sample_distance_and_condition(gpu, port, sphere_scene, mesh_scene, which):
    rng = np.random.default_rng(2)
    sc, center, rin, rout = ((sphere_scene, (0, 0, -500), 40, 130) if which == "sphere"
                             else (mesh_scene, (0, 0, -300), 30, 100))
    n = 3000 if which == "sphere" else 600
    g = GpuScene(sc)
    h = port.scene_create(sc.desc())
    try:
        rays = _march_rays(rng, n, center, rin, rout)
        rays[::9, 6] = 0.0          # nearT 0: the sequential-add path
        rays[::13, 7] = 250.0       # finite farT: shorter dt
        s = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        cond = _cond(rng, rays[:, :3], spread=3.0, active_every=3)
        got = g.sample_distance(0, rays, s, cond)
        ref = port.sample_distance(h, 0, rays, s, cond)
        same = (got[:, 0] == ref[:, 0]) & (bits(got[:, 1]) == bits(ref[:, 1]))
        assert same.mean() >= 0.995, f"march agreement {same.mean():.4f}"
        hit = same & (ref[:, 0] == 0)
        assert hit.sum() > n // 10 and (same & (ref[:, 0] == 1)).sum() > n // 10
        assert np.array_equal(bits(got[hit, 2:5]), bits(ref[hit, 2:5]))
        assert np.all(np.abs(got[hit, 5:8] - ref[hit, 5:8]) < 1e-4)
        # conditioning at the reference's hits with the next seed
        hits = np.concatenate([ref[:, :1], ref[:, 2:8]], axis=1)
        s2 = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        cg = g.sample_condition(0, hits, s2)
        cr = port.sample_condition(h, 0, hits, s2)
        assert np.array_equal(cg[:, 7], cr[:, 7]) and np.array_equal(bits(cg[:, :3]), bits(cr[:, :3]))
        act = cr[:, 7] == 1
        assert np.all(np.abs(cg[act, 3:7] - cr[act, 3:7]) <= 1e-4 * (1 + np.abs(cr[act, 3:7])))
    finally:
        port.scene_free(h)
