"""Next-event estimation and the surface BSDFs on the GPU against the CPU
oracle: sphere and mesh emitters (Sphere::sampleDirect, Mesh::sampleDirect),
shadow rays through the GP medium (GPMedium::transmittance) and through meshes
(BVH::occluded, including its start at node 0), Lambertian / specular / null
surfaces. Samples replay the reference's random numbers, so >= 97% of them must
agree bit for bit."""
import numpy as np
import pytest

from mupsi_b200 import _abi
from mupsi_b200 import scene as S
from mupsi_b200.api import GpuScene

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _replay(port, sc, w, h, passes):
    gs = GpuScene(sc)
    hh = port.scene_create(sc.desc())
    try:
        xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(w), np.arange(h), np.arange(passes),
                                                                     indexing="ij"))
        got = gs.trace(xs, ys, ks)
        ref = port.trace(hh, xs, ys, ks)
    finally:
        port.scene_free(hh)
    same = np.all(bits(got) == bits(ref), axis=1)
    return same, got, ref


def test_sphere_light_with_gp_medium(gpu, port):
    sc = S.config0_scene(40, 40, 3)
    sc.max_bounce = 6
    sc.add_sphere((160, 120, -420), 40.0, bsdf=_abi.BSDF_LAMBERTIAN, emission=(6.0, 5.0, 4.0))
    sc.add_sphere((-150, -60, -450), 50.0, bsdf=_abi.BSDF_LAMBERTIAN, albedo=(0.7, 0.5, 0.3))
    sc.add_sphere((-20, -160, -480), 45.0, bsdf=_abi.BSDF_SPECULAR)
    same, got, ref = _replay(port, sc, 40, 40, 3)
    assert same.mean() >= 0.97, same.mean()
    lit = (ref[:, 0] > 0) & (ref[:, 0] != 1.0) & (np.abs(ref[:, 0] - ref[:, 2]) > 1e-3)
    assert lit.sum() > 20  # coloured light reached the camera through NEE


def test_mesh_light_and_mesh_occluders(gpu, port):
    sc = S.config_mesh_scene(level=2, width=32, height=32, spp=2, seed=4)
    sc.max_bounce = 5
    qv = np.array([[-60, 120, -360], [60, 120, -360], [60, 120, -240], [-60, 120, -240]], np.float32)
    qf = np.array([[0, 1, 2], [0, 2, 3]], np.int32)  # normal -y: faces the scene
    mi = sc.add_mesh(S.Mesh(qv, qf))
    sc.add_mesh_primitive(mi, bsdf=_abi.BSDF_LAMBERTIAN, emission=(4.0, 4.0, 4.0))
    same, got, ref = _replay(port, sc, 32, 32, 2)
    assert same.mean() >= 0.97, same.mean()
    assert ((ref[:, 0] > 0) & (ref[:, 0] != 1.0)).sum() > 10


def test_march_stall_reports_device_limit(gpu):
    """A march whose t += dt cannot advance (dt below half an ulp of t) would
    never end in the reference; the GPU march stops it, reports
    MUPSI_ERR_DEVICE_LIMIT, and the context stays usable."""
    from mupsi_b200.lib import MupsiError
    gs = GpuScene(S.config0_scene(8, 8, 1))
    ray = np.array([[0, 0, 0, 0, 0, -1, 1000.0, 1000.0001]], np.float32)
    with pytest.raises(MupsiError) as e:
        gs.sample_distance(0, ray, np.array([7], np.uint32))
    assert e.value.code == _abi.ERR_DEVICE_LIMIT
    ok = np.array([[0, 0, -380, 0, 0, -1, 1.5e-3, np.finfo(np.float32).max]], np.float32)
    r = gs.sample_distance(0, ok, np.array([7], np.uint32))
    assert r[0, 0] == 0  # the next call works and hits the surface


def test_bvh_stack_overflow_reports_device_limit(gpu):
    """Triangles at exponentially growing x give a BVH deeper than the
    reference's 64-entry traversal stack; the GPU traversal stops and reports."""
    from mupsi_b200.api import DeviceMesh
    from mupsi_b200.lib import MupsiError
    n = 96
    xs = np.float32(2.5) ** np.arange(n, dtype=np.float32)
    v = np.zeros((3 * n, 3), np.float32)
    v[0::3, 0] = xs
    v[1::3, 0] = xs
    v[1::3, 1] = 1
    v[2::3, 0] = xs
    v[2::3, 2] = 1
    f = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    m = DeviceMesh(v, f)
    rays = np.array([[-1, 0.2, 0.2, 1, 0, 0, 0, np.finfo(np.float32).max]], np.float32)
    with pytest.raises(MupsiError) as e:
        m.intersect(rays)
    assert e.value.code == _abi.ERR_DEVICE_LIMIT
    tri, _ = m.intersect(np.array([[-1, 0.2, 0.2, -1, 0, 0, 0, 10]], np.float32))  # still usable
    assert tri[0] == 0xFFFFFFFF


def test_scene_occlusion_from_root(gpu):
    """Scene shadow rays with BVH::occluded from the root: an icosphere hanging
    between a sphere light and a floor shadows it, while the reference's start
    at node 0 (the default) lets most shadow rays through."""
    sc = S.Scene()
    sc.width = sc.height = 32
    sc.max_bounce = 3
    fv, ff = S.floor_quad()
    sc.add_mesh_primitive(sc.add_mesh(S.Mesh(fv, ff)), bsdf=_abi.BSDF_LAMBERTIAN, albedo=0.7)
    ov, of = S.displaced_icosphere(3, radius=50.0, center=(0.0, 40.0, -400.0), seed=1)
    sc.add_mesh_primitive(sc.add_mesh(S.Mesh(ov, of)), bsdf=_abi.BSDF_LAMBERTIAN, albedo=0.5)
    sc.add_sphere((0.0, 220.0, -400.0), 30.0, bsdf=_abi.BSDF_LAMBERTIAN, emission=(20.0, 20.0, 20.0))
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(32), np.arange(32), np.arange(2),
                                                                 indexing="ij"))
    ref_mode = GpuScene(sc).trace(xs, ys, ks)
    g = GpuScene(sc)
    g.set_occlusion(True)
    root_mode = g.trace(xs, ys, ks)
    darker = np.all(root_mode <= ref_mode * (1 + 1e-5) + 1e-6, axis=1)
    assert darker.all()  # the same paths; only NEE contributions can disappear
    assert (root_mode.sum(axis=1) < ref_mode.sum(axis=1) - 1e-3).sum() > 10


@pytest.mark.parametrize("kind", ["gp", "sdf_sphere", "external_gp"])
def test_deferred_shadow_rays_match_inline(gpu, kind):
    """A medium event's shadow ray (Medium::transmittance) is marched by a
    shadow pass of the next bounce iteration (the march kernel's for a GP
    medium, the field march kernel's for an SDF or external GP medium), which
    adds the NEE term before the path's next shading; the allocation-free
    trace has no room for those jobs and marches the ray inline in the shading
    kernel. Both must give the same bits, with the NEE terms present."""
    import torch
    if kind == "gp":
        sc = S.config0_scene(64, 64, 4)
        sc.add_sphere((40.0, 160.0, -380.0), 45.0, emission=(6.0, 5.0, 4.0))
    else:
        sc = S.field_scene(kind, 64, 64, 4)  # with its emissive sphere
    gs = GpuScene(sc)
    xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(64), np.arange(64), np.arange(4),
                                                                 indexing="ij"))
    deferred = gs.trace(xs, ys, ks)
    out = torch.full((len(xs), 3), -1.0, dtype=torch.float32, device="cuda")
    gs.trace_noalloc(*(torch.from_numpy(a).cuda() for a in (xs, ys, ks)), out)
    torch.cuda.synchronize()
    inline = out.cpu().numpy()
    assert np.array_equal(deferred.view(np.uint32), inline.view(np.uint32))
    if kind == "gp":
        dark = GpuScene(S.config0_scene(64, 64, 4)).trace(xs, ys, ks)
        assert (np.any(deferred != dark, axis=1)).mean() > 0.05  # the light reaches the medium's surface
