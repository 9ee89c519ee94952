"""SDFMedium, ExternalGPMedium and GridMeanFunction (medium/sdfmedium.cpp,
medium/externalgpmedium.cpp, gp/meanfunction.cpp:41-86): the C restatement
against fixtures made by the reference's own classes (per point, per ray, and
full traces of scenes loaded through Controller::load's sdf_medium /
external_gp_medium keys). All bit-exact."""
import numpy as np
import pytest

from mupsi_b200 import scene as S

KINDS = ["sdf_sphere", "sdf_mesh", "external_gp", "external_gp_mean"]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("kind", KINDS)
def test_field_medium_per_ray(port, golden, kind):
    g = golden("field_media.npz")
    h = port.scene_from(S.field_scene(kind))
    try:
        rays, seed = g[kind + "_rays"], g[kind + "_seed"]
        sd = port.sample_distance(h, 0, rays, seed)
        assert np.array_equal(bits(sd), bits(g[kind + "_sd"]))
        tr = port.transmittance(h, 0, rays, seed)
        assert np.array_equal(bits(tr), bits(g[kind + "_tr"]))
        ev = port.medium_eval(h, 0, g[kind + "_p"], g[kind + "_pseed"])
        assert np.array_equal(bits(ev), bits(g[kind + "_eval"]))
        if kind.startswith("external"):
            assert np.array_equal(bits(port.mean(h, 0, g[kind + "_p"])), bits(g[kind + "_grid"]))
    finally:
        port.scene_free(h)


@pytest.mark.parametrize("kind", KINDS)
def test_field_trace(port, golden, kind):
    g = golden("trace_field.npz")
    h = port.scene_from(S.field_scene(kind))
    try:
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g[kind]))
    finally:
        port.scene_free(h)


def test_field_json_round_trip(tmp_path):
    for kind in KINDS:
        sc = S.field_scene(kind)
        m = sc.media[0]
        obj = []
        for i, mesh in enumerate(sc.meshes):
            S.save_obj(str(tmp_path / f"{kind}{i}.obj"), mesh.vertices, mesh.faces)
            obj.append(str(tmp_path / f"{kind}{i}.obj"))
        gp = None
        if m["kind"] == "external_gp":
            m["mean_grid"].tofile(str(tmp_path / "m.bin"))
            if m["var_grid"] is not None:
                m["var_grid"].tofile(str(tmp_path / "v.bin"))
            gp = ("m.bin", "v.bin" if m["var_grid"] is not None else None)
        j, extra = sc.to_json(obj_paths=obj, grid_paths=gp)
        back = S.Scene.from_json(j, base_dir=str(tmp_path))
        b = back.media[0]
        assert b["kind"] == m["kind"] and back.primitives[0]["int_medium"] == 0
        if m["kind"] == "external_gp":
            assert np.array_equal(b["mean_grid"], m["mean_grid"].reshape(-1))
            assert (b["var_grid"] is None) == (m["var_grid"] is None)
            assert b["bmin"] == m["bmin"] and b["res"] == m["res"]
        elif m["mean_type"] == 1:
            assert np.array_equal(back.meshes[b["mesh"]].vertices, sc.meshes[m["mesh"]].vertices)


def test_grid_file_short_is_zero_padded(tmp_path):
    """GridMeanFunction reads what the file holds and leaves the rest 0."""
    np.arange(5, dtype=np.float32).tofile(str(tmp_path / "g.bin"))
    with pytest.warns(UserWarning):
        g = S.load_grid(str(tmp_path / "g.bin"), 2)
    assert g.tolist() == [0, 1, 2, 3, 4, 0, 0, 0]
