"""CPU-only checks of the host side: the library loads and exports every
symbol include/mupsi_gpu.h declares, the host BVH builder reproduces the
reference's node arrays, and scene descriptions round-trip through scene.json."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from mupsi_b200 import _abi
from mupsi_b200 import scene as S

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _declared():
    src = open(os.path.join(ROOT, "include", "mupsi_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mupsi_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from mupsi_b200 import build
    build.build()
    from mupsi_b200 import lib as L
    return L.load()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert lib.mupsi_gpu_abi_version() == 4


def test_host_bvh_build_matches_reference_fixture(lib, golden):
    from mupsi_b200.api import bvh_build_host
    g = golden("bvh_mesh.npz")
    nodes, idx, root = bvh_build_host(g["verts"], g["faces"])
    assert np.array_equal(nodes, g["nodes"]) and np.array_equal(idx, g["tri_idx"]) and root == g["root"]


@pytest.mark.parametrize("level", [0, 2, 5])
def test_host_bvh_build_matches_oracle(lib, port, level):
    from mupsi_b200.api import bvh_build_host
    v, f = S.displaced_icosphere(level, seed=level + 11)
    a = bvh_build_host(v, f)
    b = port.bvh_build(v, f)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_host_bvh_build_rejects_bad_faces(lib):
    from mupsi_b200.api import bvh_build_host
    from mupsi_b200.lib import MupsiError
    v = np.zeros((3, 3), np.float32)
    with pytest.raises(MupsiError):
        bvh_build_host(v, np.array([[0, 1, 3]], np.int32))
    nodes, idx, root = bvh_build_host(v, np.zeros((0, 3), np.int32))
    assert len(nodes) == 0


def test_scene_json_roundtrip(tmp_path):
    sc = S.config0_scene(32, 16, 5)
    j, extra = sc.to_json()
    assert not extra
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(j))
    back = S.Scene.from_json(str(p), sky=1.0)
    a, b = sc.desc(), back.desc()
    for f, _ in _abi.SceneDesc._fields_:
        if f in ("media", "meshes", "primitives"):
            continue
        va, vb = getattr(a, f), getattr(b, f)
        if hasattr(va, "__len__"):
            assert list(va) == list(vb), f
        else:
            assert va == vb, f
    assert back.media[0]["length"] == 1.0 and back.primitives[0]["int_medium"] == 0


def test_scene_json_defaults_and_errors(tmp_path):
    j = {"camera": {"pos": [0, 0, 0], "dir": [0, 0, -1]}, "primitives": [{"type": "sphere", "center": [0, 0, -5]}]}
    s = S.Scene.from_json(j)
    assert (s.width, s.height, s.max_bounce, s.cam_fov, s.gp_mode) == (256, 256, 3, 45.0, 0)
    assert s.primitives[0]["radius"] == 100.0 and s.sky is None
    with pytest.raises(ValueError):
        S.Scene.from_json({"camera": j["camera"]})
    with pytest.raises(KeyError):  # a sphere SDF needs its mean_center
        S.Scene.from_json(dict(j, sdf_medium={}))
    prim = {"type": "sphere", "center": [0, 0, -5], "int_medium": True}
    s = S.Scene.from_json(dict(j, sdf_medium={"mean_center": [0, 0, -5], "mean_radius": 2.0}, primitives=[prim]))
    assert s.media[0]["kind"] == "sdf" and s.primitives[0]["int_medium"] == 0
    # gp_medium wins over sdf_medium for int_medium primitives (controller.cpp:225-229)
    s = S.Scene.from_json(dict(j, sdf_medium={"mean_center": [0, 0, -5]},
                               gp_medium={"mean_center": [0, 0, -5]}, primitives=[prim]))
    assert len(s.media) == 1 and s.media[0]["kind"] == "gp"


def test_obj_roundtrip(tmp_path):
    v, f = S.displaced_icosphere(1, seed=1)
    p = tmp_path / "m.obj"
    S.save_obj(str(p), v, f)
    v2, f2, n2 = S.load_obj(str(p))
    assert np.array_equal(v, v2) and np.array_equal(f, f2) and n2 is None


def test_icosphere_sizes():
    for level, nf, nv in ((6, 81920, 40962), (8, 1310720, 655362)):
        assert 20 * 4**level == nf and 10 * 4**level + 2 == nv
    v, f = S.icosphere(3)
    assert len(f) == 1280 and len(v) == 642


def test_batch_scenes_parameters():
    from mupsi_b200 import _abi
    sc = S.batch_scenes()
    assert len(sc) == 64
    assert {s.width for s in sc} <= {64, 128, 256, 512} and all(s.width == s.height for s in sc)
    assert all(4 <= s.spp <= 64 and 2 <= s.max_bounce <= 10 for s in sc)
    assert sum(s.gp_mode == _abi.GP_SINGLE_REALIZATION for s in sc) == 32
    for s in sc:
        m = s.media[0]
        assert 0.25 <= m["length"] <= 4.0 and m["ppc"] in (1, 3, 8) and 20.0 <= m["radius"] <= 100.0
        assert abs(s.primitives[0]["radius"] - 1.8 * m["radius"]) < 1e-3
    again = S.batch_scenes()
    assert [(s.width, s.spp, s.media[0]["length"]) for s in sc] == [(s.width, s.spp, s.media[0]["length"])
                                                                    for s in again]


def test_autotune_coordinate_descent():
    from mupsi_b200.autotune import CANDIDATES, DEFAULT, coordinate_descent
    target = {"march_block": 96, "min_group": 16, "shade_block": 64, "wave_paths": 1 << 22, "block_rays": 4,
              "lane_rays": 0, "lane_max_tris": 1 << 18, "mu_batch": 24}

    def cost(cfg):
        return sum(abs(np.log2(cfg[k] + 1) - np.log2(target[k] + 1)) for k in target) + 1.0

    best, t, trials = coordinate_descent(cost, CANDIDATES, DEFAULT, passes=3)
    assert best == target and t == 1.0
    assert len({tuple(sorted(x["config"].items())) for x in trials}) == len(trials)


def test_tuning_file_is_valid():
    import json
    from mupsi_b200.api import TUNING_FILE
    from mupsi_b200.autotune import CANDIDATES
    if not os.path.exists(TUNING_FILE):
        pytest.skip("no tuning file committed")
    t = json.load(open(TUNING_FILE))["tuning"]
    for k, v in t.items():
        assert v in CANDIDATES[k]


def test_buffer_checks_reject_short_buffers():
    """The wrappers refuse buffers the library would over-read or over-write."""
    from mupsi_b200 import api
    api._need(np.zeros((4, 3), np.float32), (4, 3), "p")
    with pytest.raises(ValueError):
        api._need(np.zeros((4, 2), np.float32), (4, 3), "p")
    with pytest.raises(ValueError):
        api._need(np.zeros(3, np.uint32), (4,), "seed")
    api.check_buf(np.zeros((2, 3, 3), np.float32), (2, 3, 3))
    with pytest.raises(ValueError):
        api.check_buf(np.zeros((8, 8, 3), np.float32), (64, 64, 3))
    with pytest.raises(ValueError):
        api.check_buf(np.zeros((2, 3, 3), np.float64), (2, 3, 3))
