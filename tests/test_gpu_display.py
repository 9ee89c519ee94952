"""The headless progressive display (csrc/display.cpp) and the Controller
over it (controller/controller.cpp:266-375), on the GPU: frames published
through the front/back swap, cancel and restart, skip_medium against the
reference, and applyGpMedium's kernel."""
import json
import os
import time

import numpy as np
import pytest

from mupsi_b200 import controller as CT
from mupsi_b200 import scene as S
from mupsi_b200.api import GpuDisplay, GpuRenderer, GpuScene

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _wait(d, timeout=60.0):
    t0 = time.time()
    while d.running():
        assert time.time() - t0 < timeout, "display render did not finish"
        time.sleep(0.002)


def _render(sc, spp):
    r = GpuRenderer()
    r.prepare_render(GpuScene(sc))
    return r.start_render_progressive(spp)


def test_display_frames_match_progressive_render(gpu):
    sc = S.config0_scene(32, 32, 6)
    d = GpuDisplay(sc)
    assert d.current_spp() == 0 and not d.is_spp_pass_done()
    assert not np.any(d.copy_raw())  # a fresh front buffer is black
    d.start_progressive(6, passes_per_frame=1)
    seen = []
    t0 = time.time()
    while d.running() or d.is_spp_pass_done():
        if d.is_spp_pass_done():
            seen.append(d.current_spp())
            d.ack_spp_pass()
            img = d.copy_raw()
            assert np.all(np.isfinite(img))
        assert time.time() - t0 < 60
        time.sleep(0.001)
    d.stop()
    assert d.current_spp() == 6
    assert seen == sorted(seen) and seen[-1] == 6
    raw = d.copy_raw()
    assert np.array_equal(bits(raw), bits(_render(sc, 6)))
    tm = d.copy_tonemapped()
    assert np.array_equal(bits(tm), bits(raw / (np.float32(1) + raw)))
    d.start(3)  # Controller::start: one frame with every pass
    _wait(d)
    d.stop()
    assert d.current_spp() == 3 and np.array_equal(bits(d.copy_raw()), bits(_render(sc, 3)))
    d.close()


def test_display_cancel_and_restart(gpu):
    sc = S.config0_scene(64, 64, 1)
    d = GpuDisplay(sc)
    d.start_progressive(100000, passes_per_frame=1)
    t0 = time.time()
    while not d.is_spp_pass_done():
        assert time.time() - t0 < 60
        time.sleep(0.001)
    d.cancel()
    d.stop()
    n = d.current_spp()
    assert 1 <= n < 100000 and not d.running()
    assert np.all(np.isfinite(d.copy_raw()))
    d.start_progressive(4, passes_per_frame=0)  # GPU-sized frames: all 4 passes in one
    _wait(d)
    d.stop()
    assert d.current_spp() == 4
    assert np.array_equal(bits(d.copy_raw()), bits(_render(sc, 4)))
    with pytest.raises(Exception):
        d.copy_raw(np.empty((8, 8, 3), np.float32))
    d.close()


def _write_scene(tmp_path, sc, name):
    objs = []
    for i, m in enumerate(sc.meshes):
        p = str(tmp_path / f"{name}{i}.obj")
        S.save_obj(p, m.vertices, m.faces)
        objs.append(p)
    j, extra = sc.to_json(objs)
    assert not extra
    j["output"] = str(tmp_path / f"{name}.png")
    p = str(tmp_path / f"{name}.json")
    json.dump(j, open(p, "w"))
    return p


def test_controller_applies_gp_kernel_and_saves(gpu, tmp_path):
    """startProgressive rebuilds the GP medium with the UI's sigma / length /
    points per cell and lengthScale (1, 1, 1) (controller.cpp:393-425)."""
    sc = S.config0_scene(24, 24, 3)
    sc.media[0]["aniso"] = (2.0, 1.0, 1.0)
    cfg = _write_scene(tmp_path, sc, "c0")
    c = CT.Controller()
    assert c.load(cfg, sky=1.0) and c.has_gp_medium() and c.get_spp() == 3
    c.set_gp_kernel_length(1.5)
    c.start_progressive(3)
    _wait(c.display)
    c.stop()
    want = S.config0_scene(24, 24, 3)
    want.media[0]["aniso"] = (1.0, 1.0, 1.0)
    want.media[0]["length"] = 1.5
    assert np.array_equal(bits(c.copy_display_raw_to()), bits(_render(want, 3)))
    assert not np.array_equal(bits(c.copy_display_raw_to()), bits(_render(sc, 3)))
    c.save_display()
    assert os.path.getsize(str(tmp_path / "c0.png")) > 100
    assert not CT.Controller().load(str(tmp_path / "missing.json"))
    c.close()


def test_skip_medium_trace(gpu, golden):
    """PathTracerSettings::skip_medium against the reference's trace with it set."""
    g = golden("trace_skip.npz")
    gs = GpuScene(S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5))
    gs.set_skip_medium(True)
    rad = gs.trace(g["x"], g["y"], g["k"])
    assert np.all(bits(rad) == bits(g["radiance"]), axis=1).mean() >= 0.97
    gs.set_skip_medium(False)
    assert np.any(bits(gs.trace(g["x"], g["y"], g["k"])) != bits(rad))


def test_controller_skip_medium_sticks(gpu, tmp_path):
    """startProgressive(spp, skipMedium) sets the flag for this and later
    renders, Controller::start included (controller.cpp:302)."""
    sc = S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5)
    sc.primitives[1]["albedo"] = (0.8, 0.8, 0.8)  # the default, so scene.json expresses the floor
    cfg = _write_scene(tmp_path, sc, "m")
    c = CT.Controller()
    assert c.load(cfg, sky=1.0)
    c.start_progressive(2, skip_medium=True)
    _wait(c.display)
    c.stop()
    gs = GpuScene(sc)
    gs.set_skip_medium(True)
    want = _render(sc, 2)
    r = GpuRenderer()
    r.prepare_render(gs)
    skipped = r.start_render_progressive(2)
    got = c.copy_display_raw_to()
    assert np.array_equal(bits(got), bits(skipped)) and not np.array_equal(bits(got), bits(want))
    c.start()  # spp 2 from the file, still without media
    _wait(c.display)
    c.stop()
    assert np.array_equal(bits(c.copy_display_raw_to()), bits(skipped))
    c.close()
