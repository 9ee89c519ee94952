"""The reference-side binding (integration/gpu_renderer.h/.cpp) compiled
against the reference's own headers and sources (oracle/Makefile, target
`binding`): the reference's Controller::load reads a scene.json, the
RenderContext is snapshotted as Controller::start does
(controller/controller.cpp:279-292), and GpuRenderer renders it through
libmupsi_gpu.so. Its framebuffer is compared with the reference's
Renderer::startRenderProgressive (rendering/renderer.cpp:22-49) on the same
scene: the GPU replays the reference's paths, so at least 95% of the pixels
must be equal bit for bit (the bar of the framebuffer fixture test) and the
image means must agree. The host's std::atomic<bool> cancel flag reaches the
GPU render through the binding."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from mupsi_b200 import scene as S

pytestmark = pytest.mark.gpu
ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
BINDING = os.path.join(ROOT, "oracle", "_ref", "libmupsi_ref_binding.so")


@pytest.fixture(scope="module")
def binding(gpu):
    if not os.path.exists(BINDING):
        pytest.fail(f"{BINDING} missing: built by `make -C oracle binding` beside the reference tree")
    L = C.CDLL(BINDING)
    L.bind_load.restype = C.c_void_p
    L.bind_load.argtypes = [C.c_char_p, C.c_int]
    L.bind_size.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.bind_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
    L.bind_free.argtypes = [C.c_void_p]
    return L


def _load(L, sc, tmp_path, name):
    objs = []
    for i, m in enumerate(sc.meshes):
        p = str(tmp_path / f"{name}_{i}.obj")
        S.save_obj(p, m.vertices, m.faces, m.texcoords, m.face_texcoords)
        objs.append(p)
    j, _ = sc.to_json(obj_paths=objs)
    jp = tmp_path / f"{name}.json"
    jp.write_text(json.dumps(j))
    h = L.bind_load(str(jp).encode(), 1)
    assert h
    return h


def _render(L, h, gpu, spp, cancel_after=0):
    w, hh = C.c_int(), C.c_int()
    L.bind_size(h, C.byref(w), C.byref(hh))
    out = np.zeros((hh.value, w.value, 3), np.float32)
    seen = C.c_int()
    rc = L.bind_render(h, 1 if gpu else 0, spp, cancel_after, out.ctypes.data, C.byref(seen))
    return rc, out, seen.value


@pytest.mark.parametrize("which", ["config0", "mesh"])
def test_gpu_renderer_matches_reference_renderer(binding, tmp_path, which):
    if which == "config0":
        sc = S.config0_scene(32, 32, 4)
    else:  # a displaced-icosphere mesh mean (no floor: scene.json cannot give it an albedo)
        # the reference evaluates the mesh mean by BVH at every march step: a small image
        sc = S.config_mesh_scene(level=2, width=20, height=20, spp=2, seed=4)
    h = _load(binding, sc, tmp_path, which)
    try:
        rc_g, gpu, seen_g = _render(binding, h, True, sc.spp)
        rc_c, cpu, seen_c = _render(binding, h, False, sc.spp)
    finally:
        binding.bind_free(h)
    assert rc_g == 0 and rc_c == 0
    assert seen_g == sc.spp and seen_c == sc.spp
    same = np.all(gpu.view(np.uint32) == cpu.view(np.uint32), axis=2)
    assert same.mean() >= 0.95, same.mean()
    assert abs(float(gpu.mean()) - float(cpu.mean())) < 0.01
    assert (cpu[..., 0] < 0.9).mean() > 0.02  # the medium's surface is in view


def test_gpu_renderer_cancel(binding, tmp_path):
    """The host's flag, set from the progress callback after the first wave of
    a render of several waves, stops the render; set beforehand, it stops the
    render before any wave."""
    sc = S.config0_scene(64, 64, 8192)  # 33.5 M path samples: more than one wave
    h = _load(binding, sc, tmp_path, "cancel")
    try:
        rc, _, seen = _render(binding, h, True, 8192, cancel_after=1)
        assert rc == 1 and 0 < seen < 8192
        rc0, _, seen0 = _render(binding, h, True, 16, cancel_after=0)
        assert rc0 == 0 and seen0 == 16
    finally:
        binding.bind_free(h)
