"""Host side of the progressive display (controller/controller.cpp): the
skip_medium trace against the reference, the kernel applyGpMedium builds,
and Framebuffer::save's pixel conversion and file layout. GPU parts are in
test_gpu_display.py."""
import struct
import zlib

import numpy as np

from mupsi_b200 import controller as CT
from mupsi_b200 import scene as S


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_trace_skip_medium(port, golden):
    g = golden("trace_skip.npz")
    h = port.scene_from(S.config_mesh_scene(level=2, width=16, height=16, spp=2, seed=5))
    try:
        port.scene_set_skip_medium(h, True)
        rad = port.trace(h, g["x"], g["y"], g["k"])
        assert np.array_equal(bits(rad), bits(g["radiance"]))
        port.scene_set_skip_medium(h, False)
        assert np.any(bits(port.trace(h, g["x"], g["y"], g["k"])) != bits(rad))
    finally:
        port.scene_free(h)


def test_applied_kernel_resets_aniso():
    k = CT.applied_kernel(0.5, 2.0, 7)
    assert (k.sigma, k.kernel_radius, k.points_per_cell) == (0.5, 2.0, 7)
    assert list(k.aniso) == [1.0, 1.0, 1.0]


def test_tonemap8_truncates():
    v = np.float32([[[0.0, 1.0, 3.0], [np.inf, -1.0, 0.25]]])
    t = CT.tonemap8(v)
    # v/(1+v) * 255, truncated: 0, 127.5 -> 127, 191.25 -> 191; inf -> nan -> 0; -1 -> -inf -> 0; 0.2*255 = 51
    assert t.tolist() == [[[0, 127, 191], [0, 0, 51]]]


def _read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(tag + body) & 0xFFFFFFFF
        chunks[tag] = chunks.get(tag, b"") + body
        pos += 12 + n
    w, h = struct.unpack(">II", chunks[b"IHDR"][:8])
    raw = zlib.decompress(chunks[b"IDAT"])
    rows = [raw[y * (3 * w + 1) + 1:(y + 1) * (3 * w + 1)] for y in range(h)]
    assert all(raw[y * (3 * w + 1)] == 0 for y in range(h))
    return np.frombuffer(b"".join(rows), np.uint8).reshape(h, w, 3)


def test_save_png_flips_and_tonemaps(tmp_path):
    rgb = np.random.default_rng(0).uniform(0, 4, (5, 7, 3)).astype(np.float32)
    p = str(tmp_path / "out.png")
    CT.save_image(p, rgb)
    img = _read_png(p)
    assert np.array_equal(img, CT.tonemap8(rgb)[::-1])  # file row h-1-y is framebuffer row y


def test_save_hdr(tmp_path):
    rgb = np.random.default_rng(1).uniform(0.01, 40, (3, 4, 3)).astype(np.float32)
    p = str(tmp_path / "out.hdr")
    CT.save_image(p, rgb)
    data = open(p, "rb").read()
    head = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 3 +X 4\n"
    assert data.startswith(head)
    e = np.frombuffer(data[len(head):], np.uint8).reshape(3, 4, 4).astype(np.float64)
    dec = e[..., :3] * np.ldexp(1.0, (e[..., 3] - 136).astype(int))[..., None]
    # RGBE keeps 8 bits under the pixel's largest channel
    err = np.abs(dec - rgb[::-1]) / rgb[::-1].max(axis=2, keepdims=True)
    assert err.max() <= 1.0 / 128
