"""Controller (controller/controller.h, controller.cpp): scene.json loading,
render control and the double-buffered display, over the GPU path tracer.

The render thread and the front/back buffers are native (GpuDisplay,
csrc/display.cpp); this class keeps the reference's names and its
bookkeeping: the GP parameters a UI edits are applied when a progressive
render starts (Controller::applyGpMedium rebuilds the GPMedium with the
edited sigma, length scale and points per cell and a lengthScale vector of
(1, 1, 1), whatever the file said), skip_medium sticks until the next
start_progressive, and save_display writes the front frame as the
reference's Framebuffer::save does.
"""
import json
import os
import struct
import sys
import zlib

import numpy as np

from . import _abi
from . import scene as S
from .api import GpuDisplay, GpuScene, SparseSEKernel


def applied_kernel(sigma, length, points_per_cell):
    """The kernel Controller::applyGpMedium builds (controller.cpp:414-417)."""
    return SparseSEKernel(sigma, length, (1.0, 1.0, 1.0)).struct(points_per_cell)


def tonemap(v):
    """Framebuffer::tonemapped (framebuffer.cpp:37-45): Reinhard v / (1 + v)."""
    v = np.asarray(v, np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):  # v = -1 and inf divide as the float code does
        return (v / (np.float32(1.0) + v)).astype(np.float32)


def tonemap8(v):
    """Framebuffer::save's 8-bit pixels (framebuffer.cpp:62-74):
    uint8(clamp(v / (1 + v), 0, 1) * 255), truncated."""
    t = np.clip(tonemap(v), np.float32(0.0), np.float32(1.0))
    t = np.nan_to_num(t, nan=0.0)
    return (t * np.float32(255.0)).astype(np.uint8)


def write_png(path, rgb8):
    """8-bit RGB PNG (rows top first), stored with filter 0 and zlib."""
    rgb8 = np.ascontiguousarray(rgb8, np.uint8)
    h, w, _ = rgb8.shape
    raw = b"".join(b"\x00" + rgb8[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as fh:
        fh.write(b"\x89PNG\r\n\x1a\n")
        fh.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        fh.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        fh.write(chunk(b"IEND", b""))


def write_hdr(path, rgb):
    """Radiance RGBE (.hdr) with flat scanlines, rows top first."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w, _ = rgb.shape
    m = rgb.max(axis=2)
    mant, ex = np.frexp(m)
    scale = np.where(m > 1e-32, mant * 256.0 / np.where(m > 0, m, 1.0), 0.0)
    rgbe = np.zeros((h, w, 4), np.uint8)
    rgbe[..., :3] = np.clip(rgb * scale[..., None], 0, 255).astype(np.uint8)
    rgbe[..., 3] = np.where(m > 1e-32, ex + 128, 0).astype(np.uint8)
    with open(path, "wb") as fh:
        fh.write(f"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y {h} +X {w}\n".encode())
        fh.write(rgbe.tobytes())


def save_image(path, rgb):
    """Framebuffer::save (framebuffer.cpp:47-76): the image is written bottom
    row first (row h-1-y of the file is framebuffer row y); .hdr as float
    RGBE, anything else as an 8-bit tonemapped PNG. .exr needs OpenCV (cv2)."""
    flipped = np.ascontiguousarray(np.asarray(rgb, np.float32)[::-1])
    if path.endswith(".exr"):
        import cv2
        cv2.imwrite(path, flipped[..., ::-1].copy())
    elif path.endswith(".hdr"):
        write_hdr(path, flipped)
    else:
        write_png(path, tonemap8(flipped))


class Controller:
    """The reference's Controller over a GpuScene and a GpuDisplay."""

    def __init__(self):
        self.scene = None       # Scene (host description)
        self.gpu_scene = None   # GpuScene
        self.display = None     # GpuDisplay
        self._spp = 1
        self._config_path = ""
        self._output_path = "test.png"
        self._skip_medium = False
        self._gp_medium = -1     # index of the gp_medium in the scene's media
        self._has_gp_medium = False
        self._sigma, self._length, self._ppc = 1.0, 1.0, 3
        self._gp_mode = "single_realization"

    # -- loading ---------------------------------------------------------------
    def load(self, config_path, sky=None):
        """Controller::load (controller.cpp:40-264); False (with a message on
        stderr) where the reference returns false. `sky`: a constant skydrome
        (the reference's file format names only images)."""
        self.stop()
        try:
            with open(config_path) as fh:
                j = json.load(fh)
            sc = S.Scene.from_json(config_path, sky=sky)
        except (OSError, ValueError, KeyError) as e:
            print(f"Controller::load: {config_path}: {e}", file=sys.stderr)
            return False
        if self.display is not None:
            self.display.close()
        self.scene = sc
        self.gpu_scene = GpuScene(sc)
        self.display = GpuDisplay(self.gpu_scene)
        self._config_path = config_path
        self._spp = int(j.get("spp", 1))
        self._output_path = j.get("output", "test.png")
        self._has_gp_medium = "gp_medium" in j
        self._gp_medium = 0 if self._has_gp_medium else -1
        kern = j.get("kernel", {})
        self._sigma = float(kern.get("sigma", 1.0))
        self._length = float(kern.get("length_scale", 1.0))
        self._ppc = int(kern.get("points_per_cell", 3))
        self._gp_mode = j.get("gp_mode", "single_realization")
        return True

    def _require(self):
        if self.display is None:
            raise RuntimeError("no scene loaded")

    def _apply_settings(self):
        mode = _abi.GP_RENEWAL_PLUS if self._gp_mode == "renewal_plus" else _abi.GP_SINGLE_REALIZATION
        self.gpu_scene.set_gp_mode(mode)
        self.gpu_scene.set_skip_medium(self._skip_medium)

    # -- render control ----------------------------------------------------------
    def start(self):
        """Controller::start: all spp passes, shown once at the end."""
        self._require()
        self.stop()
        self._apply_settings()
        self.display.start(self._spp)

    def start_progressive(self, target_spp, skip_medium=False, passes_per_frame=1):
        """Controller::startProgressive: a frame after every `passes_per_frame`
        passes (1 as the reference; 0 for GPU-sized frames)."""
        self._require()
        self.stop()
        self._skip_medium = bool(skip_medium)
        self._apply_settings()
        if self._has_gp_medium:  # applyGpMedium (controller.cpp:393-425)
            self.gpu_scene.set_kernel(self._gp_medium, applied_kernel(self._sigma, self._length, self._ppc))
        self.display.start_progressive(target_spp, passes_per_frame)

    def cancel(self):
        if self.display is not None:
            self.display.cancel()

    def stop(self):
        if self.display is not None:
            self.display.stop()

    def is_running(self):
        return self.display is not None and self.display.running()

    def is_spp_pass_done(self):
        return self.display is not None and self.display.is_spp_pass_done()

    def ack_spp_pass(self):
        if self.display is not None:
            self.display.ack_spp_pass()

    def get_current_spp(self):
        return 0 if self.display is None else self.display.current_spp()

    # -- display -------------------------------------------------------------------
    def copy_display_to(self, dst=None):
        """copyDisplayTo: the front frame tonemapped, (h, w, 3) float32."""
        self._require()
        return self.display.copy_tonemapped(dst)

    def copy_display_raw_to(self, dst=None):
        """copyDisplayRawTo: the front frame un-tonemapped."""
        self._require()
        return self.display.copy_raw(dst)

    def save_display(self, path=None):
        """saveDisplay: the front frame to `path` (default: the config's output)."""
        self._require()
        save_image(path or self._output_path, self.display.copy_raw())

    # -- settings ------------------------------------------------------------------
    def get_spp(self):
        return self._spp

    def output_path(self):
        return self._output_path

    def set_output_path(self, path):
        self._output_path = path

    def config_path(self):
        return self._config_path

    def has_gp_medium(self):
        return self._has_gp_medium

    def gp_kernel_sigma(self):
        return self._sigma

    def set_gp_kernel_sigma(self, v):
        self._sigma = float(v)

    def gp_kernel_length(self):
        return self._length

    def set_gp_kernel_length(self, v):
        self._length = float(v)

    def gp_points_per_cell(self):
        return self._ppc

    def set_gp_points_per_cell(self, v):
        self._ppc = int(v)

    def gp_mode(self):
        return self._gp_mode

    def set_gp_mode(self, v):
        """renewal_plus or anything else (single realization), as setGpMode."""
        self._gp_mode = v

    def close(self):
        if self.display is not None:
            self.display.close()
            self.display = None
