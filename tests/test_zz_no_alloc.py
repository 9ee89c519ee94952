"""The allocation-free trace entry (mupsi_gpu_trace_samples_noalloc) against the
regular one (mupsi_gpu_trace_samples), through the C ABI.

It serves render threads and hosts that cannot allocate device memory while
rendering (cudaMalloc/cudaFree can synchronise the whole device, and some hosts
own the GPU memory budget through their own allocator), so it keeps its path
state in one static device array instead. Both entries run the same kernels on
the same samples, so their radiance must agree exactly (the tolerance the trace
tests use for a path that replays the same random numbers: bit equality). The
allocation-free entry marches shadow rays inline where the regular one defers
them to shadow passes, and it never consults a surrogate; the scenes below
cover a medium lit by an emitter and a mesh mean (BVH queries in the march).
This file is collected last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuScene
from mupsi_b200.lib import MupsiError, load

pytestmark = pytest.mark.gpu


def _samples(w, h, passes, k0=0):
    xs, ys, ks = np.meshgrid(np.arange(w), np.arange(h), np.arange(k0, k0 + passes), indexing="ij")
    return [a.ravel().astype(np.int32) for a in (xs, ys, ks)]


def _check_twice(gs, w, h, calls):
    import torch
    # calls in a row with different samples: the shared scratch must not leak state
    for k0, passes in calls:
        xs, ys, ks = _samples(w, h, passes, k0)
        assert len(xs) <= 16384
        ref = gs.trace(xs, ys, ks)
        dx, dy, dk = (torch.from_numpy(a).cuda() for a in (xs, ys, ks))
        out = torch.full((len(xs), 3), -1.0, dtype=torch.float32, device="cuda")
        gs.trace_noalloc(dx, dy, dk, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    return ref


def test_noalloc_matches_trace_samples_twice(gpu):
    ref = _check_twice(GpuScene(S.config0_scene(48, 48, 8)), 48, 48, ((0, 4), (4, 3)))
    assert (ref[:, 0] < 1).sum() > 50  # the GP surface is in view


def test_noalloc_lit_medium(gpu):
    """An emitter lights the GP medium's surface: the regular entry defers the
    shadow rays of medium events to shadow passes, this one marches them inline."""
    sc = S.config0_scene(40, 40, 4)
    sc.add_sphere((40.0, 160.0, -380.0), 45.0, emission=(6.0, 5.0, 4.0))
    ref = _check_twice(GpuScene(sc), 40, 40, ((0, 4), (4, 2)))
    dark = GpuScene(S.config0_scene(40, 40, 4)).trace(*_samples(40, 40, 2, 4))
    assert (np.any(ref != dark, axis=1)).mean() > 0.02  # the NEE terms are present


def test_noalloc_mesh_mean(gpu):
    """A displaced-icosphere mesh mean: the march's lazy BVH queries."""
    gs = GpuScene(S.config_mesh_scene(level=4, width=32, height=32, spp=4, seed=3))
    ref = _check_twice(gs, 32, 32, ((0, 4), (4, 3)))
    assert (ref[:, 0] < 1).sum() > 20


def test_noalloc_allocates_nothing(gpu):
    """After the first call (which looks up the static array), calls leave the
    device's free memory unchanged: no allocation, no pool growth."""
    import torch
    gs = GpuScene(S.config_mesh_scene(level=3, width=32, height=32, spp=4, seed=5))
    xs, ys, ks = (torch.from_numpy(a).cuda() for a in _samples(32, 32, 4))
    out = torch.empty((len(xs), 3), dtype=torch.float32, device="cuda")
    gs.trace_noalloc(xs, ys, ks, out)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        gs.trace_noalloc(xs, ys, ks, out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_limits(gpu):
    import torch
    gs = GpuScene(S.config0_scene(16, 16, 1))
    n = 16385
    z = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(MupsiError, match="exceeds the maximum of 16384"):
        gs.trace_noalloc(z, z, z, out)
    with pytest.raises(ValueError):
        gs.trace_noalloc(np.zeros(4, np.int32), np.zeros(4, np.int32), np.zeros(4, np.int32),
                         np.zeros((4, 3), np.float32))
    # host memory passed straight to the C entry is refused, not dereferenced
    hz = torch.zeros(4, dtype=torch.int32).pin_memory()
    hout = torch.zeros((4, 3), dtype=torch.float32).pin_memory()
    dz = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = [C.c_void_p(t.data_ptr()) for t in (dz, dz, hz, hout)]
    rc = load().mupsi_gpu_trace_samples_noalloc(gs.h, 4, *p, None)
    assert rc == -1
    assert b"device buffers only" in load().mupsi_gpu_last_error()
