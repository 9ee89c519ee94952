"""The allocation-free trace entry (mupsi_gpu_trace_samples_noalloc) against the
regular one (mupsi_gpu_trace_samples), through the C ABI.

It serves render threads and hosts that cannot allocate device memory while
rendering (cudaMalloc/cudaFree can synchronise the whole device, and some hosts
own the GPU memory budget through their own allocator), so it keeps its path
state in one static device array instead. Both entries run the same kernels on
the same samples, so their radiance must agree exactly (the tolerance the trace
tests use for a path that replays the same random numbers: bit equality).
This file is collected last so that a failure here comes after every other test.
"""
import numpy as np
import pytest

from mupsi_b200 import scene as S
from mupsi_b200.api import GpuScene
from mupsi_b200.lib import MupsiError

pytestmark = pytest.mark.gpu


def _samples(w, h, passes, k0=0):
    xs, ys, ks = np.meshgrid(np.arange(w), np.arange(h), np.arange(k0, k0 + passes), indexing="ij")
    return [a.ravel().astype(np.int32) for a in (xs, ys, ks)]


def test_noalloc_matches_trace_samples_twice(gpu):
    import torch
    gs = GpuScene(S.config0_scene(48, 48, 8))
    # two calls in a row with different samples: the shared scratch must not leak state
    for k0, passes in ((0, 4), (4, 3)):
        xs, ys, ks = _samples(48, 48, passes, k0)
        ref = gs.trace(xs, ys, ks)
        dx, dy, dk = (torch.from_numpy(a).cuda() for a in (xs, ys, ks))
        out = torch.full((len(xs), 3), -1.0, dtype=torch.float32, device="cuda")
        gs.trace_noalloc(dx, dy, dk, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
        assert (ref[:, 0] < 1).sum() > 50  # the GP surface is in view


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
