"""psi / grad psi / conditioned psi on the GPU against the CPU oracle and the
reference's own outputs (tests/golden/psi_sweep.npz).

Tolerance (stated): |gpu - ref| <= 1e-5 * (|ref| + S), where S is the sum of
the absolute values of the terms of that output (sigma/sqrt(Var) * sum |w h|
for psi, the same for each gradient component). S is the scale of the
rounding error of any FP32 evaluation of the sum; the test also reports the
error of both FP32 results against the FP64 sum of the same impulses."""
import numpy as np
import pytest

from oracle import bind
from mupsi_b200.api import SparseGPNoiseGenerator, SparseSEKernel

pytestmark = pytest.mark.gpu
REL = 1e-5
SWEEP = [(L, az, ppc) for L in (0.5, 1.0, 4.0) for az in (1.0, 4.0) for ppc in (1, 3, 8)]


def _inputs(rng, n):
    p = rng.uniform(-150, 150, (n, 3)).astype(np.float32)
    s = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    return p, s


def _cond(rng, p, L):
    n = len(p)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    c = np.zeros((n, 8), np.float32)
    c[:, :3] = p + d * rng.uniform(0, 3 * L, (n, 1))
    c[:, 3] = rng.normal(size=n)
    g = rng.normal(size=(n, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    c[:, 4:7] = g * rng.normal(size=(n, 1))
    c[:, 7] = 1
    return c


@pytest.mark.parametrize("L,az,ppc", SWEEP)
def test_psi_sweep(gpu, port, L, az, ppc):
    rng = np.random.default_rng(int(L * 100 + az * 10 + ppc))
    p, s = _inputs(rng, 4096)
    p[:64] = (np.round(p[:64] / L) * L).astype(np.float32)  # cell boundaries
    p[64:128] *= np.float32(1e-3)                            # near the origin, both signs
    k = bind.kernel_struct(1.0, L, (1, 1, az), ppc)
    gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, L, (1, 1, az)), ppc)
    got = gen.raw_noise(p, s)
    ref = port.psi(k, p, s)
    f64, scale = port.psi_f64(k, p, s)
    err = np.abs(got.astype(np.float64) - ref)
    tol = REL * (np.abs(ref) + scale)
    assert np.all(err <= tol), f"max err/tol {np.max(err / tol):.3g}"
    # FP32 error of both evaluations against the FP64 sum, relative to the term scale
    e_gpu = np.max(np.abs(got - f64) / scale)
    e_ref = np.max(np.abs(ref - f64) / scale)
    assert e_gpu < 1e-5 and e_ref < 1e-5
    # value-only entry is the same sum
    v = gen.raw_noise_value(p, s)
    assert np.all(np.abs(v - ref[:, 0]) <= tol[:, 0])


@pytest.mark.parametrize("L,az,ppc", [(0.5, 1.0, 3), (1.0, 1.0, 3), (4.0, 4.0, 8)])
def test_psi_conditioned(gpu, port, L, az, ppc):
    rng = np.random.default_rng(7)
    p, s = _inputs(rng, 4096)
    c = _cond(rng, p, L)
    c[::3, 7] = 0  # mixed active/inactive
    k = bind.kernel_struct(1.0, L, (1, 1, az), ppc)
    gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, L, (1, 1, az)), ppc)
    got = gen.raw_noise(p, s, cond=c)
    ref = port.psi(k, p, s, cond=c)
    _, scale = port.psi_f64(k, p, s)
    cscale = np.abs(c[:, 3:4]) + np.linalg.norm(c[:, 4:7], axis=1, keepdims=True) * 4.0 / L
    tol = REL * (np.abs(ref) + scale + cscale)
    assert np.all(np.abs(got - ref) <= tol)
    v = gen.raw_noise_value(p, s, cond=c)
    assert np.all(np.abs(v - ref[:, 0]) <= tol[:, 0])


def test_psi_against_reference_fixtures(gpu, golden):
    g = golden("psi_sweep.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    for key in keys:
        L = float(key.split("_")[0][1:])
        az = float(key.split("_")[1][1:])
        ppc = int(key.split("_")[2][1:])
        gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, L, (1, 1, az)), ppc)
        got = gen.raw_noise(g[key + "_p"], g[key + "_seed"])
        ref = g[key + "_psi"]
        # scale bound: |terms| <= 1 each, so S <= 27 ppc sigma/sqrt(Var)
        var = np.float32((ppc / L**3) * np.pi**1.5)
        smax = 27 * ppc / np.sqrt(var) * (1 + 4 * 2.0 / L)
        assert np.all(np.abs(got - ref) <= REL * (np.abs(ref) + smax)), key


def test_psi_device_buffers(gpu, port):
    import torch
    rng = np.random.default_rng(3)
    p, s = _inputs(rng, 1000)
    gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, 1.0), 3)
    host = gen.raw_noise(p, s)
    dev = gen.raw_noise(torch.from_numpy(p).cuda(), torch.from_numpy(s.view(np.int32)).cuda())
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))


def test_psi_empty_and_invalid(gpu):
    from mupsi_b200.lib import MupsiError
    gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, 1.0), 3)
    assert gen.raw_noise(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32)).shape == (0, 4)
    bad = SparseGPNoiseGenerator(SparseSEKernel(1.0, 0.0), 3)
    with pytest.raises(MupsiError):
        bad.raw_noise(np.zeros((4, 3), np.float32), np.zeros(4, np.uint32))
