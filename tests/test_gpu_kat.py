"""Known-answer tests of the integer primitives on the GPU, bit for bit.

make_seed (math/random.h:13-25), the PCG32 Random streams and next1D
(random.h:73-119), ConstantSampler::nextI (math/sampler.h:47-54) and the
truncating grid cell of SparseGPNoiseGenerator::InternalNoise with its per-cell
seeds, impulse positions and weights (gp/gpnoise.cpp:51-87) are compared with
the reference's own outputs (tests/golden/random.npz, psi fixtures) and with the
C restatement on negative, zero, cell-boundary and wrap-around inputs. These
run through the probe entries of the C ABI, which call the same device
routines the psi and trace kernels use."""
import ctypes as C

import numpy as np
import pytest

from oracle import bind
from mupsi_b200 import _abi
from mupsi_b200.lib import check, load

pytestmark = pytest.mark.gpu
HOST = _abi.MEM_HOST


def _p(a):
    return a.ctypes.data


def gpu_make_seed(args):
    args = np.ascontiguousarray(args, np.uint32)
    out = np.zeros(len(args), np.uint32)
    check(load().mupsi_gpu_probe_make_seed(len(args), args.shape[1], _p(args), _p(out), HOST, None))
    return out


def gpu_random(seeds, draws):
    seeds = np.ascontiguousarray(seeds, np.uint64)
    n = len(seeds)
    u = np.zeros((n, draws), np.uint32)
    f = np.zeros((n, draws), np.float32)
    cs = np.zeros(n, np.uint32)
    check(load().mupsi_gpu_probe_random(n, _p(seeds), draws, _p(u), _p(f), _p(cs), HOST, None))
    return u, f, cs


def gpu_impulses(kernel, p, seed):
    p = np.ascontiguousarray(p, np.float32)
    seed = np.ascontiguousarray(seed, np.uint32)
    n, ppc = len(p), kernel.points_per_cell
    cells = np.zeros((n, 27, 3), np.int32)
    cs = np.zeros((n, 27), np.uint32)
    s = np.zeros((n, 27 * ppc, 3), np.float32)
    w = np.zeros((n, 27 * ppc), np.float32)
    check(load().mupsi_gpu_probe_impulses(C.byref(kernel), n, _p(p), _p(seed), _p(cells), _p(cs), _p(s), _p(w),
                                          HOST, None))
    return s, w, cells, cs


def _edge_u32(rng, n):
    """Random u32 words mixed with the edge values of the hash's arithmetic."""
    edge = np.array([0, 1, 2, 0x7FFFFFFF, 0x80000000, 0xFFFFFFFF, 0xFFFFFFFE, 0x9E3779B9, 42], np.uint32)
    a = rng.integers(0, 2**32, (n, 5), dtype=np.uint64).astype(np.uint32)
    a[: len(edge) * 5].flat[:] = np.resize(edge, len(edge) * 5)
    return a


def test_make_seed_golden_and_edges(gpu, port, golden):
    g = golden("random.npz")
    args = np.asarray(g["seed_args"], np.int64).astype(np.uint32)
    assert np.array_equal(gpu_make_seed(args[:, :4]), np.asarray(g["seed4"], np.uint32))
    assert np.array_equal(gpu_make_seed(args), np.asarray(g["seed5"], np.uint32))
    rng = np.random.default_rng(11)
    a = _edge_u32(rng, 4096)
    # the integer casts of negative cell indices and pixel coordinates
    a[100:200, :3] = rng.integers(-(2**31), 0, (100, 3)).astype(np.int64).astype(np.uint32)
    ref4 = np.array([port.make_seed4(*map(int, r[:4])) for r in a], np.uint32)
    ref5 = np.array([port.make_seed5(*map(int, r)) for r in a], np.uint32)
    assert np.array_equal(gpu_make_seed(a[:, :4]), ref4)
    assert np.array_equal(gpu_make_seed(a), ref5)


def test_random_streams_golden_and_edges(gpu, port, golden):
    g = golden("random.npz")
    seeds = np.asarray(g["rng_seeds"], np.uint64)
    u, f, _ = gpu_random(seeds, g["rng_u32"].shape[1])
    assert np.array_equal(u, g["rng_u32"]) and np.array_equal(f.view(np.uint32), g["rng_f32"].view(np.uint32))
    _, _, cs = gpu_random(np.asarray(g["cs_seeds"], np.uint64), 0)
    assert np.array_equal(cs, np.asarray(g["cs_i"], np.uint32))
    # zero seed (becomes 1), high bits, all ones; 64 draws cover every rotation
    edge = [0, 1, 2, 42, 2**31, 2**32 - 1, 2**32, 2**63, 2**64 - 1, 0x9E3779B97F4A7C15]
    seeds = np.array(edge + list(np.random.default_rng(3).integers(0, 2**63, 54, dtype=np.uint64)), np.uint64)
    u, f, cs = gpu_random(seeds, 64)
    for i, s in enumerate(seeds):
        pu, pf = port.random_stream(int(s), 64)
        assert np.array_equal(u[i], pu) and np.array_equal(f[i].view(np.uint32), pf.view(np.uint32)), int(s)
        assert cs[i] == port.constant_sampler(int(s) & 0xFFFFFFFF)[2]
    assert np.all((f >= 0) & (f < 1))


@pytest.mark.parametrize("kr,ppc", [(1.0, 3), (0.5, 1), (4.0, 8), (0.3, 3), (3.0, 2)])
def test_grid_cells_and_impulses(gpu, port, kr, ppc):
    """Cells by truncation toward zero (not floor) at cell boundaries, at +-0 and
    tiny values of both signs, for power-of-two and other cell sizes; 1, 3 and 8
    impulses per cell take the unrolled cells whose PCG states are jumped ahead
    from the cell seed, 2 the stepped loop."""
    rng = np.random.default_rng(int(kr * 10) + ppc)
    n = 96
    p = rng.uniform(-150, 150, (n, 3)).astype(np.float32)
    p[:16] = (np.round(p[:16] / kr) * kr).astype(np.float32)              # on cell boundaries
    p[16:24] = np.nextafter(p[:8], np.float32(np.inf)).astype(np.float32)  # one ulp either side
    p[24:32] = np.nextafter(p[:8], np.float32(-np.inf)).astype(np.float32)
    p[32:48] = (rng.uniform(-1, 1, (16, 3)) * kr * 0.999).astype(np.float32)  # cell 0 from both sides
    p[48] = np.float32(-0.0)
    p[49] = np.array([-1e-30, 1e-30, -kr], np.float32)
    p[50] = np.array([1e6, -1e6, 3e4], np.float32)
    seed = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    seed[:4] = [0, 1, 0xFFFFFFFF, 42]
    k = bind.kernel_struct(1.0, kr, (1, 1, 1), ppc)
    s, w, cells, cs = gpu_impulses(k, p, seed)
    for i in range(n):
        rs, rw, rcells, rcs = port.psi_impulses(k, p[i], int(seed[i]))
        assert np.array_equal(cells[i], rcells), i
        assert np.array_equal(cs[i], rcs), i
        assert np.array_equal(s[i].view(np.uint32), rs.view(np.uint32)), i
        assert np.array_equal(w[i], rw), i
    # truncation toward zero: the cell of a small negative coordinate is 0
    assert np.all(cells[32:48, 13] == np.trunc(p[32:48] / np.float32(kr)).astype(np.int32))
