"""The multi-GPU host logic on CPU ranks (gloo, world size 2): pass sharding and
the framebuffer all_reduce give the single-process image. Each rank traces its
passes with the CPU oracle (the GPU kernels are covered by the gpu tests)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from mupsi_b200.multigpu import combine, pass_range

W = H = 10
TOTAL = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _trace_avg(k0, k1):
    from oracle import bind
    from mupsi_b200 import scene as S
    port = bind.PortOracle()
    sc = S.config0_scene(W, H, TOTAL)
    h = port.scene_create(sc.desc())
    try:
        xs, ys, ks = (a.ravel().astype(np.int32) for a in np.meshgrid(np.arange(W), np.arange(H), np.arange(k0, k1),
                                                                     indexing="ij"))
        rad = port.trace(h, xs, ys, ks).reshape(W, H, k1 - k0, 3)
    finally:
        port.scene_free(h)
    return rad.astype(np.float64).mean(axis=2)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, e = pass_range(TOTAL, world, rank)
        avg = torch.from_numpy(_trace_avg(b, e))
        img = combine(avg, e - b, TOTAL)
        out[rank] = img.numpy()
    finally:
        dist.destroy_process_group()


def test_pass_range_covers_everything():
    for total in (1, 5, 20, 64):
        for world in (1, 2, 3, 8):
            rs = [pass_range(total, world, r) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == total
            assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
            assert max(e - b for b, e in rs) - min(e - b for b, e in rs) <= 1
    with pytest.raises(ValueError):
        pass_range(4, 2, 2)


def test_two_rank_render_equals_single(port):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    ref = _trace_avg(0, TOTAL)
    for r in range(world):
        assert np.allclose(out[r], ref, rtol=0, atol=1e-12)
    assert (ref[..., 0] < 1).any() and (ref[..., 0] == 1).any()
