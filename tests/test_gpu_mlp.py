"""The surrogate MLP's tensor-core kernels (mupsi_gpu_mlp_*) against the CPU
oracle (FP64 with the same BF16 rounding points): inference, the fused
forward+backward gradient, and training to a known signed distance."""
import numpy as np
import pytest

from mupsi_b200 import surrogate as SG

pytestmark = pytest.mark.gpu

CENTER = np.array([0.0, 0.0, -300.0], np.float32)


def case(seed, n):
    rng = np.random.default_rng(seed)
    params = SG.init_params(seed)
    for k in ("b1", "b2", "b3", "b4"):
        o = SG.OFFSETS[k]
        params[o:o + 64] = rng.normal(0, 0.05, 64)
    params[SG.OFFSETS["b5"]] = 0.3
    fourier = SG.fourier_matrix(seed)
    p = (CENTER + rng.uniform(-110, 110, (n, 3))).astype(np.float32)
    t = (np.linalg.norm(p - CENTER, axis=1) - 60.0).astype(np.float32)
    return params, fourier, p, t


@pytest.mark.parametrize("n", [1, 128, 1000, 40000])
def test_infer_matches_oracle(gpu, port, n):
    params, fourier, p, _ = case(1, n)
    sm = SG.SurrogateMean(CENTER, 32.0, params, fourier)
    got = sm.infer(p)
    ref = port.mlp_forward(params, fourier, CENTER, 32.0, p)
    scale = np.abs(ref).max() + 1e-6
    err = np.abs(got - ref)
    assert err.max() <= 1e-2 * scale, err.max() / scale
    assert np.mean(err <= 1e-4 * scale) >= 0.9
    sm.close()


def test_infer_device_buffers(gpu):
    import torch
    params, fourier, p, _ = case(2, 5000)
    sm = SG.SurrogateMean(CENTER, 32.0, params, fourier)
    host = sm.infer(p)
    dev = sm.infer(torch.tensor(p, device="cuda"))
    assert np.array_equal(host, dev.cpu().numpy())


@pytest.mark.parametrize("n", [77, 1000, 20000])
def test_gradient_matches_oracle(gpu, port, n):
    params, fourier, p, t = case(3, n)
    sm = SG.SurrogateMean(CENTER, 32.0, params, fourier)
    g, loss = sm.grad(p, t)
    ref, ref_loss = port.mlp_grad(params, fourier, CENTER, 32.0, p, t)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for name, (a, b) in {"W1": (0, 6144), "b1": (6144, 6208), "W2": (6208, 10304), "b2": (10304, 10368),
                         "W3": (10368, 14464), "W4": (14528, 18624), "b4": (18624, 18688), "w5": (18688, 18752),
                         "b5": (18752, 18753)}.items():
        err = np.abs(g[a:b] - ref[a:b]).max()
        assert err <= 1e-2 * np.abs(ref[a:b]).max() + 1e-9, (name, err, np.abs(ref[a:b]).max())
    sm.close()


def test_training_fits_a_signed_distance(gpu):
    rng = np.random.default_rng(5)
    p = (CENTER + rng.uniform(-110, 110, (1 << 18, 3))).astype(np.float32)
    t = (np.linalg.norm(p - CENTER, axis=1) - 60.0).astype(np.float32)
    sm = SG.SurrogateMean(CENTER, 32.0, seed=5)
    losses = sm.train(p, t, steps=2000, batch=16384, lr=3e-3, lr_final=1e-5, seed=1)
    q = (CENTER + rng.uniform(-100, 100, (20000, 3))).astype(np.float32)
    err = np.abs(sm.infer(q) - (np.linalg.norm(q - CENTER, axis=1) - 60.0))
    print("loss", losses[:3], losses[-3:], "held-out mean/max error", err.mean(), err.max())
    assert losses[-50:].mean() < 0.002 * losses[:5].mean(), (losses[:5], losses[-5:])
    assert err.mean() < 1.0 and err.max() < 6.0, (err.mean(), err.max())
    sm.close()
