"""The surrogate MLP's CPU oracle (FP64 with the GPU's BF16 rounding points)
against an independent torch-CPU FP64 autograd of the same network, and the
oracle's gradient against central finite differences of its own loss."""
import numpy as np
import torch

from mupsi_b200 import surrogate as SG


def torch_net(params, fourier, center, y_scale, p, bf16=True):
    """The network of include/mupsi_gpu.h in torch float64. With bf16, operands
    are rounded where the GPU stores BF16 (straight-through in the backward)."""
    def rnd(x):
        if not bf16:
            return x
        r = x.float().to(torch.bfloat16).double()
        return x + (r - x).detach()

    P = params
    x = torch.tensor(p, dtype=torch.float64) - torch.tensor(center, dtype=torch.float64)
    u = x @ torch.tensor(fourier, dtype=torch.float64).T
    h = rnd(torch.cat([torch.sin(u), torch.cos(u)], dim=1))
    o = SG.OFFSETS
    for w, b, k in [("W1", "b1", 96), ("W2", "b2", 64), ("W3", "b3", 64), ("W4", "b4", 64)]:
        W = rnd(P[o[w]:o[w] + 64 * k].view(64, k))
        h = rnd(torch.relu(h @ W.T + P[o[b]:o[b] + 64]))
    y = h @ rnd(P[o["w5"]:o["w5"] + 64]) + P[o["b5"]]
    return y * y_scale


def setup(n=64, seed=3):
    rng = np.random.default_rng(seed)
    params = SG.init_params(seed)
    params[SG.OFFSETS["b1"]:SG.OFFSETS["b1"] + 64] = rng.normal(0, 0.1, 64)
    fourier = SG.fourier_matrix(seed)
    center = np.array([0.0, 0.0, -300.0], np.float32)
    p = (center + rng.uniform(-100, 100, (n, 3))).astype(np.float32)
    target = rng.normal(0, 20, n).astype(np.float32)
    return params, fourier, center, 32.0, p, target


def test_forward_matches_torch(port):
    params, fourier, center, ys, p, _ = setup()
    got = port.mlp_forward(params, fourier, center, ys, p)
    ref = torch_net(torch.tensor(params, dtype=torch.float64), fourier, center, ys, p).numpy()
    assert np.allclose(got, ref, rtol=2e-3, atol=2e-3 * np.abs(ref).max())
    exact = torch_net(torch.tensor(params, dtype=torch.float64), fourier, center, ys, p, bf16=False).numpy()
    # BF16 rounding moves the output by a few percent of its range at most
    assert np.abs(got - exact).max() < 0.05 * np.abs(exact).max()


def test_gradient_matches_torch_autograd(port):
    params, fourier, center, ys, p, target = setup()
    g, loss = port.mlp_grad(params, fourier, center, ys, p, target)
    P = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    y = torch_net(P, fourier, center, ys, p) / ys
    L = ((y - torch.tensor(target, dtype=torch.float64) / ys) ** 2).mean()
    L.backward()
    ref = P.grad.numpy()
    assert abs(loss - L.item()) <= 1e-3 * L.item()
    for name, (a, b) in {"W1": (0, 6144), "b1": (6144, 6208), "W2": (6208, 10304), "W4": (14528, 18624),
                         "w5": (18688, 18752), "b5": (18752, 18753)}.items():
        err = np.abs(g[a:b] - ref[a:b]).max()
        assert err <= 2e-2 * np.abs(ref[a:b]).max() + 1e-9, (name, err, np.abs(ref[a:b]).max())


def test_gradient_finite_differences(port):
    """Central differences of the oracle's own loss on the output bias, the one
    parameter no BF16 rounding follows (elsewhere the loss is a staircase at
    the BF16 steps and the autograd comparison above applies)."""
    params, fourier, center, ys, p, target = setup(n=32)
    g, _ = port.mlp_grad(params, fourier, center, ys, p, target)
    i = SG.OFFSETS["b5"]
    h = 1e-3
    up, dn = params.copy(), params.copy()
    up[i] += h
    dn[i] -= h
    _, lu = port.mlp_grad(up, fourier, center, ys, p, target)
    _, ld = port.mlp_grad(dn, fourier, center, ys, p, target)
    fd = (lu - ld) / (2 * h)
    assert abs(fd - g[i]) <= 5e-3 * max(abs(fd), 1e-6) + 1e-7, (fd, g[i])
