"""Learned surrogate for a mesh mean (no reference counterpart).

A Fourier-feature MLP mu_hat(p) (include/mupsi_gpu.h, mupsi_mlp_desc) trained on
exact signed distances that the GPU's own BVH mean produces, for a scene's
mesh-mean medium, so that a march can skip steps far from the surface without
a BVH closest-point query. The exact BVH mean stays in use inside the band
|mu_hat| <= band, at conditioning points and for every hit.

Everything here drives the C ABI (libmupsi_gpu.so): the network's forward,
backward and Adam kernels run on the GPU.
"""
import ctypes as C

import numpy as np

from . import _abi
from .api import check_buf
from .lib import check, load

PARAMS = 18753
FREQS = 48
HIDDEN = 64
FEATURES = 2 * FREQS
# offsets of the parameter vector: W1[64][96], b1, (W_l[64][64], b_l) x 3, w5[64], b5
OFFSETS = {"W1": 0, "b1": 6144, "W2": 6208, "b2": 10304, "W3": 10368, "b3": 14464, "W4": 14528, "b4": 18624,
           "w5": 18688, "b5": 18752}


def init_params(seed=0):
    """He-uniform weights for the ReLU layers, small output layer, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)

    def he(fan_in, n):
        lim = np.sqrt(6.0 / fan_in)
        return rng.uniform(-lim, lim, n).astype(np.float32)

    p[0:6144] = he(FEATURES, 6144)
    for l in range(3):
        o = 6208 + l * 4160
        p[o:o + 4096] = he(HIDDEN, 4096)
    p[18688:18752] = rng.uniform(-np.sqrt(3.0 / HIDDEN), np.sqrt(3.0 / HIDDEN), 64).astype(np.float32)
    return p


def fourier_matrix(seed=0, sigma=1.0 / 20.0):
    """B (48 x 3), entries N(0, sigma^2): angular frequencies in radians per
    scene unit, features sin/cos(B (p - center))."""
    rng = np.random.default_rng(seed + 7919)
    return (rng.normal(size=(FREQS, 3)) * sigma).astype(np.float32)


class MlpDesc(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("y_scale", C.c_float), ("fourier", C.c_float * (FREQS * 3)),
                ("params", C.POINTER(C.c_float))]


class TrainArgs(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("lr_final", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64)]


def _dev(a):
    try:
        import torch
        return isinstance(a, torch.Tensor) and a.is_cuda
    except Exception:  # pragma: no cover
        return False


def _ptr(a):
    return a.data_ptr() if _dev(a) else a.ctypes.data


def _stream():
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.current_stream().cuda_stream
    except Exception:  # pragma: no cover
        pass
    return None


class SurrogateMean:
    """The network on the device (mupsi_gpu_mlp_*)."""

    def __init__(self, center, y_scale=32.0, params=None, fourier=None, seed=0):
        self.center = np.asarray(center, np.float32)
        self.y_scale = float(y_scale)
        self.fourier = fourier_matrix(seed) if fourier is None else np.ascontiguousarray(fourier, np.float32)
        init = init_params(seed) if params is None else np.ascontiguousarray(params, np.float32)
        d = MlpDesc()
        d.center[:] = [float(v) for v in self.center]
        d.y_scale = self.y_scale
        d.fourier[:] = [float(v) for v in self.fourier.ravel()]
        d.params = init.ctypes.data_as(C.POINTER(C.c_float))
        h = C.c_void_p()
        check(load().mupsi_gpu_mlp_create(C.addressof(d), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            load().mupsi_gpu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(PARAMS, np.float32)
        check(load().mupsi_gpu_mlp_get_params(self.h, out.ctypes.data))
        return out

    def infer(self, p, out=None):
        """mu_hat at points p (n, 3): numpy (host) or CUDA tensor (device)."""
        dev = _dev(p)
        n = p.shape[0]
        if tuple(p.shape) != (n, 3):
            raise ValueError("p must be (n, 3)")
        if out is None:
            if dev:
                import torch
                out = torch.empty(n, dtype=torch.float32, device=p.device)
            else:
                out = np.empty(n, np.float32)
        if not dev:
            p = np.ascontiguousarray(p, np.float32)
        check_buf(out, (n,))
        check(load().mupsi_gpu_mlp_infer(self.h, n, _ptr(p), _ptr(out), _abi.MEM_DEVICE if dev else _abi.MEM_HOST,
                                         _stream()))
        return out

    def grad(self, p, target):
        """(dL/dparams float32, L) over the points, from the GPU backward kernels."""
        dev = _dev(p)
        if not dev:
            p = np.ascontiguousarray(p, np.float32)
            target = np.ascontiguousarray(target, np.float32)
        _points_targets(p, target)
        g = np.zeros(PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        check(load().mupsi_gpu_mlp_grad(self.h, p.shape[0], _ptr(p), _ptr(target), g.ctypes.data, loss.ctypes.data,
                                        _abi.MEM_DEVICE if dev else _abi.MEM_HOST, _stream()))
        return g, float(loss[0])

    def train(self, p, target, steps=2000, batch=16384, lr=3e-3, lr_final=1e-4, betas=(0.9, 0.999), eps=1e-8,
              seed=0):
        """Adam on minibatches drawn from (p, target); returns the per-step losses."""
        dev = _dev(p)
        if not dev:
            p = np.ascontiguousarray(p, np.float32)
            target = np.ascontiguousarray(target, np.float32)
        _points_targets(p, target)
        a = TrainArgs(steps, batch, lr, lr_final, betas[0], betas[1], eps, seed)
        losses = np.zeros(steps, np.float32)
        check(load().mupsi_gpu_mlp_train(self.h, p.shape[0], _ptr(p), _ptr(target), C.addressof(a),
                                         losses.ctypes.data, _abi.MEM_DEVICE if dev else _abi.MEM_HOST, _stream()))
        return losses


def _points_targets(p, target):
    """The library reads n points (n, 3) and n targets (n,)."""
    n = p.shape[0]
    if tuple(p.shape) != (n, 3) or tuple(target.shape) != (n,):
        raise ValueError("need points (n, 3) and targets (n,)")


def training_points(vertices, faces, n, box_lo, box_hi, seed=0, normal_sigma=2.0):
    """n points: half uniform in the box [box_lo, box_hi], half on the surface
    (area-weighted triangle, uniform barycentric) moved along the face normal by
    N(0, normal_sigma^2)."""
    rng = np.random.default_rng(seed)
    v = np.asarray(vertices, np.float64)
    f = np.asarray(faces, np.int64)
    n_box = n // 2
    n_surf = n - n_box
    lo, hi = np.asarray(box_lo, np.float64), np.asarray(box_hi, np.float64)
    box = lo + (hi - lo) * rng.random((n_box, 3))
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    cr = np.cross(b - a, c - a)
    area = np.linalg.norm(cr, axis=1)
    tri = rng.choice(len(f), size=n_surf, p=area / area.sum())
    r1, r2 = rng.random(n_surf), rng.random(n_surf)
    s = np.sqrt(r1)
    u, w = 1.0 - s, s * (1.0 - r2)
    pts = u[:, None] * a[tri] + w[:, None] * b[tri] + (s * r2)[:, None] * c[tri]
    nrm = cr[tri] / np.maximum(area[tri], 1e-30)[:, None]
    pts += nrm * rng.normal(0.0, normal_sigma, n_surf)[:, None]
    out = np.concatenate([box, pts]).astype(np.float32)
    return out[rng.permutation(n)]


def attach(gpu_scene, medium, surrogate, band=3.0, scale=1.5, margin=1.0, max_requests=8):
    """Let gpu_scene's marches use `surrogate` for medium `medium` (None
    detaches): a prediction m with |m| > band gives |m|/scale - margin <= |mu|."""
    check(load().mupsi_gpu_scene_set_surrogate(gpu_scene.h, medium, surrogate.h if surrogate else None, band, scale,
                                               margin, max_requests))
    gpu_scene._surrogate = surrogate


def bound_margin(pred, exact, band=3.0, scale=1.5, safety=2.0):
    """Margin for attach(): `safety` x the largest violation of |mu| >= |m|/scale
    over held-out points with |m| > band (or a wrong sign there), at least 0.5."""
    pred = np.asarray(pred, np.float64)
    exact = np.asarray(exact, np.float64)
    far = np.abs(pred) > band
    if not far.any():
        return 0.5
    viol = np.abs(pred[far]) / scale - np.abs(exact[far])
    viol = np.where(np.sign(pred[far]) != np.sign(exact[far]), np.abs(pred[far]) / scale, viol)
    return float(max(0.5, safety * max(0.0, viol.max())))
