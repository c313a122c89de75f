"""Learned per-element reluctivity warm start (no counterpart in the reference).

A small MLP predicts, for every nonlinear element, the reluctivity nu_e it will
have at the end of the next time step's Newton solve, from features available
before the solve: |B| at the previous two steps, the source magnitude, and the
material. The prediction only seeds the first Jacobian of the step; plain
spline-based Newton then runs to the same residual tolerance, so a bad
prediction costs iterations, never accuracy.

The network's forward and backward passes are the tensor-core kernels of
libmagasm (mag_mlp_*); this module holds the feature/target normalisation and
the training loop.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

NUM_FEATURES = 4


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of W1[64][4] b1 W2 b2 W3 b3 w4 b4 (float32)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2.0 / 4), (64, 4)), np.zeros(64),
             rng.normal(0, np.sqrt(2.0 / 64), (64, 64)), np.zeros(64),
             rng.normal(0, np.sqrt(2.0 / 64), (64, 64)), np.zeros(64),
             rng.normal(0, np.sqrt(1.0 / 64), 64), np.zeros(1)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


class MLP:
    """Thin handle over the mag_mlp_* entry points."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0):
        self._lib = _lib.lib()
        self.num_params = self._lib.mag_mlp_num_params()
        p = init_params(seed) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters")
        h = C.c_void_p()
        _lib.check(self._lib.mag_mlp_create(p.ctypes.data_as(C.POINTER(C.c_float)), C.byref(h)))
        self._h = h

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params, dtype=np.float32)
        _lib.check(self._lib.mag_mlp_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self._lib.mag_mlp_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def forward(self, feats: torch.Tensor, want_z: bool = False):
        n = feats.shape[0]
        y = torch.empty(n, dtype=torch.float32, device="cuda")
        z = torch.empty((n, 3, 64), dtype=torch.float32, device="cuda") if want_z else None
        _lib.check(self._lib.mag_mlp_forward(self._h, _ptr(feats), n, _ptr(y), _ptr(z), _lib.stream_ptr()))
        return y, z

    def gradient(self, feats, target, loss_scale: float):
        n = feats.shape[0]
        y = torch.empty(n, dtype=torch.float32, device="cuda")
        z = torch.empty((n, 3, 64), dtype=torch.float32, device="cuda")
        g = torch.empty(self.num_params, dtype=torch.float32, device="cuda")
        _lib.check(self._lib.mag_mlp_gradient(self._h, _ptr(feats), _ptr(target), n, C.c_float(loss_scale),
                                              _ptr(y), _ptr(z), _ptr(g), _lib.stream_ptr()))
        return y, g

    def train_step(self, feats, target, lr: float, y=None, z=None):
        n = feats.shape[0]
        y = torch.empty(n, dtype=torch.float32, device="cuda") if y is None else y
        z = torch.empty((n, 3, 64), dtype=torch.float32, device="cuda") if z is None else z
        _lib.check(self._lib.mag_mlp_train_step(self._h, _ptr(feats), _ptr(target), n, C.c_float(lr),
                                                _ptr(y), _ptr(z), _lib.stream_ptr()))
        return y

    def train_epoch(self, feats, target, perm, batch: int, lr: float, xb, tb, y, z, loss=None):
        """One epoch of train_step over minibatches in the order of the device permutation
        perm (int64); the minibatches are gathered on the device (mag_mlp_train_epoch)."""
        _lib.check(self._lib.mag_mlp_train_epoch(self._h, _ptr(feats), _ptr(target), feats.shape[0], _ptr(perm),
                                                 int(batch), C.c_float(lr), _ptr(xb), _ptr(tb), _ptr(y), _ptr(z),
                                                 _ptr(loss), _lib.stream_ptr()))

    def predict_nu(self, feats, rows, nu_out, y_scale, y_shift, nu_min, nu_max):
        n = feats.shape[0]
        _lib.check(self._lib.mag_mlp_predict_nu(self._h, _ptr(feats), n, _ptr(rows), y_scale, y_shift, nu_min,
                                                nu_max, _ptr(nu_out), _lib.stream_ptr()))

    def check(self):
        _lib.check(self._lib.mag_mlp_check(self._h, _lib.stream_ptr()))

    def set_spin_limit(self, polls: int = 0):
        """Polls before a tensor-core completion wait gives up (0: the default bound)."""
        _lib.check(self._lib.mag_mlp_set_spin_limit(self._h, int(polls)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mag_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NuPredictor:
    """Features -> log(nu) regression with input/target standardisation."""

    def __init__(self, seed: int = 0):
        self.mlp = MLP(seed=seed)
        self.x_mean = np.zeros(NUM_FEATURES)
        self.x_std = np.ones(NUM_FEATURES)
        self.y_mean, self.y_std = 0.0, 1.0

    def _norm(self, feats: torch.Tensor) -> torch.Tensor:
        m = torch.as_tensor(self.x_mean, dtype=torch.float32, device=feats.device)
        s = torch.as_tensor(self.x_std, dtype=torch.float32, device=feats.device)
        return ((feats.float() - m) / s).contiguous()

    def fit(self, feats: torch.Tensor, nu: torch.Tensor, epochs: int = 20, batch: int = 8192,
            lr: float = 2e-3, seed: int = 0):
        """Adam on the mean-squared error of standardised log(nu); returns the loss history."""
        x = feats.double()
        self.x_mean = x.mean(0).cpu().numpy()
        self.x_std = np.maximum(x.std(0).cpu().numpy(), 1e-6)
        ly = torch.log(nu.double())
        self.y_mean, self.y_std = float(ly.mean()), max(float(ly.std()), 1e-6)
        xn = self._norm(feats)
        tn = ((ly - self.y_mean) / self.y_std).float().contiguous()
        n = xn.shape[0]
        # permutations drawn on the device, minibatches gathered and the loss summed there:
        # the host only enqueues launches, and the steps run back to back on the GPU
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        batch = min(batch, n)
        ybuf = torch.empty(batch, dtype=torch.float32, device="cuda")
        zbuf = torch.empty((batch, 3, 64), dtype=torch.float32, device="cuda")
        xb = torch.empty((batch, 4), dtype=torch.float32, device="cuda")
        tb = torch.empty(batch, dtype=torch.float32, device="cuda")
        loss = torch.zeros(epochs, dtype=torch.float32, device="cuda")
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device="cuda")
            self.mlp.train_epoch(xn, tn, perm, batch, lr, xb, tb, ybuf, zbuf, loss[ep:ep + 1])
        self.mlp.check()
        # mean squared error per row of each epoch (before each minibatch's step)
        return (loss.double() / ((n // batch) * batch)).tolist()

    def predict_nu(self, feats: torch.Tensor, rows: torch.Tensor, nu_out: torch.Tensor, nu_min: float,
                   nu_max: float):
        """nu_out[rows[i]] = clamp(exp(prediction_i)) on the GPU (no host round trip)."""
        self.mlp.predict_nu(self._norm(feats), rows, nu_out, self.y_std, self.y_mean, nu_min, nu_max)
        return nu_out
