"""Learned warm start of the corrector solve: a U-Net (libnlf.so, tensor-core BF16 convolutions) predicts the 6
unit-strain correctors of a density cell, and the prediction is the u0 of `LinearHomogenization.C_full` /
`solve` (nlfiber/linear.py:209-212 and :231-236 take u0; the reference always passes zeros). PCG then runs to
the same tolerance from that start, so the network only changes the iteration count, never the converged C.

Tensors are torch CUDA tensors throughout (the library takes device pointers); the network's 18 output channels
are u (6 cases x 3 components, case-major) divided by nx, channels-last.
"""
import ctypes

import numpy as np

from ._lib import check, lib, ptr

OUT = 18


def _torch():
    import torch
    return torch


class UNet:
    """The warm-start network (architecture in include/nlf.h and oracle/unet_ref.py)."""

    def __init__(self, widths=(16, 32, 64), seed=0):
        h = ctypes.c_void_p()
        check(lib.nlf_unet_create(ctypes.byref(h), *(int(w) for w in widths), int(seed)))
        self._h = h
        self._lib = lib
        self.widths = tuple(int(w) for w in widths)
        self.n_params = int(lib.nlf_unet_param_count(h))
        self.stream = None

    def __del__(self):
        h = getattr(self, "_h", None)
        lb = getattr(self, "_lib", None)  # the module global may be gone while the interpreter shuts down
        if h is not None and h.value and lb is not None:
            lb.nlf_unet_destroy(h)
            self._h = None

    def get_params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        check(lib.nlf_unet_get_params(self._h, p.ctypes.data, self.stream))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(np.asarray(p, dtype=np.float32))
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.size}")
        check(lib.nlf_unet_set_params(self._h, p.ctypes.data, self.stream))

    @staticmethod
    def _f32(a):
        torch = _torch()
        if not (torch.is_tensor(a) and a.is_cuda):
            a = torch.as_tensor(np.asarray(a), device="cuda")
        return a.to(torch.float32).contiguous()

    def forward(self, rho):
        """rho (nb, nx, ny, nz) -> y (nb, nx, ny, nz, 18), CUDA float32."""
        torch = _torch()
        rho = self._f32(rho)
        nb, nx, ny, nz = rho.shape
        y = torch.empty((nb, nx, ny, nz, OUT), dtype=torch.float32, device=rho.device)
        check(lib.nlf_unet_forward(self._h, nb, nx, ny, nz, ptr(rho), ptr(y), self.stream))
        return y

    def loss_grad(self, rho, target, weight, want_grad=False):
        """(loss, gradient or None) of sum_v weight[v] sum_c (y - target)^2 / 18; the gradient is kept for
        adam_step."""
        rho, target, weight = self._f32(rho), self._f32(target), self._f32(weight)
        nb, nx, ny, nz = rho.shape
        loss = ctypes.c_double()
        g = np.empty(self.n_params, dtype=np.float32) if want_grad else None
        check(lib.nlf_unet_backward(self._h, nb, nx, ny, nz, ptr(rho), ptr(target), ptr(weight),
                                    ctypes.byref(loss), None if g is None else g.ctypes.data, self.stream))
        return loss.value, g

    def adam_step(self, lr, betas=(0.9, 0.999), eps=1e-8):
        check(lib.nlf_unet_adam_step(self._h, float(lr), float(betas[0]), float(betas[1]), float(eps),
                                     self.stream))


def corrector_channels(u, nx=None):
    """u (ncell, 6, nx, ny, nz, 3) -> (ncell, nx, ny, nz, 18) float32 = u / nx (the network's targets)."""
    torch = _torch()
    u = torch.as_tensor(u)
    nx = u.shape[2] if nx is None else nx
    return (u.permute(0, 2, 3, 4, 1, 5).reshape(u.shape[0], *u.shape[2:5], OUT) / nx).to(torch.float32).contiguous()


def corrector_fields(y):
    """(ncell, nx, ny, nz, 18) -> u0 (ncell, 6, nx, ny, nz, 3) float64, the inverse of corrector_channels."""
    torch = _torch()
    n, nx, ny, nz, _ = y.shape
    return (y.reshape(n, nx, ny, nz, 6, 3).permute(0, 4, 1, 2, 3, 5) * nx).to(torch.float64).contiguous()


def loss_weights(rho, emin, p=3.0):
    """Per-voxel weights of the loss: the stiffness scale s(rho) (nlfiber/linear.py:137-141), so that void
    voxels, whose displacement does not enter C, do not steer the fit. Unnormalised."""
    torch = _torch()
    rho = torch.as_tensor(rho)
    return (emin + (1.0 - emin) * rho.clamp(0.0, 1.0) ** p).to(torch.float32)


def train(net, rho, target, weight, steps, batch=4, lr=2e-3, lr_end=None, seed=0):
    """Adam on random mini-batches of (rho, target, weight) (CUDA tensors, leading dimension = cells), the
    weights normalised to sum 1 per batch; cosine decay from lr to lr_end (default lr / 20). Returns the
    per-step losses."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    n = rho.shape[0]
    lr_end = lr / 20 if lr_end is None else lr_end
    losses = []
    for it in range(steps):
        idx = torch.as_tensor(rng.choice(n, size=min(batch, n), replace=False), device=rho.device)
        w = weight[idx]
        w = w / w.sum()
        loss, _ = net.loss_grad(rho[idx], target[idx], w)
        a = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * it / max(steps - 1, 1)))
        net.adam_step(a)
        losses.append(loss)
    return losses


class WarmStart:
    """u0 for LinearHomogenization.C_full_batched from the network's prediction."""

    def __init__(self, net):
        self.net = net

    def u0(self, rho):
        """rho (ncell, nx, ny, nz) -> u0 (ncell, 6, nx, ny, nz, 3), CUDA float64."""
        return corrector_fields(self.net.forward(rho))
