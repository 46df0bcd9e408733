"""Image-space losses of the training step and the target smoothing.

``smooth_image`` mirrors GaussianSmoothingGpu.smoothImage
(Projects/CustomTFOperators/GaussianSmoothingGpu.py:12-37);
``image_l1_loss`` the masked L1 of HPCMeshDL.compute_rendering_loss
(Projects/HoloportedCharacters/HPCMeshDL.py:669-688); ``sum_squares_loss``
the reduction applied to the silhouette residuals.  Each returns device
tensors and runs on the current CUDA stream.
"""
from __future__ import annotations

import torch

from . import _lib
from .renderer import _f32, _stream


def smooth_image(image: torch.Tensor, size: int, mean: float, std: float) -> torch.Tensor:
    """Per-channel (2 size + 1)^2 Gaussian blur with zero padding of
    images [..., H, W, C] (C <= 4); size 0 or std 0 returns the input."""
    x = _f32(image, "image")
    if size == 0 or std == 0.0:
        return image
    H, W, Cn = x.shape[-3], x.shape[-2], x.shape[-1]
    n = x.numel() // (H * W * Cn)
    out = torch.empty_like(x)
    _lib.call("hc_gaussian_smooth", _stream(), n, H, W, Cn, int(size), float(mean), float(std), _lib.ptr(x),
              _lib.ptr(out))
    return out


def image_l1_loss(render: torch.Tensor, target: torch.Tensor, face: torch.Tensor, mask: torch.Tensor | None = None):
    """(loss [1], d loss / d render) of sum|255 (R - T)| * mask * (face >= 0) / count_nonzero."""
    r, t = _f32(render, "render"), _f32(target, "target")
    f = face.to(torch.int32).contiguous()
    m = mask.to(torch.uint8).contiguous() if mask is not None else None
    loss = torch.empty((1,), device=r.device)
    grad = torch.empty_like(r)
    ws = torch.empty((2,), device=r.device, dtype=torch.float64)
    _lib.call("hc_image_l1_loss", _stream(), f.numel(), _lib.ptr(r), _lib.ptr(t), _lib.ptr(f), _lib.ptr(m),
              _lib.ptr(ws), _lib.ptr(loss), _lib.ptr(grad))
    return loss, grad


def sum_squares_loss(x: torch.Tensor, weight: float = 1.0):
    """(weight * sum x^2 [1], 2 weight x)."""
    x = _f32(x, "x")
    loss = torch.empty((1,), device=x.device)
    grad = torch.empty_like(x)
    ws = torch.empty((1,), device=x.device, dtype=torch.float64)
    _lib.call("hc_sum_squares_loss", _stream(), x.numel(), _lib.ptr(x), float(weight), _lib.ptr(ws), _lib.ptr(loss),
              _lib.ptr(grad))
    return loss, grad
