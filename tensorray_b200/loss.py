"""Image losses of the inverse-rendering loop, on the device.

Mirrors pyTensorRay/loss.py:34-83 (names, argument meaning and results):
L1 and L2 image losses with NaN differences zeroed, and their image-pyramid
forms. A pyramid has min(5, floor(log2(min(H, W))) + 1) levels. Each level
halves the previous one with a 2x2 box filter, repeating the last row or
column when a side is odd. Level i's loss is weighted by 4^i. Images are
(H, W, 3) tensors. Everything runs as device tensor operations, so the
loss and its image gradient dL/dI never leave the GPU.
"""
from __future__ import annotations

import math

import torch


def compute_render_loss_L2(img: torch.Tensor, target_img: torch.Tensor, weight: float) -> torch.Tensor:
    """0.5 * sum((img - target)^2) * weight (loss.py:34-38)."""
    diff = (img - target_img).nan_to_num(nan=0.0)
    return 0.5 * diff.square().sum() * weight


def compute_render_loss_L1(img: torch.Tensor, target_img: torch.Tensor, weight: float) -> torch.Tensor:
    """sum(|img - target|) * weight (loss.py:41-46)."""
    diff = (img - target_img).nan_to_num(nan=0.0)
    return diff.abs().sum() * weight


def downsample(img: torch.Tensor) -> torch.Tensor:
    """2x2 box filter; an odd side repeats its last row/column (loss.py:49-54)."""
    if img.shape[0] % 2 == 1:
        img = torch.cat((img, img[-1:]), dim=0)
    if img.shape[1] % 2 == 1:
        img = torch.cat((img, img[:, -1:]), dim=1)
    return (img[0::2, 0::2] + img[1::2, 0::2] + img[0::2, 1::2] + img[1::2, 1::2]) * 0.25


def pyramid_levels(height: int, width: int) -> int:
    return min(5, int(min(math.log2(height), math.log2(width))) + 1)


def build_pyramid(img: torch.Tensor) -> list:
    """The image and its successive 2x2 reductions (loss.py:57-65)."""
    levels = pyramid_levels(img.shape[0], img.shape[1])
    out = []
    for i in range(levels):
        out.append(img)
        if i < levels - 1:
            img = downsample(img)
    return out


def compute_render_loss_pyramid_L1(img: torch.Tensor, target_pyramid: list, weight: float) -> torch.Tensor:
    """sum_i 4^i * L1(level i) (loss.py:68-74)."""
    loss = img.new_zeros(())
    for i, level in enumerate(build_pyramid(img)):
        loss = loss + compute_render_loss_L1(level, target_pyramid[i], weight) * (4.0 ** i)
    return loss


def compute_render_loss_pyramid_L2(img: torch.Tensor, target_pyramid: list, weight: float) -> torch.Tensor:
    """sum_i 4^i * L2(level i) (loss.py:77-83)."""
    loss = img.new_zeros(())
    for i, level in enumerate(build_pyramid(img)):
        loss = loss + compute_render_loss_L2(level, target_pyramid[i], weight) * (4.0 ** i)
    return loss


LOSSES = {"l1": compute_render_loss_L1, "l2": compute_render_loss_L2,
          "pyramid_l1": compute_render_loss_pyramid_L1, "pyramid_l2": compute_render_loss_pyramid_L2}


def loss_and_grad(kind: str, img: torch.Tensor, target, weight: float = 1.0):
    """Loss of one (H, W, 3) image and dL/dI, by torch's reverse mode on the
    device. `target` is an image for "l1"/"l2" and a pyramid
    (build_pyramid(target)) for the pyramid losses."""
    fn = LOSSES[kind]
    x = img.detach().requires_grad_(True)
    with torch.enable_grad():
        loss = fn(x, target, weight)
        (g,) = torch.autograd.grad(loss, x)
    return loss.detach(), g
