"""Residual U-Net corrector of the hybrid rollout.

Layer plan of ``TorchResidualUNet``
(``src/hybrid_flood/benchmark/pytorch_residual_net.py:79-170``, the PyTorch
twin of the Flax ``ml/residual_net.py:43-111``): per level two k×k
convolutions with an activation each; a 2×2 stride-2 convolution (TF ``SAME``
padding) into the next level's width; on the way up a 2×2 stride-2 transposed
convolution, the skip concatenated after it, and two convolutions; a zero-
initialised 1×1 head.  Submodule names equal the reference's so its
``state_dict`` loads unchanged.

On the B200 the network runs in bfloat16 with ``channels_last`` tensors (NHWC
in memory): the feature kernel writes NHWC bfloat16 directly and the correction
kernel reads the bfloat16 NHWC residual in place, so the hand-off around the
convolutions (cuDNN, tensor cores) needs no layout or dtype conversion.  Each
convolution's bias and ReLU run as one in-place pass (``swe_bias_act_nhwc``)
over its channels-last output instead of the framework's broadcast add and a
separate activation pass; other layouts, devices and activations use torch ops.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import torch
import torch.nn.functional as F
from torch import nn

class _BiasAct(torch.autograd.Function):
    """y <- act(y + bias) in place on a CUDA channels-last convolution output."""

    @staticmethod
    def forward(ctx, y, bias, relu):
        from . import _lib

        lib = _lib.load()
        b = bias.detach().to(torch.float32).contiguous()
        rc = lib.swe_bias_act_nhwc(ctypes.c_void_p(y.data_ptr()), y.numel(), y.shape[1], ctypes.c_void_p(b.data_ptr()),
                                   1 if relu else 0, 1 if y.dtype == torch.bfloat16 else 0, y.device.index,
                                   ctypes.c_void_p(torch.cuda.current_stream(y.device).cuda_stream))
        _lib.check(rc, "swe_bias_act_nhwc")
        ctx.mark_dirty(y)
        ctx.relu = relu
        ctx.save_for_backward(y)
        return y

    @staticmethod
    def backward(ctx, g):
        (y,) = ctx.saved_tensors
        if ctx.relu:
            g = g * (y > 0).to(g.dtype)
        return g, g.float().sum(dim=(0, 2, 3)), None


def _fusable(y: torch.Tensor) -> bool:
    return (y.is_cuda and y.dtype in (torch.bfloat16, torch.float32) and y.dim() == 4
            and y.is_contiguous(memory_format=torch.channels_last))


def conv_bias_act(conv: nn.Module, x: torch.Tensor, relu: bool) -> torch.Tensor:
    """``act(conv(x))`` with the bias and ReLU fused into one pass where the layout allows."""
    transposed = isinstance(conv, nn.ConvTranspose2d)
    if transposed:
        y = F.conv_transpose2d(x, conv.weight, None, conv.stride, conv.padding)
    else:
        y = F.conv2d(x, conv.weight, None, conv.stride, conv.padding)
    if conv.bias is not None and _fusable(y):
        return _BiasAct.apply(y, conv.bias, relu)
    if conv.bias is not None:
        y = y + conv.bias.view(1, -1, 1, 1)
    return F.relu(y) if relu else y


_ACTIVATIONS = {
    "relu": lambda: nn.ReLU(),
    "gelu": lambda: nn.GELU(approximate="tanh"),  # Flax's default GELU is the tanh form
    "silu": lambda: nn.SiLU(),
    "tanh": lambda: nn.Tanh(),
}


def make_activation(name: str) -> nn.Module:
    key = name.lower()
    if key not in _ACTIVATIONS:
        raise ValueError(f"Unsupported activation {name!r}; choose one of {sorted(_ACTIVATIONS)}.")
    return _ACTIVATIONS[key]()


# Inference with cuDNN's fused convolution + bias + ReLU (and + add + ReLU):
# used when no gradient is needed, on CUDA channels-last tensors with ReLU.
# SWE_UNET_FUSED=0 keeps the separate bias/activation pass.
_FUSED = {"on": __import__("os").environ.get("SWE_UNET_FUSED", "1") != "0"}


def _fused_ok(x: torch.Tensor) -> bool:
    return (_FUSED["on"] and not torch.is_grad_enabled() and x.is_cuda and x.dim() == 4
            and x.dtype in (torch.bfloat16, torch.float16, torch.float32)
            and x.is_contiguous(memory_format=torch.channels_last))


def _conv_relu(conv: nn.Conv2d, x: torch.Tensor) -> torch.Tensor:
    """relu(conv(x) + bias) in one cuDNN call."""
    return torch.cudnn_convolution_relu(x, conv.weight, conv.bias, list(conv.stride), list(conv.padding),
                                        list(conv.dilation), conv.groups)


class ConvPair(nn.Module):
    """Two same-size k×k convolutions, each followed by the activation."""

    def __init__(self, cin: int, cout: int, k: int, activation: str) -> None:
        super().__init__()
        self.conv_1 = nn.Conv2d(cin, cout, k, padding=k // 2)
        self.activation_1 = make_activation(activation)
        self.conv_2 = nn.Conv2d(cout, cout, k, padding=k // 2)
        self.activation_2 = make_activation(activation)
        self.relu = activation.lower() == "relu"

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        if self.relu and _fused_ok(x):
            return _conv_relu(self.conv_2, _conv_relu(self.conv_1, x))
        if self.relu:
            return conv_bias_act(self.conv_2, conv_bias_act(self.conv_1, x, True), True)
        return self.activation_2(self.conv_2(self.activation_1(self.conv_1(x))))

    def forward_split(self, up: torch.Tensor, skip: torch.Tensor) -> torch.Tensor:
        """forward(cat(up, skip)) without the concatenation: conv_1's weight is split
        along its input channels, conv(up, W_up) is computed first and added,
        with the bias and ReLU, inside the fused convolution over the skip."""
        c = up.shape[1]
        w = self.conv_1.weight
        z = F.conv2d(up, w[:, :c].contiguous(memory_format=torch.channels_last), None, self.conv_1.stride,
                     self.conv_1.padding)
        y = torch.cudnn_convolution_add_relu(skip, w[:, c:].contiguous(memory_format=torch.channels_last), z, 1.0,
                                             self.conv_1.bias, list(self.conv_1.stride), list(self.conv_1.padding),
                                             list(self.conv_1.dilation), self.conv_1.groups)
        return _conv_relu(self.conv_2, y)


def pad_same_stride2(x: torch.Tensor) -> torch.Tensor:
    """TF/Flax ``SAME`` padding of a 2×2 stride-2 window: an odd extent gets one
    trailing row/column, an even one none."""
    ph, pw = x.shape[-2] % 2, x.shape[-1] % 2
    return F.pad(x, (0, pw, 0, ph)) if (ph or pw) else x


class ResidualUNet(nn.Module):
    """U-Net residual corrector; NCHW in and out (``channels_last`` memory preferred)."""

    def __init__(self, *, input_channels: int, depth: int, channels: Sequence[int], activation: str = "relu",
                 kernel_size: int = 3, output_channels: int = 3) -> None:
        super().__init__()
        if depth < 1:
            raise ValueError("U-Net depth must be positive.")
        if len(channels) < depth:
            raise ValueError("The channel list must contain at least one value per U-Net depth.")
        if kernel_size < 1 or kernel_size % 2 == 0:
            raise ValueError("The convolution kernel size must be a positive odd integer.")
        widths = [int(c) for c in channels[:depth]]
        self.widths = tuple(widths)
        self.depth = depth
        self.encoders = nn.ModuleList()
        self.downsample = nn.ModuleList()
        cin = int(input_channels)
        for level, w in enumerate(widths):
            self.encoders.append(ConvPair(cin, w, kernel_size, activation))
            cin = w
            if level + 1 < depth:
                self.downsample.append(nn.Conv2d(w, widths[level + 1], kernel_size=2, stride=2))
                cin = widths[level + 1]
        self.upsample = nn.ModuleList()
        self.decoders = nn.ModuleList()
        for w in reversed(widths[:-1]):
            self.upsample.append(nn.ConvTranspose2d(cin, w, kernel_size=2, stride=2))
            self.decoders.append(ConvPair(2 * w, w, kernel_size, activation))
            cin = w
        self.residual_head = nn.Conv2d(cin, int(output_channels), kernel_size=1)
        nn.init.zeros_(self.residual_head.weight)
        nn.init.zeros_(self.residual_head.bias)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        skips = []
        for level, enc in enumerate(self.encoders):
            x = enc(x)
            skips.append(x)
            if level + 1 < self.depth:
                x = conv_bias_act(self.downsample[level], pad_same_stride2(x), False)
        for up, dec, skip in zip(self.upsample, self.decoders, reversed(skips[:-1])):
            x = conv_bias_act(up, x, False)
            if x.shape[-2:] != skip.shape[-2:]:
                x = F.interpolate(x, size=skip.shape[-2:], mode="bilinear", align_corners=False)
            if dec.relu and _fused_ok(x) and _fused_ok(skip):
                x = dec.forward_split(x, skip)
            else:
                x = dec(torch.cat((x, skip), dim=1))
        return conv_bias_act(self.residual_head, x, False)


def count_parameters(model: nn.Module) -> int:
    return sum(p.numel() for p in model.parameters() if p.requires_grad)


def corrector_4level(input_channels: int = 5, output_channels: int = 1) -> ResidualUNet:
    """The 4-level (32, 64, 128, 256) corrector on (h, hu, hv, z, rain) -> depth."""
    return ResidualUNet(input_channels=input_channels, depth=4, channels=(32, 64, 128, 256),
                        output_channels=output_channels)
