"""The corrector with its bias+ReLU epilogue fused (swe_bias_act_nhwc, channels-last
CUDA tensors) against the same network through plain torch ops: forward values
and parameter gradients (TF32 off; float32 to 1e-4, bfloat16 to its precision)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _net(seed=0):
    from hybrid_flood_b200.unet import ResidualUNet

    torch.manual_seed(seed)
    net = ResidualUNet(input_channels=5, depth=3, channels=(8, 16, 32), output_channels=1)
    with torch.no_grad():
        for p in net.parameters():
            p.normal_(0, 0.2)
    return net


def test_fused_epilogue_matches_torch_ops_forward_and_backward(cuda_device, monkeypatch):
    # Both networks run channels-last, so their convolutions are the same cuDNN
    # calls and give the same pre-activations; only the epilogue differs (the
    # reference's runs as torch ops).  With different convolution layouts an
    # activation within rounding of zero can fall on either side of the ReLU,
    # which moves a weight gradient by far more than rounding.  Deterministic
    # cuDNN algorithms keep the weight gradients' summation order the same in
    # both (the default ones may add split partial sums in any order).
    from hybrid_flood_b200 import unet

    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    monkeypatch.setattr(torch.backends.cudnn, "deterministic", True)
    ref = _net().to(cuda_device, memory_format=torch.channels_last)
    fused = _net().to(cuda_device, memory_format=torch.channels_last)
    x = torch.randn(2, 5, 37, 45, device=cuda_device).contiguous(memory_format=torch.channels_last)
    with monkeypatch.context() as m:
        m.setattr(unet, "_fusable", lambda y: False)
        y_ref = ref(x)
    y = fused(x)
    torch.testing.assert_close(y, y_ref, rtol=1e-5, atol=1e-6)
    y_ref.square().mean().backward()
    y.square().mean().backward()
    for (n, a), (_, b) in zip(ref.named_parameters(), fused.named_parameters()):
        # Rounding of a sum of ~3000 products, well below the effect of a wrong
        # mask element or bias term (relative 1e-2 and more).
        atol = 1e-5 * float(a.grad.abs().max())
        torch.testing.assert_close(b.grad, a.grad, rtol=1e-3, atol=atol, msg=lambda m, n=n: f"{n}: {m}")


def test_fused_epilogue_bf16_and_odd_channels(cuda_device):
    from hybrid_flood_b200 import _lib
    from hybrid_flood_b200.solver import _ptr, _stream

    ref = _net(1).to(cuda_device)
    fused = _net(1).to(cuda_device, dtype=torch.bfloat16, memory_format=torch.channels_last)
    x = torch.randn(2, 5, 64, 64, device=cuda_device)
    with torch.no_grad():
        y = fused(x.to(torch.bfloat16).contiguous(memory_format=torch.channels_last)).float()
        y_ref = ref(x)
    assert float((y - y_ref).norm() / y_ref.norm()) < 3e-2
    # the kernel alone: odd channel count (scalar path) and a multiple of 8 (vector path), in place
    lib = _lib.load()
    for c, dt in ((3, torch.bfloat16), (16, torch.bfloat16), (5, torch.float32)):
        t = torch.randn(2, c, 7, 9, device=cuda_device).to(dt).contiguous(memory_format=torch.channels_last)
        b = torch.randn(c, device=cuda_device)
        want = torch.relu(t.float() + b.view(1, -1, 1, 1))
        rc = lib.swe_bias_act_nhwc(_ptr(t), t.numel(), c, _ptr(b), 1, int(dt == torch.bfloat16), cuda_device.index,
                                   _stream(cuda_device))
        assert rc == 0
        torch.testing.assert_close(t.float(), want, rtol=1e-2 if dt == torch.bfloat16 else 1e-6, atol=1e-2)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_cudnn_fused_inference_matches_the_separate_epilogue(cuda_device, dtype):
    """Inference through cuDNN's fused convolution + bias + ReLU, with the decoder's
    skip concatenation replaced by two convolutions on the split weight summed
    inside the fused call, equals the path with the separate epilogue pass."""
    from hybrid_flood_b200 import unet

    torch.backends.cudnn.allow_tf32 = False
    net = _net(2).to(cuda_device, dtype=dtype, memory_format=torch.channels_last).eval()
    x = torch.randn(3, 5, 40, 52, device=cuda_device).to(dtype).contiguous(memory_format=torch.channels_last)
    with torch.no_grad():
        unet._FUSED["on"] = False
        want = net(x).float()
        unet._FUSED["on"] = True
        got = net(x).float()
    rel = float((got - want).norm() / want.norm())
    assert rel < (1e-5 if dtype == torch.float32 else 2e-2), rel
