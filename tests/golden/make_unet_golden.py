"""Generate ``unet_d3_odd.npz`` from the UNMODIFIED reference residual U-Net.

Run in a container where the reference project is mounted (it is not needed,
and not read, anywhere else):

    python tests/golden/make_unet_golden.py --reference /root/reference

It imports ``TorchResidualUNet`` from the reference's
``src/hybrid_flood/benchmark/pytorch_residual_net.py`` (PyTorch only), builds
a depth-3 (4, 8, 16), 6-in / 3-out network (the reference tests' layer plan,
narrowed to keep the fixture small), fills every parameter from a seeded
normal draw (the reference zero-initialises the head,
which would make the output trivially zero), and saves the parameters, an
odd-sized input batch (2 x 6 x 37 x 45, so the SAME padding and the bilinear
skip alignment are exercised) and the float32 CPU output.  It also records the
parameter count of the full (16, 32, 64) network, which the reference's tests
pin at 150,883.
"""

from __future__ import annotations

import argparse
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    args = ap.parse_args()
    sys.path.insert(0, str(pathlib.Path(args.reference) / "src"))
    import torch
    from hybrid_flood.benchmark.pytorch_residual_net import TorchResidualUNet, count_torch_parameters

    torch.manual_seed(0)
    full = TorchResidualUNet(input_channels=6, depth=3, channels=(16, 32, 64), output_channels=3)
    net = TorchResidualUNet(input_channels=6, depth=3, channels=(4, 8, 16), output_channels=3)
    gen = torch.Generator().manual_seed(1)
    with torch.no_grad():
        for p in net.parameters():
            p.copy_(torch.randn(p.shape, generator=gen) * 0.3)
    x = torch.randn((2, 6, 37, 45), generator=gen)
    with torch.no_grad():
        y = net(x)
    arrays = {f"param/{k}": v.numpy() for k, v in net.state_dict().items()}
    np.savez_compressed(HERE / "unet_d3_odd.npz", x=x.numpy(), y=y.numpy(),
                        n_params=np.int64(count_torch_parameters(net)),
                        n_params_16_32_64=np.int64(count_torch_parameters(full)), **arrays)
    print("unet_d3_odd.npz", count_torch_parameters(net), count_torch_parameters(full), float(y.abs().max()))


if __name__ == "__main__":
    main()
